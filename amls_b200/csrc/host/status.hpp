// Status codes and exception-to-code translation at the C ABI.
#pragma once
#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "amls_b200.h"

namespace amls_b200 {

void setLastError(const std::string& msg);
const char* lastError();

// An error carrying its C ABI status code.
struct AmlsError : std::runtime_error {
    int code;
    AmlsError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline int fail(int code, const std::string& msg) {
    setLastError(msg);
    return code;
}

// Run f, translating every exception into a status code (none crosses the ABI).
template <class F>
int guarded(F&& f) {
    try {
        setLastError("");
        return f();
    } catch (const AmlsError& e) {
        return fail(e.code, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(AMLS_ERR_INVALID_ARGUMENT, e.what());
    } catch (const std::bad_alloc& e) {
        return fail(AMLS_ERR_OOM, std::string("host allocation failed: ") + e.what());
    } catch (const std::exception& e) {
        const std::string m = e.what();
        if (m.rfind("METIS", 0) == 0) return fail(AMLS_ERR_PARTITION, m);
        return fail(AMLS_ERR_NUMERIC, m);
    } catch (...) {
        return fail(AMLS_ERR_NUMERIC, "unknown error");
    }
}

}  // namespace amls_b200
