// Separator worker process.  The METIS library keeps process-wide state (its
// random generator), so concurrent calls in one process interfere; the
// partitioner runs the independent halves of the recursive bisection in
// worker processes instead, each an instance of this program talking over a
// socket on stdin/stdout.
//
// Protocol (native byte order, the parent is on the same machine):
//   request:  int64 n, int64 nnz, int64 xadj[n + 1], int64 adjncy[nnz]
//   response: int64 status (METIS code), then int64 part[n] when status is 1
// The worker exits on end of input.
#include <unistd.h>

#include <cerrno>
#include <cstdint>
#include <vector>

#include "host/metis_call.hpp"

namespace {
bool readAll(int fd, void* p, size_t bytes, bool& eofAtStart) {
    char* c = static_cast<char*>(p);
    size_t got = 0;
    eofAtStart = false;
    while (got < bytes) {
        const ssize_t r = read(fd, c + got, bytes - got);
        if (r == 0) {
            eofAtStart = got == 0;
            return false;
        }
        if (r < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        got += static_cast<size_t>(r);
    }
    return true;
}
bool writeAll(int fd, const void* p, size_t bytes) {
    const char* c = static_cast<const char*>(p);
    size_t put = 0;
    while (put < bytes) {
        const ssize_t r = write(fd, c + put, bytes - put);
        if (r < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        put += static_cast<size_t>(r);
    }
    return true;
}
}  // namespace

int main() {
    std::vector<int64_t> xadj, adjncy, part;
    for (;;) {
        int64_t hdr[2];
        bool eof = false;
        if (!readAll(0, hdr, sizeof(hdr), eof)) return eof ? 0 : 1;
        const int64_t n = hdr[0], nnz = hdr[1];
        if (n < 0 || nnz < 0) return 1;
        xadj.resize(static_cast<size_t>(n) + 1);
        adjncy.resize(static_cast<size_t>(nnz) + 1);
        part.assign(static_cast<size_t>(n) + 1, 0);
        if (!readAll(0, xadj.data(), sizeof(int64_t) * (static_cast<size_t>(n) + 1), eof)) return 1;
        if (nnz > 0 && !readAll(0, adjncy.data(), sizeof(int64_t) * static_cast<size_t>(nnz), eof)) return 1;
        const int64_t status = n > 0 ? amls_b200::metisSeparator(n, xadj.data(), adjncy.data(), part.data())
                                     : amls_b200::kMetisOk;
        if (!writeAll(1, &status, sizeof(status))) return 1;
        if (status == amls_b200::kMetisOk && n > 0 &&
            !writeAll(1, part.data(), sizeof(int64_t) * static_cast<size_t>(n)))
            return 1;
    }
}
