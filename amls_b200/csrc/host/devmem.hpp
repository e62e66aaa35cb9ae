// Device memory helpers: RAII buffers on the stream-ordered allocator and a
// byte blob for descriptor tables (built on the host, uploaded in one copy).
#pragma once
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "amls_b200.h"
#include "host/status.hpp"

namespace amls_b200 {

inline void cudaCheck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const int code = (e == cudaErrorMemoryAllocation) ? AMLS_ERR_OOM : AMLS_ERR_CUDA;
    cudaGetLastError();  // clear sticky-free errors
    throw AmlsError(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// A device allocation owned by the handle (freed on reset/destruction).
class DevBuf {
public:
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        bytes_ = 0;
    }
    // ensure capacity (contents not preserved when growing)
    void* ensure(size_t bytes) {
        if (bytes <= bytes_ && p_) return p_;
        release();
        size_t b = bytes < 256 ? 256 : bytes;
        cudaCheck(cudaMalloc(&p_, b), "cudaMalloc");
        bytes_ = b;
        return p_;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p_); }
    size_t bytes() const { return bytes_; }

private:
    void* p_ = nullptr;
    size_t bytes_ = 0;
};

// Host-built table blob; add() returns a byte offset, dev<T>(off) the
// device pointer after upload().
class Blob {
public:
    template <class T>
    size_t add(const T* data, size_t count) {
        size_t off = (h_.size() + 15) & ~size_t(15);
        h_.resize(off + sizeof(T) * count);
        if (count) std::memcpy(h_.data() + off, data, sizeof(T) * count);
        return off;
    }
    template <class T>
    size_t add(const std::vector<T>& v) { return add(v.data(), v.size()); }
    void clear() { h_.clear(); }
    void upload(DevBuf& buf, cudaStream_t s) {
        buf.ensure(h_.size() + 16);
        if (!h_.empty())
            cudaCheck(cudaMemcpyAsync(buf.as<char>(), h_.data(), h_.size(), cudaMemcpyHostToDevice, s),
                      "blob upload");
        base_ = buf.as<char>();
    }
    template <class T>
    T* dev(size_t off) const { return reinterpret_cast<T*>(base_ + off); }
    size_t size() const { return h_.size(); }

private:
    std::vector<char> h_;
    char* base_ = nullptr;
};

}  // namespace amls_b200
