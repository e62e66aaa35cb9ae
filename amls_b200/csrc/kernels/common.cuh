// Shared device helpers for the AMLS kernels (sm_100a, FP64).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "launch.hpp"

namespace amls_b200 {

__device__ __forceinline__ void setStatus(int* status, int code, int where) {
    if (status) {
        // first failure wins; where = node / matrix id
        if (atomicCAS(status, 0, code) == 0) status[1] = where;
    }
}

template <int N>
__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
    for (int o = N / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; `red` must hold at least blockDim.x/32 doubles.  All
// threads receive the result.
__device__ __forceinline__ double blockSum(double v, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warpSum<32>(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < nw) ? red[threadIdx.x] : 0.0;
    if (wid == 0) t = warpSum<32>(t);
    if (threadIdx.x == 0) red[0] = t;
    __syncthreads();
    t = red[0];
    __syncthreads();
    return t;
}

// Block-wide sum with one barrier: every warp reduces the per-warp partials
// itself (same order in every warp, so all threads get the same bits).
// `red` holds 64 doubles used alternately (parity flips per call); two calls
// in a row are safe because the second writes the other half and a third
// call's barrier follows the first call's reads.
__device__ __forceinline__ double blockSum1(double v, double* red, int& parity) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    double* r = red + 32 * parity;
    parity ^= 1;
    v = warpSum<32>(v);
    if (lane == 0) r[wid] = v;
    __syncthreads();
    return warpSum<32>(lane < nw ? r[lane] : 0.0);
}

__device__ __forceinline__ double blockMax(double v, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < nw) ? red[threadIdx.x] : 0.0;
    if (wid == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
    }
    if (threadIdx.x == 0) red[0] = t;
    __syncthreads();
    t = red[0];
    __syncthreads();
    return t;
}

}  // namespace amls_b200
