// Adjacency graph of |K| + |M| for the nested dissection, on the GPU: for
// every vertex the merge of the sorted column lists of its K and M rows
// without the vertex itself (the graph the reference builds for METIS,
// src/partition/metis_partitioner.cpp:20-45, with sorted neighbour lists as
// its inducedSubgraph hands them over, :48-73).  One thread per vertex:
// a count pass, then (after the host's prefix sum) a fill pass.
#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
int graphGrid(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t g = (n + 255) / 256;
    return static_cast<int>(g < 8LL * sms ? g : 8LL * sms);
}

template <bool FILL>
__device__ __forceinline__ int64_t mergeRow(int64_t v, const int64_t* __restrict__ kp, const int32_t* __restrict__ kc,
                                            const int64_t* __restrict__ mp, const int32_t* __restrict__ mc,
                                            int64_t* __restrict__ out) {
    int64_t a = kp[v], ae = kp[v + 1], b = mp[v], be = mp[v + 1];
    int64_t cnt = 0, last = -1;
    while (a < ae || b < be) {
        int64_t c;
        if (b >= be || (a < ae && kc[a] <= mc[b])) c = kc[a++];
        else c = mc[b++];
        if (c == v || c == last) continue;
        if (FILL) out[cnt] = c;
        ++cnt;
        last = c;
    }
    return cnt;
}
}  // namespace

__global__ void graphCountKernel(int64_t n, const int64_t* __restrict__ kp, const int32_t* __restrict__ kc,
                                 const int64_t* __restrict__ mp, const int32_t* __restrict__ mc,
                                 int64_t* __restrict__ cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        cnt[v] = mergeRow<false>(v, kp, kc, mp, mc, nullptr);
}

__global__ void graphFillKernel(int64_t n, const int64_t* __restrict__ kp, const int32_t* __restrict__ kc,
                                const int64_t* __restrict__ mp, const int32_t* __restrict__ mc,
                                const int64_t* __restrict__ xadj, int64_t* __restrict__ adj) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        mergeRow<true>(v, kp, kc, mp, mc, adj + xadj[v]);
}

cudaError_t launchGraphCount(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp, const int32_t* mc,
                             int64_t* cnt, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    graphCountKernel<<<graphGrid(n), 256, 0, s>>>(n, kp, kc, mp, mc, cnt);
    return cudaGetLastError();
}

cudaError_t launchGraphFill(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp, const int32_t* mc,
                            const int64_t* xadj, int64_t* adj, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    graphFillKernel<<<graphGrid(n), 256, 0, s>>>(n, kp, kc, mp, mc, xadj, adj);
    return cudaGetLastError();
}

}  // namespace amls_b200
