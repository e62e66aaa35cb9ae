// Data-movement kernels of the AMLS pipeline: front assembly scatter,
// symmetrisation, batched transposes, row-segment gathers, M-norms and the
// final un-permutation.  All HBM-bound: grid-stride loops sized to the SM
// count, coalesced on the contiguous side.
#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
int gridFor(int64_t work, int threads) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int64_t g = (work + threads - 1) / threads;
    const int64_t cap = (int64_t)sms * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}
}  // namespace

__global__ void zeroKernel(double* __restrict__ p, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = 0.0;
}

cudaError_t launchZero(double* p, int64_t count, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    zeroKernel<<<gridFor(count, 256), 256, 0, s>>>(p, count);
    return cudaGetLastError();
}

// Each CSR entry has at most one destination in the front pools (its
// column's owner front); destinations are distinct, so a plain store-add.
__global__ void scatterAddKernel(const double* __restrict__ vals, const int64_t* __restrict__ dst,
                                 int64_t nnz, double scale, double* __restrict__ pool) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = dst[e];
        if (o >= 0) pool[o] += scale * vals[e];
    }
}

cudaError_t launchScatterAdd(const double* vals, const int64_t* dst, int64_t nnz, double scale,
                             double* pool, cudaStream_t s) {
    if (nnz <= 0) return cudaSuccess;
    scatterAddKernel<<<gridFor(nnz, 256), 256, 0, s>>>(vals, dst, nnz, scale, pool);
    return cudaGetLastError();
}

// C[j + j*p] = w[j]
__global__ void setDiagonalKernel(double* __restrict__ C, const double* __restrict__ w, int64_t p) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < p;
         j += (int64_t)gridDim.x * blockDim.x)
        C[j + j * p] = w[j];
}

cudaError_t launchSetDiagonal(double* C, const double* w, int64_t p, cudaStream_t s) {
    if (p <= 0) return cudaSuccess;
    setDiagonalKernel<<<gridFor(p, 256), 256, 0, s>>>(C, w, p);
    return cudaGetLastError();
}

// A = (A + A^T) / 2 on the leading n x n block of each front (one CTA per
// front, 32x32 tile pairs through shared memory).
__global__ void symmetrizeKernel(const FrontDesc* __restrict__ descs) {
    __shared__ double t1[32][33], t2[32][33];
    const FrontDesc F = descs[blockIdx.x];
    const int n = F.n;
    const int nt = (n + 31) / 32;
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 32 x 8
    for (int bj = 0; bj < nt; ++bj)
        for (int bi = bj; bi < nt; ++bi) {
            // tile (bi, bj) and its mirror (bj, bi)
            for (int r = ty; r < 32; r += 8) {
                const int gi = bi * 32 + tx, gj = bj * 32 + r;
                t1[r][tx] = (gi < n && gj < n) ? F.F[gi + (int64_t)gj * F.ld] : 0.0;
                const int hi = bj * 32 + tx, hj = bi * 32 + r;
                t2[r][tx] = (hi < n && hj < n) ? F.F[hi + (int64_t)hj * F.ld] : 0.0;
            }
            __syncthreads();
            for (int r = ty; r < 32; r += 8) {
                const int gi = bi * 32 + tx, gj = bj * 32 + r;
                // element (gi, gj) pairs with (gj, gi) = t2[tx][r]
                const double avg = 0.5 * (t1[r][tx] + t2[tx][r]);
                if (gi < n && gj < n) F.F[gi + (int64_t)gj * F.ld] = avg;
                const int hi = bj * 32 + tx, hj = bi * 32 + r;
                if (hi < n && hj < n) F.F[hi + (int64_t)hj * F.ld] = 0.5 * (t2[r][tx] + t1[tx][r]);
            }
            __syncthreads();
        }
}

cudaError_t launchSymmetrize(const FrontDesc* d, int nDesc, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    symmetrizeKernel<<<nDesc, 256, 0, s>>>(d);
    return cudaGetLastError();
}

// out (c x r) = in (r x c)^T, tiles of 32x32 listed in `tiles` (m0 = row
// tile of in, n0 = column tile of in).
__global__ void transposeKernel(const CopyDesc* __restrict__ descs, const TileRef* __restrict__ tiles) {
    __shared__ double t[32][33];
    const TileRef tr = tiles[blockIdx.x];
    const CopyDesc D = descs[tr.desc];
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
    for (int r = ty; r < 32; r += 8) {
        const int i = tr.m0 + tx, j = tr.n0 + r;
        t[r][tx] = (i < D.r && j < D.c) ? D.in[i + (int64_t)j * D.ldin] : 0.0;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int j = tr.n0 + tx, i = tr.m0 + r;   // out(j, i)
        if (i < D.r && j < D.c) D.out[j + (int64_t)i * D.ldout] = t[tx][r];
    }
}

cudaError_t launchTransposeBatched(const CopyDesc* d, const TileRef* tiles, int nTiles,
                                   cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    transposeKernel<<<nTiles, 256, 0, s>>>(d, tiles);
    return cudaGetLastError();
}

// Contiguous segment copies: out[dstOff[g] + t] = in[srcOff[g] + t], t < len[g]
// (one CTA per segment).
__global__ void gatherSegKernel(const double* __restrict__ in, const int64_t* __restrict__ srcOff,
                                double* __restrict__ out, const int64_t* __restrict__ dstOff,
                                const int32_t* __restrict__ len) {
    const int g = blockIdx.x;
    const int L = len[g];
    const double* src = in + srcOff[g];
    double* dst = out + dstOff[g];
    for (int t = threadIdx.x; t < L; t += blockDim.x) dst[t] = src[t];
}

cudaError_t launchGatherRows(const double* in, const int64_t* srcOff, double* out,
                             const int64_t* dstOff, const int32_t* len, int nSeg,
                             cudaStream_t s) {
    if (nSeg <= 0) return cudaSuccess;
    gatherSegKernel<<<nSeg, 128, 0, s>>>(in, srcOff, out, dstOff, len);
    return cudaGetLastError();
}

// norms[j] = sum_d x[d,j] * sum_{c in row d} M[d,c] x[c,j] over the original
// M (CSR), with x[o, j] = zt[j + inv[o]*m] (zt in permuted order)
// one warp per row d at a time; each thread keeps partial sums for columns
// j = lane + 32*t (t < 16, m <= 512 per pass), flushed by atomics per CTA.
__global__ void __launch_bounds__(256) mnormKernel(const int64_t* __restrict__ rp,
                                                   const int32_t* __restrict__ ci,
                                                   const double* __restrict__ v, int64_t n,
                                                   const int64_t* __restrict__ inv,
                                                   const double* __restrict__ zt, int64_t ldz,
                                                   int m, int j0, double* __restrict__ norms) {
    constexpr int T = 16;
    __shared__ double part[8][T * 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double acc[T];
#pragma unroll
    for (int t = 0; t < T; ++t) acc[t] = 0.0;
    const int64_t gw = blockIdx.x * 8 + wid, GW = (int64_t)gridDim.x * 8;
    for (int64_t d = gw; d < n; d += GW) {
        double row[T];
#pragma unroll
        for (int t = 0; t < T; ++t) row[t] = 0.0;
        for (int64_t e = rp[d]; e < rp[d + 1]; ++e) {
            const double a = v[e];
            const double* zc = zt + inv[ci[e]] * ldz;
#pragma unroll
            for (int t = 0; t < T; ++t) {
                const int j = j0 + lane + 32 * t;
                if (j < m) row[t] = fma(a, zc[j], row[t]);
            }
        }
        const double* zd = zt + inv[d] * ldz;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            const int j = j0 + lane + 32 * t;
            if (j < m) acc[t] = fma(zd[j], row[t], acc[t]);
        }
    }
#pragma unroll
    for (int t = 0; t < T; ++t) part[wid][lane + 32 * t] = acc[t];
    __syncthreads();
    for (int q = threadIdx.x; q < T * 32; q += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += part[w][q];
        const int j = j0 + q;
        if (j < m) atomicAdd(norms + j, s);
    }
}

cudaError_t launchMNorm(const int64_t* rp, const int32_t* ci, const double* v, int64_t n,
                        const int64_t* inv, const double* zt, int64_t ldz, int m, double* norms,
                        cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(norms, 0, sizeof(double) * (size_t)m, s);
    if (e != cudaSuccess) return e;
    for (int j0 = 0; j0 < m; j0 += 512) {
        mnormKernel<<<gridFor(n * 32, 256), 256, 0, s>>>(rp, ci, v, n, inv, zt, ldz, m, j0, norms);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Z[perm[d] + j*n] = zt[j + d*ldz] / sqrt(norms[j]); 32 x 32 tiles (d, j).
__global__ void unpermuteKernel(const double* __restrict__ zt, int64_t ldz, int m, int64_t n,
                                const int64_t* __restrict__ perm, const double* __restrict__ norms,
                                double* __restrict__ Z) {
    __shared__ double t[32][33];
    const int64_t d0 = (int64_t)blockIdx.x * 32;
    const int j0 = blockIdx.y * 32;
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
    for (int r = ty; r < 32; r += 8) {
        const int64_t d = d0 + r;
        const int j = j0 + tx;
        t[r][tx] = (d < n && j < m) ? zt[j + d * ldz] : 0.0;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int j = j0 + r;
        const int64_t d = d0 + tx;
        if (d < n && j < m) {
            const double s = 1.0 / sqrt(fmax(norms[j], 1e-300));
            Z[perm[d] + (int64_t)j * n] = t[tx][r] * s;
        }
    }
}

cudaError_t launchUnpermute(const double* zt, int64_t ldz, int m, int64_t n, const int64_t* perm,
                            const double* norms, double* Z, cudaStream_t s) {
    if (n <= 0 || m <= 0) return cudaSuccess;
    dim3 grid((unsigned)((n + 31) / 32), (unsigned)((m + 31) / 32));
    unpermuteKernel<<<grid, 256, 0, s>>>(zt, ldz, m, n, perm, norms, Z);
    return cudaGetLastError();
}

__global__ void reciprocalKernel(const double* __restrict__ in, double* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = 1.0 / in[i];
}

cudaError_t launchReciprocal(const double* in, double* out, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    reciprocalKernel<<<(n + 255) / 256, 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}

// SpMM in the transposed layout: for every permuted row d (original row
// o = perm[d]) Rt[:, d] = sum_e M[o, c_e] * Qt[:, inv[c_e]], with Qt and Rt
// m x n column-major (ld = m): one CTA per row at a time, the row's
// (value, column) pairs staged in shared memory, threads over the m
// contiguous entries of each referenced column.
__global__ void __launch_bounds__(128) spmmTKernel(const int64_t* __restrict__ rp,
                                                   const int32_t* __restrict__ ci,
                                                   const double* __restrict__ v, int64_t n,
                                                   const int64_t* __restrict__ perm,
                                                   const int64_t* __restrict__ inv,
                                                   const double* __restrict__ Qt, int m,
                                                   double* __restrict__ Rt) {
    constexpr int kStage = 512;
    __shared__ double sv[kStage];
    __shared__ int64_t sc[kStage];
    for (int64_t d = blockIdx.x; d < n; d += gridDim.x) {
        const int64_t o = perm[d];
        const int64_t e0 = rp[o], e1 = rp[o + 1];
        for (int j0 = 0; j0 < m; j0 += 4 * 128) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int64_t eb = e0; eb < e1; eb += kStage) {
                const int cnt = (int)((e1 - eb) < kStage ? (e1 - eb) : kStage);
                __syncthreads();
                for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
                    sv[t] = v[eb + t];
                    sc[t] = inv[ci[eb + t]] * (int64_t)m;
                }
                __syncthreads();
                for (int t = 0; t < cnt; ++t) {
                    const double a = sv[t];
                    const double* q = Qt + sc[t];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int j = j0 + threadIdx.x + 128 * u;
                        if (j < m) acc[u] = fma(a, q[j], acc[u]);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = j0 + threadIdx.x + 128 * u;
                if (j < m) Rt[j + d * (int64_t)m] = acc[u];
            }
        }
    }
}

cudaError_t launchSpmmT(const int64_t* rp, const int32_t* ci, const double* v, int64_t n,
                        const int64_t* perm, const int64_t* inv, const double* Qt, int m,
                        double* Rt, cudaStream_t s) {
    if (n <= 0 || m <= 0) return cudaSuccess;
    spmmTKernel<<<gridFor(n * 128, 128), 128, 0, s>>>(rp, ci, v, n, perm, inv, Qt, m, Rt);
    return cudaGetLastError();
}

// The same product over row groups: consecutive original rows grp[g] ..
// grp[g+1]-1 (at most kSpmmGroup) share one column pattern, as the DOFs of
// one mesh node do, so every gathered column of Qt (m doubles from L2) feeds
// all rows of the group.  One CTA per group, thread t owns columns
// j0 + t + 256 u (u < U).
template <int U>
__global__ void __launch_bounds__(256) spmmGroupKernel(const int64_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci,
                                                       const double* __restrict__ v, int64_t ngrp,
                                                       const int64_t* __restrict__ grp,
                                                       const int64_t* __restrict__ inv,
                                                       const double* __restrict__ Qt, int m,
                                                       int64_t ld, double* __restrict__ Rt) {
    constexpr int kStage = 256;
    __shared__ double sv[kSpmmGroup][kStage];
    __shared__ int64_t sc[kStage];
    for (int64_t g = blockIdx.x; g < ngrp; g += gridDim.x) {
        const int64_t o0 = grp[g];
        const int G = (int)(grp[g + 1] - o0);
        const int64_t cnt = rp[o0 + 1] - rp[o0];
        for (int j0 = 0; j0 < m; j0 += 256 * U) {
            double acc[kSpmmGroup][U];
#pragma unroll
            for (int r = 0; r < kSpmmGroup; ++r)
#pragma unroll
                for (int u = 0; u < U; ++u) acc[r][u] = 0.0;
            for (int64_t eb = 0; eb < cnt; eb += kStage) {
                const int c = (int)((cnt - eb) < kStage ? (cnt - eb) : kStage);
                __syncthreads();
                for (int t = threadIdx.x; t < c; t += blockDim.x) {
                    sc[t] = inv[ci[rp[o0] + eb + t]] * ld;
                    for (int r = 0; r < G; ++r) sv[r][t] = v[rp[o0 + r] + eb + t];
                }
                __syncthreads();
#pragma unroll 2
                for (int t = 0; t < c; ++t) {
                    const double* q = Qt + sc[t];
                    double x[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int j = j0 + threadIdx.x + 256 * u;
                        x[u] = j < m ? q[j] : 0.0;
                    }
#pragma unroll
                    for (int r = 0; r < kSpmmGroup; ++r)
                        if (r < G) {
                            const double a = sv[r][t];
#pragma unroll
                            for (int u = 0; u < U; ++u) acc[r][u] = fma(a, x[u], acc[r][u]);
                        }
                }
            }
#pragma unroll
            for (int r = 0; r < kSpmmGroup; ++r)
                if (r < G) {
                    double* out = Rt + inv[o0 + r] * ld;
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int j = j0 + threadIdx.x + 256 * u;
                        if (j < m) out[j] = acc[r][u];
                    }
                }
        }
    }
}

cudaError_t launchSpmmGroupT(const int64_t* rp, const int32_t* ci, const double* v, int64_t ngrp,
                             const int64_t* grp, const int64_t* inv, const double* Qt, int m,
                             int64_t ld, double* Rt, cudaStream_t s) {
    if (ngrp <= 0 || m <= 0) return cudaSuccess;
    const int grid = gridFor(ngrp * 256, 256);
    const int u = (m + 255) / 256;
    if (u <= 1)
        spmmGroupKernel<1><<<grid, 256, 0, s>>>(rp, ci, v, ngrp, grp, inv, Qt, m, ld, Rt);
    else if (u == 2)
        spmmGroupKernel<2><<<grid, 256, 0, s>>>(rp, ci, v, ngrp, grp, inv, Qt, m, ld, Rt);
    else if (u == 3)
        spmmGroupKernel<3><<<grid, 256, 0, s>>>(rp, ci, v, ngrp, grp, inv, Qt, m, ld, Rt);
    else
        spmmGroupKernel<4><<<grid, 256, 0, s>>>(rp, ci, v, ngrp, grp, inv, Qt, m, ld, Rt);
    return cudaGetLastError();
}

// out = a*x + b*y (+ c*z when z is given), elementwise
__global__ void axpby3Kernel(int64_t n, double a, const double* __restrict__ x, double b,
                             const double* __restrict__ y, double c, const double* __restrict__ z,
                             double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double v = a * x[i] + b * y[i];
        if (z) v += c * z[i];
        out[i] = v;
    }
}

cudaError_t launchAxpby3(int64_t n, double a, const double* x, double b, const double* y,
                         double c, const double* z, double* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    axpby3Kernel<<<gridFor(n, 256), 256, 0, s>>>(n, a, x, b, y, c, z, out);
    return cudaGetLastError();
}

// A = (A + A^T) / 2 on the leading n x n block of each descriptor, one CTA
// per 32x32 tile pair (TileRef: desc, m0 = bi, n0 = bj, bi >= bj).
__global__ void symmetrizeTilesKernel(const FrontDesc* __restrict__ descs,
                                      const TileRef* __restrict__ tiles) {
    __shared__ double t1[32][33], t2[32][33];
    const TileRef tr = tiles[blockIdx.x];
    const FrontDesc F = descs[tr.desc];
    const int n = F.n, bi = tr.m0, bj = tr.n0;
    const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
    for (int r = ty; r < 32; r += 8) {
        const int gi = bi * 32 + tx, gj = bj * 32 + r;
        t1[r][tx] = (gi < n && gj < n) ? F.F[gi + (int64_t)gj * F.ld] : 0.0;
        const int hi = bj * 32 + tx, hj = bi * 32 + r;
        t2[r][tx] = (hi < n && hj < n) ? F.F[hi + (int64_t)hj * F.ld] : 0.0;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int gi = bi * 32 + tx, gj = bj * 32 + r;
        if (gi < n && gj < n) F.F[gi + (int64_t)gj * F.ld] = 0.5 * (t1[r][tx] + t2[tx][r]);
        const int hi = bj * 32 + tx, hj = bi * 32 + r;
        if (hi < n && hj < n) F.F[hi + (int64_t)hj * F.ld] = 0.5 * (t2[r][tx] + t1[tx][r]);
    }
}

cudaError_t launchSymmetrizeTiles(const FrontDesc* d, const TileRef* tiles, int nTiles,
                                  cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    symmetrizeTilesKernel<<<nTiles, 256, 0, s>>>(d, tiles);
    return cudaGetLastError();
}

}  // namespace amls_b200
