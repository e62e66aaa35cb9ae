// Data-movement kernels of the AMLS pipeline: front assembly scatter,
// symmetrisation, batched transposes, the products
// with M over super-rows (and the M-norms fused into them) and the final
// un-permutation.  Memory-bound (HBM or L2): grid-stride loops sized to the
// SM count, coalesced on the contiguous side.
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

// Z[perm[d] + j*n] = zt[j + d*ldz] / sqrt(norms[j]); 32 x 32 tiles (d, j).
__global__ void unpermuteKernel(const double* __restrict__ zt, int64_t ldz, int m, int64_t n,
                                const int64_t* __restrict__ perm, const double* __restrict__ norms,
                                double* __restrict__ Z, const int32_t* __restrict__ pencil) {
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
            const double nj = norms[(pencil ? (int64_t)pencil[d] * m : 0) + j];
            // a pencil with fewer eigenpairs than m has zero columns there
            const double s = nj > 0.0 ? 1.0 / sqrt(nj) : 0.0;
            Z[perm[d] + (int64_t)j * n] = t[tx][r] * s;
        }
    }
}

cudaError_t launchUnpermute(const double* zt, int64_t ldz, int m, int64_t n, const int64_t* perm,
                            const double* norms, double* Z, cudaStream_t s, const int32_t* pencil) {
    if (n <= 0 || m <= 0) return cudaSuccess;
    dim3 grid((unsigned)((n + 31) / 32), (unsigned)((m + 31) / 32));
    unpermuteKernel<<<grid, 256, 0, s>>>(zt, ldz, m, n, perm, norms, Z, pencil);
    return cudaGetLastError();
}

// Sparse products with M in the transposed layout, over super-rows: up to
// kSpmmSuperRows consecutive original rows (the DOFs of a few neighbouring
// mesh nodes) whose column patterns mostly overlap, stored as one dense
// block over the union of their patterns (vals[t * kSpmmSuperRows + r] for
// union column t, row r; zeros where a row has no entry).  Every gathered
// column of Qt (m contiguous doubles: Qt[j + inv[c] * ld]) then feeds all
// rows of the super-row from registers, so the gathers, which bound the
// product (a column is referenced once per neighbouring node), drop by the
// pattern overlap.  One CTA of kSpmmThreads per super-row at a time; thread
// t owns columns j0 + t + kSpmmThreads u (u < U).
namespace {
constexpr int kSpmmThreads = 128;
constexpr int kSpmmStage = 128;

template <int U, bool DOT>
__device__ __forceinline__ void superRow(const SpmmSuper& S, const int32_t* __restrict__ ucols,
                                         const double* __restrict__ vals, const int64_t* __restrict__ inv,
                                         const double* __restrict__ Qt, int m, int64_t ld, int j0,
                                         double* __restrict__ Rt, double* __restrict__ Rt2, double (&dot)[U],
                                         double* sv, int64_t* sc) {
    constexpr int R = kSpmmSuperRows;
    double acc[R][U];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int u = 0; u < U; ++u) acc[r][u] = 0.0;
    const int32_t* cols = ucols + S.colOff;
    const double* blk = vals + S.valOff;
    for (int eb = 0; eb < S.len; eb += kSpmmStage) {
        const int c = (S.len - eb) < kSpmmStage ? (S.len - eb) : kSpmmStage;
        __syncthreads();
        for (int i = threadIdx.x; i < c * R; i += kSpmmThreads) sv[i] = blk[(int64_t)eb * R + i];
        for (int t = threadIdx.x; t < c; t += kSpmmThreads) sc[t] = inv[cols[eb + t]] * ld;
        __syncthreads();
#pragma unroll 4
        for (int t = 0; t < c; ++t) {
            const double* q = Qt + sc[t];
            double x[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = j0 + threadIdx.x + kSpmmThreads * u;
                x[u] = j < m ? q[j] : 0.0;
            }
            const double2* a2 = reinterpret_cast<const double2*>(sv + t * R);
#pragma unroll
            for (int r2 = 0; r2 < R / 2; ++r2) {
                const double2 a = a2[r2];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    acc[2 * r2][u] = fma(a.x, x[u], acc[2 * r2][u]);
                    acc[2 * r2 + 1][u] = fma(a.y, x[u], acc[2 * r2 + 1][u]);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (r < S.rows) {
            const int64_t o = inv[S.row0 + r] * ld;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = j0 + threadIdx.x + kSpmmThreads * u;
                if (j < m) {
                    if (DOT) dot[u] = fma(Qt[o + j], acc[r][u], dot[u]);
                    else {
                        Rt[o + j] = acc[r][u];
                        if (Rt2) Rt2[o + j] = acc[r][u];
                    }
                }
            }
        }
}
}  // namespace

template <int U>
__global__ void __launch_bounds__(kSpmmThreads) spmmSuperKernel(const SpmmSuper* __restrict__ sup, int64_t nsup,
                                                                const int32_t* __restrict__ ucols,
                                                                const double* __restrict__ vals,
                                                                const int64_t* __restrict__ inv,
                                                                const double* __restrict__ Qt, int m, int64_t ld,
                                                                double* __restrict__ Rt, double* __restrict__ Rt2) {
    __shared__ __align__(16) double sv[kSpmmStage * kSpmmSuperRows];
    __shared__ int64_t sc[kSpmmStage];
    double dot[U];
    for (int64_t g = blockIdx.x; g < nsup; g += gridDim.x) {
        const SpmmSuper S = sup[g];
        for (int j0 = 0; j0 < m; j0 += kSpmmThreads * U)
            superRow<U, false>(S, ucols, vals, inv, Qt, m, ld, j0, Rt, Rt2, dot, sv, sc);
    }
}

// norms[j] += sum over the super-row's rows o of x[o, j] (M x)[o, j]; the
// j chunk is blockIdx.y, one atomic per thread and column at the end
template <int U>
__global__ void __launch_bounds__(kSpmmThreads) mnormSuperKernel(const SpmmSuper* __restrict__ sup, int64_t nsup,
                                                                 const int32_t* __restrict__ ucols,
                                                                 const double* __restrict__ vals,
                                                                 const int64_t* __restrict__ inv,
                                                                 const double* __restrict__ zt, int m, int64_t ld,
                                                                 double* __restrict__ norms) {
    __shared__ __align__(16) double sv[kSpmmStage * kSpmmSuperRows];
    __shared__ int64_t sc[kSpmmStage];
    const int j0 = blockIdx.y * kSpmmThreads * U;
    double dot[U];
#pragma unroll
    for (int u = 0; u < U; ++u) dot[u] = 0.0;
    int cur = -1;                       // pencil of the sums in dot[]
    auto flush = [&]() {
        if (cur < 0) return;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = j0 + threadIdx.x + kSpmmThreads * u;
            if (j < m) atomicAdd(norms + (int64_t)cur * m + j, dot[u]);
            dot[u] = 0.0;
        }
    };
    for (int64_t g = blockIdx.x; g < nsup; g += gridDim.x) {
        const int pc = sup[g].pencil;   // uniform over the CTA
        if (pc != cur) {
            flush();
            cur = pc;
        }
        superRow<U, true>(sup[g], ucols, vals, inv, zt, m, ld, j0, nullptr, nullptr, dot, sv, sc);
    }
    flush();
}

namespace {
// columns per thread: the smallest of 2, 4, 6, 8 covering m (8 beyond 1024)
int spmmU(int m) {
    const int u = (m + kSpmmThreads - 1) / kSpmmThreads;
    return u <= 2 ? 2 : u <= 4 ? 4 : u <= 6 ? 6 : 8;
}
}  // namespace

cudaError_t launchSpmmSuperT(const SpmmSuper* sup, int64_t nsup, const int32_t* ucols, const double* vals,
                             const int64_t* inv, const double* Qt, int m, int64_t ld, double* Rt,
                             cudaStream_t s, double* Rt2) {
    if (nsup <= 0 || m <= 0) return cudaSuccess;
    const int grid = gridFor(nsup * kSpmmThreads, kSpmmThreads);
    switch (spmmU(m)) {
        case 2: spmmSuperKernel<2><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, Qt, m, ld, Rt, Rt2); break;
        case 4: spmmSuperKernel<4><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, Qt, m, ld, Rt, Rt2); break;
        case 6: spmmSuperKernel<6><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, Qt, m, ld, Rt, Rt2); break;
        default: spmmSuperKernel<8><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, Qt, m, ld, Rt, Rt2); break;
    }
    return cudaGetLastError();
}

cudaError_t launchMNormSuper(const SpmmSuper* sup, int64_t nsup, const int32_t* ucols, const double* vals,
                             const int64_t* inv, const double* zt, int m, int64_t ld, double* norms,
                             int pencils, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(norms, 0, sizeof(double) * (size_t)(m > 0 ? m : 0) * (size_t)pencils, s);
    if (e != cudaSuccess || nsup <= 0 || m <= 0) return e;
    const int u = spmmU(m);
    const dim3 grid(gridFor(nsup * kSpmmThreads, kSpmmThreads), (m + kSpmmThreads * u - 1) / (kSpmmThreads * u));
    switch (u) {
        case 2: mnormSuperKernel<2><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, zt, m, ld, norms); break;
        case 4: mnormSuperKernel<4><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, zt, m, ld, norms); break;
        case 6: mnormSuperKernel<6><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, zt, m, ld, norms); break;
        default: mnormSuperKernel<8><<<grid, kSpmmThreads, 0, s>>>(sup, nsup, ucols, vals, inv, zt, m, ld, norms); break;
    }
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

// A = (A + A^T) / 2 on the leading n x n block of each descriptor, or with
// MIRROR the strict upper triangle copied from the lower one (A[i,j] =
// A[j,i], i < j); one CTA per 32x32 tile pair (TileRef: desc, m0 = bi,
// n0 = bj, bi >= bj, in tile units).
template <bool MIRROR>
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
        if (!MIRROR) {
            const int hi = bj * 32 + tx, hj = bi * 32 + r;
            t2[r][tx] = (hi < n && hj < n) ? F.F[hi + (int64_t)hj * F.ld] : 0.0;
        }
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int hi = bj * 32 + tx, hj = bi * 32 + r;
        if (MIRROR) {
            if (hi < hj && hj < n) F.F[hi + (int64_t)hj * F.ld] = t1[tx][r];
        } else {
            const int gi = bi * 32 + tx, gj = bj * 32 + r;
            if (gi < n && gj < n) F.F[gi + (int64_t)gj * F.ld] = 0.5 * (t1[r][tx] + t2[tx][r]);
            if (hi < n && hj < n) F.F[hi + (int64_t)hj * F.ld] = 0.5 * (t2[r][tx] + t1[tx][r]);
        }
    }
}

cudaError_t launchSymmetrizeTiles(const FrontDesc* d, const TileRef* tiles, int nTiles,
                                  cudaStream_t s, bool mirror) {
    if (nTiles <= 0) return cudaSuccess;
    if (mirror) symmetrizeTilesKernel<true><<<nTiles, 256, 0, s>>>(d, tiles);
    else symmetrizeTilesKernel<false><<<nTiles, 256, 0, s>>>(d, tiles);
    return cudaGetLastError();
}

}  // namespace amls_b200
