// Batched FP64 GEMM with gather/scatter epilogues, and the front extend-add
// update (SYRK + SYR2K of the eliminated front, scattered into ancestors).
//
// B200 has no FP64 tcgen05 kind; FP64 runs on the DFMA pipe, so these are
// register-tiled CUDA-core kernels: 64x64 output tile per CTA, 256 threads,
// 4x4 accumulators per thread, K staged through shared memory in slices of
// 16 with register prefetch of the next slice (one barrier per slice).
// Thread (tx, ty) owns rows tx + 16*i and columns ty + 16*j so that the
// epilogue stores of a warp are contiguous in a column.
#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
constexpr int NT = 256;
constexpr int TM = 64, TN = 64, TK = 16;   // tiles of the front-update kernel

// Register-tiled batched GEMM: tile (16*RM) x (16*RN), K slice KS, thread
// (tx, ty) owns rows tx + 16*i and columns ty + 16*j.
template <int RM, int RN, int KS>
struct GemmTile {
    static constexpr int BM = 16 * RM, BN = 16 * RN;
    static constexpr int LA = BM * KS / NT, LB = BN * KS / NT;   // loads per thread

    __device__ static void loadA(const GemmDesc& D, int m0, int k0, int kEnd, double (&r)[LA]) {
#pragma unroll
        for (int u = 0; u < LA; ++u) {
            const int idx = threadIdx.x + NT * u;
            int i, k;
            if (D.flags & kTransA) { k = idx % KS; i = idx / KS; }
            else { i = idx % BM; k = idx / BM; }
            const int gi = m0 + i, gk = k0 + k;
            double v = 0.0;
            if (gi < D.M && gk < kEnd) {
                if (D.flags & kTransA) v = D.A[gk + (int64_t)gi * D.lda];
                else if (D.flags & kGatherA) v = D.A[gi + (int64_t)D.aMap[gk] * D.lda];
                else v = D.A[gi + (int64_t)gk * D.lda];
            }
            r[u] = v;
        }
    }
    __device__ static void storeA(const GemmDesc& D, const double (&r)[LA], double (*As)[BM + 2]) {
#pragma unroll
        for (int u = 0; u < LA; ++u) {
            const int idx = threadIdx.x + NT * u;
            int i, k;
            if (D.flags & kTransA) { k = idx % KS; i = idx / KS; }
            else { i = idx % BM; k = idx / BM; }
            As[k][i] = r[u];
        }
    }
    __device__ static void loadB(const GemmDesc& D, int n0, int k0, int kEnd, double (&r)[LB]) {
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int idx = threadIdx.x + NT * u;
            int j, k;
            if (D.flags & kTransB) { j = idx % BN; k = idx / BN; }
            else { k = idx % KS; j = idx / KS; }
            const int gj = n0 + j, gk = k0 + k;
            double v = 0.0;
            if (gj < D.N && gk < kEnd) {
                if (D.flags & kTransB) v = D.B[gj + (int64_t)gk * D.ldb];
                else v = D.B[gk + (int64_t)gj * D.ldb];
            }
            r[u] = v;
        }
    }
    __device__ static void storeB(const GemmDesc& D, const double (&r)[LB], double (*Bs)[BN + 2]) {
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int idx = threadIdx.x + NT * u;
            int j, k;
            if (D.flags & kTransB) { j = idx % BN; k = idx / BN; }
            else { k = idx % KS; j = idx / KS; }
            Bs[k][j] = r[u];
        }
    }
};

template <int RM, int RN, int KS>
__device__ __forceinline__ void gemmTileBody(const GemmDesc* __restrict__ descs,
                                             const TileRef* __restrict__ tiles) {
    using G = GemmTile<RM, RN, KS>;
    __shared__ double As[2][KS][G::BM + 2];
    __shared__ double Bs[2][KS][G::BN + 2];
    const TileRef t = tiles[blockIdx.x];
    const GemmDesc D = descs[t.desc];
    const int m0 = t.m0, n0 = t.n0;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[RM][RN];
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int j = 0; j < RN; ++j) acc[i][j] = 0.0;
    // split-K: this CTA covers k in [kBeg, kEnd) (the whole K when kChunk = 0);
    // triangular B: only k <= last column of the tile (kTriKUpTo) or
    // k >= first column of the tile (kTriKFrom) contribute
    int kBeg = D.kChunk > 0 ? t.pad * D.kChunk : 0;
    int kEnd = D.kChunk > 0 ? min(D.K, kBeg + D.kChunk) : D.K;
    if (D.flags & kTriKUpTo) kEnd = min(kEnd, n0 + G::BN);
    if (D.flags & kTriKFrom) kBeg = max(kBeg, n0);
    double ra[G::LA], rb[G::LB];
    int cur = 0;
    if (kEnd > kBeg) {
        G::loadA(D, m0, kBeg, kEnd, ra);
        G::loadB(D, n0, kBeg, kEnd, rb);
        G::storeA(D, ra, As[0]);
        G::storeB(D, rb, Bs[0]);
    }
    __syncthreads();
    for (int k0 = kBeg; k0 < kEnd; k0 += KS) {
        const bool more = k0 + KS < kEnd;
        if (more) {
            G::loadA(D, m0, k0 + KS, kEnd, ra);
            G::loadB(D, n0, k0 + KS, kEnd, rb);
        }
#pragma unroll
        for (int kk = 0; kk < KS; ++kk) {
            double a[RM], b[RN];
#pragma unroll
            for (int i = 0; i < RM; ++i) a[i] = As[cur][kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < RN; ++j) b[j] = Bs[cur][kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < RM; ++i)
#pragma unroll
                for (int j = 0; j < RN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (more) {
            G::storeA(D, ra, As[cur ^ 1]);
            G::storeB(D, rb, Bs[cur ^ 1]);
        }
        __syncthreads();
        cur ^= 1;
    }
    // epilogue
#pragma unroll
    for (int j = 0; j < RN; ++j) {
        const int col = n0 + ty + 16 * j;
        if (col >= D.N) continue;
        const double cs = (D.flags & kColScale) ? D.colScale[col] : 1.0;
#pragma unroll
        for (int i = 0; i < RM; ++i) {
            const int row = m0 + tx + 16 * i;
            if (row >= D.M) continue;
            double v = D.alpha * acc[i][j] * cs;
            if (D.flags & kRowScale) v *= D.rowScale[row];
            if (D.flags & kScatter) {
                double* dst = D.C + D.colOff[col] + D.rowIdx[row];
                if (D.flags & kAtomic) atomicAdd(dst, v);
                else if (D.flags & kAccumulate) *dst += v;
                else *dst = v;
            } else {
                double* dst = D.C + row + (int64_t)col * D.ldc;
                if (D.kChunk > 0) atomicAdd(dst, v);   // split-K partial (C pre-zeroed)
                else if (D.flags & kAccumulate) *dst = v + D.beta * (*dst);
                else *dst = v;
            }
        }
    }
}
}  // namespace

__global__ void __launch_bounds__(NT) gemmBatchedKernel(const GemmDesc* __restrict__ descs,
                                                        const TileRef* __restrict__ tiles) {
    gemmTileBody<4, 4, 16>(descs, tiles);
}

// 128 x 128 tiles, 8 x 8 accumulators per thread: twice the FMAs per shared
// memory load of the 64 x 64 variant, for the large products.
__global__ void __launch_bounds__(NT, 1) gemmBatchedBigKernel(const GemmDesc* __restrict__ descs,
                                                              const TileRef* __restrict__ tiles) {
    gemmTileBody<8, 8, 8>(descs, tiles);
}

cudaError_t launchGemmBatchedBig(const GemmDesc* dDescs, const TileRef* dTiles, int nTiles,
                                 cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    gemmBatchedBigKernel<<<nTiles, NT, 0, s>>>(dDescs, dTiles);
    return cudaGetLastError();
}

cudaError_t launchGemmBatched(const GemmDesc* dDescs, const TileRef* dTiles, int nTiles,
                              cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    gemmBatchedKernel<<<nTiles, NT, 0, s>>>(dDescs, dTiles);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// front extend-add: UK = A A^T, UM = A B^T + B A^T, scattered (subtracted)
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) frontUpdateKernel(const FrontUpdDesc* __restrict__ descs,
                                                        const TileRef* __restrict__ tiles,
                                                        double* __restrict__ kPool,
                                                        double* __restrict__ mPool) {
    __shared__ double Ap[TK][TM + 2], Bp[TK][TM + 2], Aq[TK][TN + 2], Bq[TK][TN + 2];
    const TileRef t = tiles[blockIdx.x];
    const FrontUpdDesc D = descs[t.desc];
    const int p0 = t.m0, q0 = t.n0;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double aK[4][4], aM[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) aK[i][j] = aM[i][j] = 0.0;

    for (int k0 = 0; k0 < D.n; k0 += TK) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int idx = threadIdx.x + NT * u;
            const int r = idx % TM, k = idx / TM;
            const int gk = k0 + k;
            const bool kin = gk < D.n;
            const int gp = p0 + r, gq = q0 + r;
            const int64_t cofs = (int64_t)gk * D.ld;
            Ap[k][r] = (kin && gp < D.s) ? D.A[gp + cofs] : 0.0;
            Bp[k][r] = (kin && gp < D.s) ? D.B[gp + cofs] : 0.0;
            Aq[k][r] = (kin && gq < D.s) ? D.A[gq + cofs] : 0.0;
            Bq[k][r] = (kin && gq < D.s) ? D.B[gq + cofs] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            double ap[4], bp[4], aq[4], bq[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ap[i] = Ap[kk][tx + 16 * i];
                bp[i] = Bp[kk][tx + 16 * i];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                aq[j] = Aq[kk][ty + 16 * j];
                bq[j] = Bq[kk][ty + 16 * j];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    aK[i][j] = fma(ap[i], aq[j], aK[i][j]);
                    aM[i][j] = fma(ap[i], bq[j], fma(bp[i], aq[j], aM[i][j]));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int q = q0 + ty + 16 * j;
        if (q >= D.s) continue;
        const int pm = D.pmin[q];
        const int64_t co = D.colOff[q];
        const int rb = D.rowBase[q];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int p = p0 + tx + 16 * i;
            if (p >= D.s || p < pm) continue;
            const int64_t o = co + D.rowIdx[rb + p];
            atomicAdd(kPool + o, -aK[i][j]);
            atomicAdd(mPool + o, -aM[i][j]);
        }
    }
}

cudaError_t launchFrontUpdate(const FrontUpdDesc* dDescs, const TileRef* dTiles, int nTiles,
                              double* kPool, double* mPool, cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    frontUpdateKernel<<<nTiles, NT, 0, s>>>(dDescs, dTiles, kPool, mPool);
    return cudaGetLastError();
}

}  // namespace amls_b200
