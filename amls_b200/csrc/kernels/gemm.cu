// Batched FP64 GEMM with gather/scatter epilogues, and the front extend-add
// update (SYRK + SYR2K of the eliminated front, scattered into ancestors).
//
// B200 has no FP64 tcgen05 kind; its FP64 tensor-core path is the warp-level
// DMMA (mma.sync .f64), which these kernels use: 64 x 64 output tile per CTA,
// 4 warps as 2 (M) x 2 (N), warp tile 32 x 32 = 2 x 4 fragments of
// m16n8k16 (the front update: 8 warps of 32 x 16), operands streamed global -> shared memory with cp.async through a
// three-deep ring of K slices of 16 (one barrier per slice, no register
// staging).  The operand layout (transposed A / B, gathered A columns) is a
// template parameter selected per CTA from the descriptor, so the copy loops
// carry no per-element branches.
#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
constexpr int NT = 256;            // front update
constexpr int kGemmThreads = 128;  // batched GEMM: 4 warps of 32 x 32
constexpr int kFJ = 4;             // n8 fragments per warp (warp tile 32 x 8 kFJ)

constexpr int kBM = kGemmTile, kBN = kGemmTile;   // 64 x 64
constexpr int kKs = 16;                            // K slice
constexpr int kStages = 3;
constexpr int kLdA = kBM + 4, kLdB = kBN + 4;      // = 4 mod 16 doubles
constexpr int kStage = kKs * (kLdA + kLdB);        // doubles per stage
constexpr size_t kGemmSmem = sizeof(double) * kStages * kStage;
constexpr int kLA = kBM * kKs / kGemmThreads, kLB = kBN * kKs / kGemmThreads;

__device__ __forceinline__ void dmma16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
    asm("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
          "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// 8-byte asynchronous copy; src_size 0 writes zeros and reads nothing
__device__ __forceinline__ void cpAsync8(double* dst, const double* src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }

// one K slice of op(A) (kBM x kKs) and op(B) (kKs x kBN) into shared memory,
// stored k-major: As[k][i], Bs[k][j]; global reads coalesced on the
// contiguous side of each layout
// Gathered A (GA): the column indices aMap[gk] of a slice, loaded one slice
// ahead into registers so that the address of a gathered copy never waits
// on the map.
template <bool GA>
__device__ __forceinline__ void loadMap(const GemmDesc& D, int k0, int kEnd, int32_t (&am)[kLA]) {
    if constexpr (GA) {
#pragma unroll
        for (int u = 0; u < kLA; ++u) {
            const int gk = k0 + (threadIdx.x + kGemmThreads * u) / kBM;
            am[u] = gk < kEnd ? D.aMap[gk] : 0;
        }
    }
}

template <bool TA, bool TB, bool GA>
__device__ __forceinline__ void issueSlice(const GemmDesc& D, int m0, int n0, int k0, int kEnd,
                                           double* As, double* Bs, const int32_t (&am)[kLA]) {
#pragma unroll
    for (int u = 0; u < kLA; ++u) {
        const int idx = threadIdx.x + kGemmThreads * u;
        const int i = TA ? idx / kKs : idx % kBM;
        const int k = TA ? idx % kKs : idx / kBM;
        const int gi = m0 + i, gk = k0 + k;
        const bool ok = gi < D.M && gk < kEnd;
        const double* src = D.A;
        if (ok) {
            if (TA) src = D.A + gk + (int64_t)gi * D.lda;
            else if (GA) src = D.A + gi + (int64_t)am[u] * D.lda;
            else src = D.A + gi + (int64_t)gk * D.lda;
        }
        cpAsync8(As + k * kLdA + i, src, ok);
    }
#pragma unroll
    for (int u = 0; u < kLB; ++u) {
        const int idx = threadIdx.x + kGemmThreads * u;
        const int j = TB ? idx % kBN : idx / kKs;
        const int k = TB ? idx / kBN : idx % kKs;
        const int gj = n0 + j, gk = k0 + k;
        const bool ok = gj < D.N && gk < kEnd;
        const double* src = D.B;
        if (ok) src = TB ? D.B + gj + (int64_t)gk * D.ldb : D.B + gk + (int64_t)gj * D.ldb;
        cpAsync8(Bs + k * kLdB + j, src, ok);
    }
}

template <bool TA, bool TB, bool GA>
__device__ __forceinline__ void gemmTile(const GemmDesc& D, const TileRef& t, double* sm) {
    const int m0 = t.m0, n0 = t.n0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    double acc[2][kFJ][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < kFJ; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;
    // split-K range; triangular B restricts k to <= the tile's last column
    // (kTriKUpTo) or >= its first column (kTriKFrom), triangular A to <= the
    // tile's last row (kTriAUpTo)
    int kBeg = D.kChunk > 0 ? t.pad * D.kChunk : 0;
    int kEnd = D.kChunk > 0 ? min(D.K, kBeg + D.kChunk) : D.K;
    if (D.flags & kTriKUpTo) kEnd = min(kEnd, n0 + kBN);
    if (D.flags & kTriKFrom) kBeg = max(kBeg, n0);
    if (D.flags & kTriAUpTo) kEnd = min(kEnd, m0 + kBM);
    const int nSlices = kEnd > kBeg ? (kEnd - kBeg + kKs - 1) / kKs : 0;
    int32_t am[kLA];
#pragma unroll
    for (int st = 0; st < kStages - 1; ++st) {
        if (st < nSlices) {
            double* base = sm + st * kStage;
            loadMap<GA>(D, kBeg + st * kKs, kEnd, am);
            issueSlice<TA, TB, GA>(D, m0, n0, kBeg + st * kKs, kEnd, base, base + kKs * kLdA, am);
        }
        cpAsyncCommit();
    }
    if (kStages - 1 < nSlices) loadMap<GA>(D, kBeg + (kStages - 1) * kKs, kEnd, am);
    for (int sl = 0; sl < nSlices; ++sl) {
        cpAsyncWait<kStages - 2>();
        __syncthreads();
        const int nx = sl + kStages - 1;
        if (nx < nSlices) {
            double* base = sm + (nx % kStages) * kStage;
            issueSlice<TA, TB, GA>(D, m0, n0, kBeg + nx * kKs, kEnd, base, base + kKs * kLdA, am);
            if (nx + 1 < nSlices) loadMap<GA>(D, kBeg + (nx + 1) * kKs, kEnd, am);
        }
        cpAsyncCommit();
        const double* As = sm + (sl % kStages) * kStage;
        const double* Bs = As + kKs * kLdA;
        // fragments: A element (row g (+8), k tg + 4 q), B element (k tg + 4 q, col g)
        double a[2][8], b[kFJ][4];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = wm + 16 * i + g;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                a[i][2 * q] = As[(tg + 4 * q) * kLdA + r];
                a[i][2 * q + 1] = As[(tg + 4 * q) * kLdA + r + 8];
            }
        }
#pragma unroll
        for (int j = 0; j < kFJ; ++j) {
            const int c = wn + 8 * j + g;
#pragma unroll
            for (int q = 0; q < 4; ++q) b[j][q] = Bs[(tg + 4 * q) * kLdB + c];
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < kFJ; ++j) dmma16x8x16(acc[i][j], a[i], b[j]);
    }
    cpAsyncWait<0>();
    // epilogue: fragment (i, j) element q sits at row wm + 16 i + g + 8 (q / 2),
    // column wn + 8 j + 2 tg + (q % 2)
#pragma unroll
    for (int j = 0; j < kFJ; ++j)
#pragma unroll
        for (int q2 = 0; q2 < 2; ++q2) {
            const int col = n0 + wn + 8 * j + 2 * tg + q2;
            if (col >= D.N) continue;
            const double cs = (D.flags & kColScale) ? D.colScale[col] : 1.0;
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row = m0 + wm + 16 * i + g + 8 * h;
                    if (row >= D.M) continue;
                    double v = D.alpha * acc[i][j][2 * h + q2] * cs;
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

__global__ void __launch_bounds__(kGemmThreads, 3) gemmBatchedKernel(const GemmDesc* __restrict__ descs,
                                                        const TileRef* __restrict__ tiles) {
    extern __shared__ double gemmSmem[];
    const TileRef t = tiles[blockIdx.x];
    const GemmDesc D = descs[t.desc];
    if (t.m0 >= D.M || t.n0 >= D.N) return;          // tile outside a shrunk descriptor
    const bool ta = D.flags & kTransA, tb = D.flags & kTransB, ga = D.flags & kGatherA;
    if (ga) {
        if (tb) gemmTile<false, true, true>(D, t, gemmSmem);
        else gemmTile<false, false, true>(D, t, gemmSmem);
    } else if (ta) {
        if (tb) gemmTile<true, true, false>(D, t, gemmSmem);
        else gemmTile<true, false, false>(D, t, gemmSmem);
    } else {
        if (tb) gemmTile<false, true, false>(D, t, gemmSmem);
        else gemmTile<false, false, false>(D, t, gemmSmem);
    }
}

cudaError_t launchGemmBatched(const GemmDesc* dDescs, const TileRef* dTiles, int nTiles,
                              cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(gemmBatchedKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kGemmSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    gemmBatchedKernel<<<nTiles, kGemmThreads, kGemmSmem, s>>>(dDescs, dTiles);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// front extend-add: UK = A A^T, UM = A B^T + B A^T, scattered (subtracted)
// ------------------------------------------------------------------------
// The front update on the FP64 tensor cores: tile (p0, q0) of the s x s
// update, operands A = L_Si and B = R_i^T rows p (M side) and rows q (N side)
// through the same cp.async ring as the GEMM (four 64 x 16 slices per stage),
// three m16n8k16 DMMA products per fragment pair (UK += Ap Aq^T,
// UM += Ap Bq^T + Bp Aq^T), then the extend-add scatter (subtract, atomic)
// into the ancestors' K and M fronts for p >= pmin[q].
namespace {
constexpr int kFuStage = 4 * kKs * kLdA;   // Ap, Bp, Aq, Bq slices
constexpr size_t kFuSmem = sizeof(double) * kStages * kFuStage;

__device__ __forceinline__ void fuIssueSlice(const FrontUpdDesc& D, int p0, int q0, int k0, double* st) {
    // 4 operands x 64 rows x 16 k = 4096 elements, 16 per thread
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int idx = threadIdx.x + NT * u;
        const int op = idx >> 10, e = idx & 1023;
        const int r = e % 64, k = e / 64;
        const int gk = k0 + k;
        const int gr = (op < 2 ? p0 : q0) + r;
        const bool ok = gr < D.s && gk < D.n;
        const double* base = (op == 0 || op == 2) ? D.A : D.B;
        const double* src = ok ? base + gr + (int64_t)gk * D.ld : D.A;
        cpAsync8(st + op * kKs * kLdA + k * kLdA + r, src, ok);
    }
}
}  // namespace

__global__ void __launch_bounds__(NT) frontUpdateKernel(const FrontUpdDesc* __restrict__ descs,
                                                        const TileRef* __restrict__ tiles,
                                                        double* __restrict__ kPool,
                                                        double* __restrict__ mPool) {
    extern __shared__ double fuSmem[];
    const TileRef t = tiles[blockIdx.x];
    const FrontUpdDesc D = descs[t.desc];
    const int p0 = t.m0, q0 = t.n0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
    double aK[2][2][4], aM[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) aK[i][j][q] = aM[i][j][q] = 0.0;
    const int nSlices = (D.n + kKs - 1) / kKs;
#pragma unroll
    for (int st = 0; st < kStages - 1; ++st) {
        if (st < nSlices) fuIssueSlice(D, p0, q0, st * kKs, fuSmem + st * kFuStage);
        cpAsyncCommit();
    }
    for (int sl = 0; sl < nSlices; ++sl) {
        cpAsyncWait<kStages - 2>();
        __syncthreads();
        const int nx = sl + kStages - 1;
        if (nx < nSlices) fuIssueSlice(D, p0, q0, nx * kKs, fuSmem + (nx % kStages) * kFuStage);
        cpAsyncCommit();
        const double* Ap = fuSmem + (sl % kStages) * kFuStage;
        const double* Bp = Ap + kKs * kLdA;
        const double* Aq = Bp + kKs * kLdA;
        const double* Bq = Aq + kKs * kLdA;
        double ap[2][8], bp[2][8], aq[2][4], bq[2][4];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = wm + 16 * i + g;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ap[i][2 * q] = Ap[(tg + 4 * q) * kLdA + r];
                ap[i][2 * q + 1] = Ap[(tg + 4 * q) * kLdA + r + 8];
                bp[i][2 * q] = Bp[(tg + 4 * q) * kLdA + r];
                bp[i][2 * q + 1] = Bp[(tg + 4 * q) * kLdA + r + 8];
            }
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int c = wn + 8 * j + g;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                aq[j][q] = Aq[(tg + 4 * q) * kLdA + c];
                bq[j][q] = Bq[(tg + 4 * q) * kLdA + c];
            }
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                dmma16x8x16(aK[i][j], ap[i], aq[j]);
                dmma16x8x16(aM[i][j], ap[i], bq[j]);
                dmma16x8x16(aM[i][j], bp[i], aq[j]);
            }
    }
    cpAsyncWait<0>();
    // fragment (i, j) element e: row p = p0 + wm + 16 i + g + 8 (e / 2),
    // column q = q0 + wn + 8 j + 2 tg + (e % 2)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            const int q = q0 + wn + 8 * j + 2 * tg + e2;
            if (q >= D.s) continue;
            const int pm = D.pmin[q];
            const int64_t co = D.colOff[q];
            const int rb = D.rowBase[q];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int p = p0 + wm + 16 * i + g + 8 * h;
                    if (p >= D.s || p < pm) continue;
                    const int64_t o = co + D.rowIdx[rb + p];
                    atomicAdd(kPool + o, -aK[i][j][2 * h + e2]);
                    atomicAdd(mPool + o, -aM[i][j][2 * h + e2]);
                }
        }
}

cudaError_t launchFrontUpdate(const FrontUpdDesc* dDescs, const TileRef* dTiles, int nTiles,
                              double* kPool, double* mPool, cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(frontUpdateKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kFuSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    frontUpdateKernel<<<nTiles, NT, kFuSmem, s>>>(dDescs, dTiles, kPool, mPool);
    return cudaGetLastError();
}

}  // namespace amls_b200
