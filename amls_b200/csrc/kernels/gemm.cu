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
// An operand slice is stored in shared memory in the order it is contiguous
// in global memory, so that consecutive cp.async writes land in consecutive
// banks: k-major ([k][row], row pitch kLdA / kLdB) when rows are contiguous,
// row-major ([row][k], pitch kLdK) when k is.  Both pitches are 4 mod 16
// doubles, which keeps the fragment loads at two wavefronts per warp.
constexpr int kLdA = kBM + 4, kLdB = kBN + 4;
constexpr int kLdK = kKs + 4;
constexpr int kOpSlot = (kKs * kLdA > kBM * kLdK) ? kKs * kLdA : kBM * kLdK;   // doubles per operand
constexpr int kStage = 2 * kOpSlot;                // doubles per stage
constexpr size_t kGemmSmem = sizeof(double) * kStages * kStage;

__device__ __forceinline__ void dmma16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
    asm("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
          "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Asynchronous copies to a shared-space address; a source size below the
// copy size zero-fills the rest (0: nothing is read).
__device__ __forceinline__ void cpAsync8(unsigned dst, const double* src, int bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cpAsync16(unsigned dst, const double* src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }

// Copy plan of one operand of a tile.  A K slice of the operand (64 rows x
// 16 k) is stored in shared memory in the order it is contiguous in global
// memory:
//   row layout ([k][row], pitch kLdA; rows contiguous, or gathered columns
//   whose rows are contiguous): 8-byte copies, thread t copies row t % 64 of
//   k = t / 64 + 2u (u < 8); 16-byte copies, rows 2 (t % 32) and the next of
//   k = t / 32 + 4u (u < 4);
//   k layout ([row][k], pitch kLdK; k contiguous): 8-byte copies, thread t
//   copies k = t % 16 of rows t / 16 + 8u (u < 8); 16-byte copies, k =
//   2 (t % 8) and the next of rows t / 8 + 16u (u < 4).
// A thread's copies in a slice differ by a constant source step, and the
// next slice is a constant step further, so a copy costs one address add, a
// size select and the copy.  16-byte copies need a 16-byte aligned operand
// with an even leading dimension (and an even first k for the k layout);
// otherwise the plan uses 8-byte copies.
struct CopyPlan {
    const double* p;    // source of copy u = 0 in the next slice (gathered: row base)
    const double* safe; // operand base: the source of copies that read nothing
    int64_t stepU;      // source step between copies u
    int64_t ld;
    int rowsLeft;       // row layout: valid rows from the thread's first row
    int rq;             // k layout: the thread's first row
    int rows;           // k layout: valid rows of the tile
    int sub;            // row layout: the thread's first k; k layout: the thread's k
    unsigned dst;       // shared offset (bytes) of copy u = 0 within the operand slot
    bool vec;
};

__device__ __forceinline__ bool aligned16(const double* p) {
    return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

__device__ __forceinline__ CopyPlan planRow(const double* base, int64_t ld, int row0, int rows, int kBeg,
                                            bool gather, int t = threadIdx.x) {
    CopyPlan c;
    c.vec = aligned16(base) && (ld & 1) == 0;
    const int r = c.vec ? 2 * (t & 31) : (t & 63);
    c.sub = c.vec ? (t >> 5) : (t >> 6);
    c.rowsLeft = rows - r;
    c.ld = ld;
    c.stepU = (c.vec ? 4 : 2) * ld;
    c.safe = base;
    c.p = gather ? base + row0 + r : base + row0 + r + (int64_t)(kBeg + c.sub) * ld;
    c.dst = 8u * static_cast<unsigned>(c.sub * kLdA + r);
    return c;
}

__device__ __forceinline__ CopyPlan planK(const double* base, int64_t ld, int row0, int rows, int kBeg) {
    CopyPlan c;
    const int t = threadIdx.x;
    c.vec = aligned16(base) && (ld & 1) == 0 && (kBeg & 1) == 0;
    c.sub = c.vec ? 2 * (t & 7) : (t & 15);
    c.rq = c.vec ? (t >> 3) : (t >> 4);
    c.rows = rows;
    c.ld = ld;
    c.stepU = (c.vec ? 16 : 8) * ld;
    c.safe = base;
    c.p = base + (int64_t)(row0 + c.rq) * ld + kBeg + c.sub;
    c.dst = 8u * static_cast<unsigned>(c.rq * kLdK + c.sub);
    return c;
}

// one slice of a row-layout operand; kLeft = valid k from the slice start;
// map (gathered columns) = the column indices of the thread's copies
template <bool GATHER>
__device__ __forceinline__ void issueRow(CopyPlan& c, unsigned slot, int kLeft, const int32_t (&map)[8]) {
    if (c.vec) {
        const int rb = c.rowsLeft >= 2 ? 16 : (c.rowsLeft == 1 ? 8 : 0);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int b = c.sub + 4 * u < kLeft ? rb : 0;
            const double* src = GATHER ? c.p + (int64_t)map[u] * c.ld : c.p + u * c.stepU;
            cpAsync16(slot + c.dst + 8u * 4 * kLdA * u, b ? src : c.safe, b);
        }
    } else {
        const int rb = c.rowsLeft > 0 ? 8 : 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int b = c.sub + 2 * u < kLeft ? rb : 0;
            const double* src = GATHER ? c.p + (int64_t)map[u] * c.ld : c.p + u * c.stepU;
            cpAsync8(slot + c.dst + 8u * 2 * kLdA * u, b ? src : c.safe, b);
        }
    }
    if (!GATHER) c.p += kKs * c.ld;
}

__device__ __forceinline__ void issueK(CopyPlan& c, unsigned slot, int kLeft) {
    if (c.vec) {
        const int kb = c.sub + 1 < kLeft ? 16 : (c.sub < kLeft ? 8 : 0);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int b = c.rq + 16 * u < c.rows ? kb : 0;
            cpAsync16(slot + c.dst + 8u * 16 * kLdK * u, b ? c.p + u * c.stepU : c.safe, b);
        }
    } else {
        const int kb = c.sub < kLeft ? 8 : 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int b = c.rq + 8 * u < c.rows ? kb : 0;
            cpAsync8(slot + c.dst + 8u * 8 * kLdK * u, b ? c.p + u * c.stepU : c.safe, b);
        }
    }
    c.p += kKs;
}

// Gathered A: the column indices of the thread's copies of slice k0, loaded
// one slice ahead so that the address of a gathered copy never waits on the
// map (out-of-range k read index 0: their copies are zero-filled).
__device__ __forceinline__ void loadMap(const GemmDesc& D, const CopyPlan& c, int k0, int kEnd,
                                        int32_t (&am)[8]) {
    const int ks = c.vec ? 4 : 2;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int gk = k0 + c.sub + ks * u;
        am[u] = (u < (c.vec ? 4 : 8) && gk < kEnd) ? D.aMap[gk] : 0;
    }
}

template <bool TA, bool TB, bool GA>
__device__ __forceinline__ void issueSlice(CopyPlan& pa, CopyPlan& pb, unsigned slot, int kLeft,
                                           const int32_t (&am)[8]) {
    if (TA) issueK(pa, slot, kLeft);
    else issueRow<GA>(pa, slot, kLeft, am);
    if (TB) issueRow<false>(pb, slot + 8u * kOpSlot, kLeft, am);
    else issueK(pb, slot + 8u * kOpSlot, kLeft);
}

// K range of a tile: split-K chunk; triangular B restricts k to <= the
// tile's last column (kTriKUpTo) or >= its first column (kTriKFrom),
// triangular A to <= the tile's last row (kTriAUpTo)
struct TileRange {
    int kBeg, kEnd, nSlices;
};
__device__ __forceinline__ TileRange tileRange(const GemmDesc& D, const TileRef& t) {
    TileRange r;
    r.kBeg = D.kChunk > 0 ? t.pad * D.kChunk : 0;
    r.kEnd = D.kChunk > 0 ? min(D.K, r.kBeg + D.kChunk) : D.K;
    if (D.flags & kTriKUpTo) r.kEnd = min(r.kEnd, t.n0 + kBN);
    if (D.flags & kTriKFrom) r.kBeg = max(r.kBeg, t.n0);
    if (D.flags & kTriAUpTo) r.kEnd = min(r.kEnd, t.m0 + kBM);
    r.nSlices = r.kEnd > r.kBeg ? (r.kEnd - r.kBeg + kKs - 1) / kKs : 0;
    return r;
}

__device__ __forceinline__ void zeroAcc(double (&acc)[2][kFJ][4]) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < kFJ; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;
}

// One K slice from shared memory into the accumulators.  Fragments: A
// element (MMA row g (+8), k tg + 4 q), B element (k tg + 4 q, MMA col g).
// An operand in the row layout is read two rows at a time (16-byte loads):
// MMA rows g and g + 8 of a 16-row block are tile rows 2g and 2g + 1, and MMA
// col g of n8 fragments 2p and 2p + 1 are tile cols 16p + 2g and 16p + 2g + 1;
// the epilogue maps the accumulators back.
template <bool TA, bool TB>
__device__ __forceinline__ void computeSlice(double (&acc)[2][kFJ][4], const double* As, const double* Bs) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    double a[2][8], b[kFJ][4];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = tg + 4 * q;
            if (TA) {
                const int r = wm + 16 * i + g;
                a[i][2 * q] = As[r * kLdK + k];
                a[i][2 * q + 1] = As[(r + 8) * kLdK + k];
            } else {
                const double2 v = *reinterpret_cast<const double2*>(As + k * kLdA + wm + 16 * i + 2 * g);
                a[i][2 * q] = v.x;
                a[i][2 * q + 1] = v.y;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = tg + 4 * q;
        if (TB) {
#pragma unroll
            for (int jp = 0; jp < kFJ / 2; ++jp) {
                const double2 v = *reinterpret_cast<const double2*>(Bs + k * kLdB + wn + 16 * jp + 2 * g);
                b[2 * jp][q] = v.x;
                b[2 * jp + 1][q] = v.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kFJ; ++j) b[j][q] = Bs[(wn + 8 * j + g) * kLdK + k];
        }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < kFJ; ++j) dmma16x8x16(acc[i][j], a[i], b[j]);
}

// Epilogue: fragment (i, j) element q sits at MMA row wm + 16 i + g + 8 (q / 2),
// MMA column wn + 8 j + 2 tg + (q % 2); tile row and column as the fragment
// loads relabelled them.
template <bool TA, bool TB>
__device__ __forceinline__ void storeTile(const GemmDesc& D, int m0, int n0, const double (&acc)[2][kFJ][4]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
#pragma unroll
    for (int j = 0; j < kFJ; ++j)
#pragma unroll
        for (int q2 = 0; q2 < 2; ++q2) {
            const int col = TB ? n0 + wn + 16 * (j / 2) + 4 * tg + 2 * q2 + (j % 2)
                               : n0 + wn + 8 * j + 2 * tg + q2;
            if (col >= D.N) continue;
            const double cs = (D.flags & kColScale) ? D.colScale[col] : 1.0;
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row = TA ? m0 + wm + 16 * i + g + 8 * h : m0 + wm + 16 * i + 2 * g + h;
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

template <bool TA, bool TB, bool GA>
__device__ __forceinline__ void gemmTile(const GemmDesc& D, const TileRef& t, double* sm) {
    double acc[2][kFJ][4];
    zeroAcc(acc);
    const TileRange R = tileRange(D, t);
    const int kBeg = R.kBeg, kEnd = R.kEnd, nSlices = R.nSlices;
    const int m0 = t.m0, n0 = t.n0;
    const int mRows = min(kBM, D.M - m0), nRows = min(kBN, D.N - n0);
    CopyPlan pa = TA ? planK(D.A, D.lda, m0, mRows, kBeg) : planRow(D.A, D.lda, m0, mRows, kBeg, GA);
    CopyPlan pb = TB ? planRow(D.B, D.ldb, n0, nRows, kBeg, false) : planK(D.B, D.ldb, n0, nRows, kBeg);
    const unsigned sm0 = static_cast<unsigned>(__cvta_generic_to_shared(sm));
    int32_t am[8];
#pragma unroll
    for (int st = 0; st < kStages - 1; ++st) {
        if (st < nSlices) {
            if (GA) loadMap(D, pa, kBeg + st * kKs, kEnd, am);
            issueSlice<TA, TB, GA>(pa, pb, sm0 + 8u * st * kStage, kEnd - kBeg - st * kKs, am);
        }
        cpAsyncCommit();
    }
    if (GA && kStages - 1 < nSlices) loadMap(D, pa, kBeg + (kStages - 1) * kKs, kEnd, am);
    for (int sl = 0; sl < nSlices; ++sl) {
        cpAsyncWait<kStages - 2>();
        __syncthreads();
        const int nx = sl + kStages - 1;
        if (nx < nSlices) {
            issueSlice<TA, TB, GA>(pa, pb, sm0 + 8u * (nx % kStages) * kStage, kEnd - kBeg - nx * kKs, am);
            if (GA && nx + 1 < nSlices) loadMap(D, pa, kBeg + (nx + 1) * kKs, kEnd, am);
        }
        cpAsyncCommit();
        const double* As = sm + (sl % kStages) * kStage;
        computeSlice<TA, TB>(acc, As, As + kOpSlot);
    }
    cpAsyncWait<0>();
    storeTile<TA, TB>(D, m0, n0, acc);
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

// Operand slots of a stage: Ap, Bp, Aq, Bq (64 rows x 16 k each, [k][row]).
// Threads 0..127 copy the A slices (rows p, rows q), threads 128..255 the B
// slices, each through the GEMM's row-layout copy plans.
constexpr unsigned kFuOpBytes = 8u * kKs * kLdA;
__device__ __forceinline__ void fuIssueSlice(CopyPlan& cp, CopyPlan& cq, unsigned st, int kLeft) {
    const int32_t none[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const unsigned opB = threadIdx.x >= 128 ? 1u : 0u;
    issueRow<false>(cp, st + opB * kFuOpBytes, kLeft, none);
    issueRow<false>(cq, st + (2u + opB) * kFuOpBytes, kLeft, none);
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
    const double* src = threadIdx.x < 128 ? D.A : D.B;
    const int ct = threadIdx.x & 127;
    CopyPlan cp = planRow(src, D.ld, p0, min(64, D.s - p0), 0, false, ct);
    CopyPlan cq = planRow(src, D.ld, q0, min(64, D.s - q0), 0, false, ct);
    const unsigned sm0 = static_cast<unsigned>(__cvta_generic_to_shared(fuSmem));
#pragma unroll
    for (int st = 0; st < kStages - 1; ++st) {
        if (st < nSlices) fuIssueSlice(cp, cq, sm0 + 8u * st * kFuStage, D.n - st * kKs);
        cpAsyncCommit();
    }
    for (int sl = 0; sl < nSlices; ++sl) {
        cpAsyncWait<kStages - 2>();
        __syncthreads();
        const int nx = sl + kStages - 1;
        if (nx < nSlices) fuIssueSlice(cp, cq, sm0 + 8u * (nx % kStages) * kFuStage, D.n - nx * kKs);
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
