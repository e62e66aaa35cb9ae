// Mixed-precision batched GEMM on the 5th-generation tensor cores: FP64
// operands split into BF16 pairs, products on tcgen05.mma (kind::f16, FP32
// accumulation in tensor memory), FP64 epilogue.  Same descriptors, flags
// and epilogues as the FP64 batched GEMM (gemm.cu), with 128 x 128 tiles.
//
// Split products ("BF16x3"): x = x_hi + x_lo with x_hi = bf16(x),
// x_lo = bf16(x - x_hi), and
//   A B ~= A_hi B_hi + A_hi B_lo + A_lo B_hi
// (the dropped A_lo B_lo and the representation error leave a relative error
// of about 2^-16 per product; FP32 accumulation).  Used for the M-side
// congruence and projection products of the AMLS approximation, whose
// result the FP64 refinement corrects; the factor of K stays FP64.
//
// Per CTA (256 threads): one 128 x 128 output tile, K in slices of 32 through
// a two-stage shared-memory ring.  All threads load a slice from global
// memory, split it and store the four BF16 operands (A_hi, A_lo, B_hi, B_lo)
// in the canonical K-major no-swizzle layout (8-row x 16-byte core matrices:
// core (g, c) of an operand at (4 g + c) * 128 bytes, so LBO = 128 B between
// the two K halves of an MMA and SBO = 512 B between 8-row groups); one
// thread issues 2 k-steps x 3 tcgen05.mma (M 128, N 128, K 16) per slice and
// commits them to the stage's mbarrier, which the loaders wait on before
// reusing the stage.  The accumulator (128 lanes x 128 FP32 columns of
// tensor memory) is read back with tcgen05.ld (warp w: lanes 32 (w % 4),
// columns 64 (w / 4)).  Two CTAs share an SM (64 KB of shared memory and 128
// tensor-memory columns each), so one CTA's global loads and split overlap
// the other's.  Every mbarrier wait is bounded; on a timeout the
// kernel records kDevTimeout in the status word, waits (bounded) for its
// own MMAs, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
constexpr int kThreads = 256;
constexpr int kMB = kGemmTileMixed, kNB = kGemmTileMixed;    // 128 x 128
constexpr int kKS = 32;                                      // K per stage
constexpr int kOpBytes = kMB * kKS * 2;                      // one BF16 operand slice: 8 KB
constexpr int kStageBytes = 4 * kOpBytes;                    // A_hi, A_lo, B_hi, B_lo
constexpr int kStages = 2;
constexpr size_t kSmem = size_t(kStages) * kStageBytes;
constexpr uint32_t kTmemCols = 128;
constexpr long long kWaitLimit = 1ll << 26;

// instruction descriptor: D FP32, A and B BF16, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kNB >> 3) << 17) |
                            (uint32_t(kMB >> 4) << 24);

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor, K-major, no swizzle, version 1
__device__ __forceinline__ uint64_t ummaDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= uint64_t((addr >> 4) & 0x3FFF);
    d |= uint64_t((lbo >> 4) & 0x3FFF) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFF) << 32;
    d |= uint64_t(1) << 46;
    return d;
}

__device__ __forceinline__ void mmaBf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void commitTo(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smemAddr(bar))
                 : "memory");
}

// bounded wait for the completion of the phase with the given parity
__device__ __forceinline__ bool waitParity(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smemAddr(bar);
    for (long long it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// One 8-element K chunk of one operand row into the hi/lo slices: row r (of
// 128), chunk c (of 4) -> byte offset ((r / 8) * 4 + c) * 128 + (r % 8) * 16.
// The split goes through FP32: x32 = fp32(x), hi = bf16(x32), lo =
// bf16(x32 - hi) (the subtraction is exact), so x = hi + lo + r with
// |r| <= (2^-17 + 2^-24) |x|, the same order as splitting in FP64; per pair
// of elements it costs two FP64->FP32 conversions, two FP32 subtractions and
// two packed FP32->BF16x2 conversions.
__device__ __forceinline__ void storeChunk(uint8_t* hiBase, uint8_t* loBase, int r, int c,
                                           const double (&x)[8]) {
    uint4 h, l;
    uint32_t* hw = &h.x;
    uint32_t* lw = &l.x;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float a = static_cast<float>(x[2 * e]), b = static_cast<float>(x[2 * e + 1]);
        const __nv_bfloat162 hb = __floats2bfloat162_rn(a, b);
        const float2 hf = __bfloat1622float2(hb);
        const __nv_bfloat162 lb = __floats2bfloat162_rn(a - hf.x, b - hf.y);
        hw[e] = *reinterpret_cast<const uint32_t*>(&hb);
        lw[e] = *reinterpret_cast<const uint32_t*>(&lb);
    }
    const int off = ((r >> 3) * 4 + c) * 128 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(hiBase + off) = h;
    *reinterpret_cast<uint4*>(loBase + off) = l;
}

// slice [k0, k0 + 32) of op(A) rows m0.. and op(B) columns n0.. into a stage
__device__ __forceinline__ void loadSlice(const GemmDesc& D, int m0, int n0, int k0, int kEnd,
                                          uint8_t* st) {
    const bool ta = D.flags & kTransA, tb = D.flags & kTransB, ga = D.flags & kGatherA;
    // 128 rows x 4 chunks per operand = 512 chunks, 2 per thread
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int idx = threadIdx.x + kThreads * u;
        const int r = idx % kMB, c = idx / kMB;
        double x[8];
        const int gi = m0 + r;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int gk = k0 + c * 8 + e;
            double v = 0.0;
            if (gi < D.M && gk < kEnd) {
                if (ta) v = D.A[gk + (int64_t)gi * D.lda];
                else if (ga) v = D.A[gi + (int64_t)D.aMap[gk] * D.lda];
                else v = D.A[gi + (int64_t)gk * D.lda];
            }
            x[e] = v;
        }
        storeChunk(st, st + kOpBytes, r, c, x);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int idx = threadIdx.x + kThreads * u;
        const int r = idx % kNB, c = idx / kNB;
        double x[8];
        const int gj = n0 + r;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int gk = k0 + c * 8 + e;
            double v = 0.0;
            if (gj < D.N && gk < kEnd) v = tb ? D.B[gj + (int64_t)gk * D.ldb] : D.B[gk + (int64_t)gj * D.ldb];
            x[e] = v;
        }
        storeChunk(st + 2 * kOpBytes, st + 3 * kOpBytes, r, c, x);
    }
}

__device__ __forceinline__ void epilogueStore(const GemmDesc& D, int row, int col, double acc) {
    if (row >= D.M || col >= D.N) return;
    double v = D.alpha * acc;
    if (D.flags & kColScale) v *= D.colScale[col];
    if (D.flags & kRowScale) v *= D.rowScale[row];
    if (D.flags & kScatter) {
        double* dst = D.C + D.colOff[col] + D.rowIdx[row];
        if (D.flags & kAtomic) atomicAdd(dst, v);
        else if (D.flags & kAccumulate) *dst += v;
        else *dst = v;
    } else {
        double* dst = D.C + row + (int64_t)col * D.ldc;
        if (D.kChunk > 0) atomicAdd(dst, v);
        else if (D.flags & kAccumulate) *dst = v + D.beta * (*dst);
        else *dst = v;
    }
}
}  // namespace

__global__ void __launch_bounds__(kThreads, 2) gemmMixedKernel(const GemmDesc* __restrict__ descs,
                                                               const TileRef* __restrict__ tiles,
                                                               int* status) {
    extern __shared__ __align__(128) uint8_t mxSmem[];
    __shared__ __align__(8) uint64_t bar[kStages];
    __shared__ uint32_t tmemSlot;
    __shared__ int failed;
    const TileRef t = tiles[blockIdx.x];
    const GemmDesc D = descs[t.desc];
    const int m0 = t.m0, n0 = t.n0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smemAddr(&tmemSlot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(&bar[s])));
        asm volatile("fence.mbarrier_init.release.cluster;");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmemSlot;

    int kBeg = D.kChunk > 0 ? t.pad * D.kChunk : 0;
    int kEnd = D.kChunk > 0 ? min(D.K, kBeg + D.kChunk) : D.K;
    if (D.flags & kTriKUpTo) kEnd = min(kEnd, n0 + kNB);
    if (D.flags & kTriKFrom) kBeg = max(kBeg, n0);
    if (D.flags & kTriAUpTo) kEnd = min(kEnd, m0 + kMB);
    const int nSlices = kEnd > kBeg ? (kEnd - kBeg + kKS - 1) / kKS : 0;

    int issued = 0;                       // slices whose MMAs were committed
    for (int sl = 0; sl < nSlices; ++sl) {
        const int s = sl & 1;
        uint8_t* st = mxSmem + s * kStageBytes;
        if (sl >= kStages && !failed) {
            // the MMAs of slice sl - 2 have finished reading this stage
            if (!waitParity(&bar[s], uint32_t(((sl - kStages) / kStages) & 1)) && lane == 0) failed = 1;
        }
        __syncthreads();
        if (failed) break;
        loadSlice(D, m0, n0, kBeg + sl * kKS, kEnd, st);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t base = smemAddr(st);
#pragma unroll
            for (int ks = 0; ks < kKS / 16; ++ks) {
                const uint32_t off = ks * 2 * 128;
                const uint64_t aHi = ummaDesc(base + off, 128, 512);
                const uint64_t aLo = ummaDesc(base + kOpBytes + off, 128, 512);
                const uint64_t bHi = ummaDesc(base + 2 * kOpBytes + off, 128, 512);
                const uint64_t bLo = ummaDesc(base + 3 * kOpBytes + off, 128, 512);
                mmaBf16(tmem, aHi, bHi, (sl > 0 || ks > 0) ? 1u : 0u);
                mmaBf16(tmem, aHi, bLo, 1u);
                mmaBf16(tmem, aLo, bHi, 1u);
            }
            commitTo(&bar[s]);
        }
        ++issued;
    }
    // all MMAs done: the last commit tracks every earlier one of this thread
    if (issued > 0) {
        const int last = issued - 1;
        if (!waitParity(&bar[last & 1], uint32_t((last / kStages) & 1)) && lane == 0) failed = 1;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    __syncthreads();
    if (failed) {
        if (tid == 0) setStatus(status, kDevTimeout, blockIdx.x);
    } else {
        // warp w reads lanes 32 (w % 4) .. + 31 (rows), columns 64 (w / 4) .. + 63
        const int rowBase = 32 * (warp & 3), colBase = 64 * (warp >> 2);
        const int row = m0 + rowBase + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < 64; c0 += 8) {
            uint32_t r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (nSlices > 0) {
                const uint32_t taddr = tmem + (uint32_t(rowBase) << 16) + uint32_t(colBase + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            }
#pragma unroll
            for (int j = 0; j < 8; ++j)
                epilogueStore(D, row, n0 + colBase + c0 + j, static_cast<double>(__uint_as_float(r[j])));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

cudaError_t launchGemmBatchedMixed(const GemmDesc* dDescs, const TileRef* dTiles, int nTiles,
                                   int* status, cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(gemmMixedKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    gemmMixedKernel<<<nTiles, kThreads, kSmem, s>>>(dDescs, dTiles, status);
    return cudaGetLastError();
}

}  // namespace amls_b200
