// Shift-invert Lanczos (SIL) on the node pencils (K^_ii, M^_ii): the
// reference's node-local sparse eigensolver (src/amls/shift_invert_lanczos.hpp:
// 32-203), used for the nodes its sparsity rule picks
// (src/amls/eigenpair_solver.hpp:68-82).
//
//   sigma = -max(1e-10, 1e-9 max_j |K^_jj|)            (:134-135, :178)
//   A = K^ - sigma M^ = L L^T,  B = A^-1 = L^-T L^-1    (:35-41)
//   M-inner-product Lanczos on C = A^-1 M^ with full reorthogonalisation
//   (:44-85): w = C q_j, alpha_j = q_j^T M w, two Gram-Schmidt passes
//   against q_0 .. q_j, beta_j = ||w||_M, q_{j+1} = w / beta_j; the start
//   vector is the reference's Eigen Random vector after std::srand(12345).
//
// Layout per node (order n): B (n x n), Q, MQ = M Q (n x n, column l = q_l),
// QT = Q^T (so both Gram-Schmidt products read contiguous memory), vectors
// w, mw, coef, alpha, beta (n each), and the node's M^ as a local CSR whose
// values are read from the M front (lower triangle) at run time.
//
// The iteration runs in one cooperative kernel over all SIL nodes of a
// batch: per step seven grid-wide phases, each a flat list of warp-sized
// units (a row, or a basis vector) spread evenly over the grid, with warp
// shuffle reductions in a fixed order (deterministic); data written by other
// CTAs inside the kernel is read with L2 loads (__ldcg).
#include <cooperative_groups.h>

#include <cmath>

#include "common.cuh"
#include "launch.hpp"

namespace cg = cooperative_groups;

namespace amls_b200 {

namespace {
constexpr int kSilThreads = 256;
constexpr int kSilWarps = kSilThreads / 32;

// std::rand() of the Microsoft C runtime (the reference's documented MSYS2
// mingw64 toolchain): x <- 214013 x + 2531011 (mod 2^32), value
// (x >> 16) & 0x7fff.  The state after `calls` updates from `seed`, by
// binary powering of the affine map (any element computable on its own).
__device__ __forceinline__ uint32_t lcgState(uint32_t seed, uint32_t calls) {
    uint32_t a = 214013u, c = 2531011u;     // f^(2^k)
    uint32_t A = 1u, C = 0u;                // accumulated map
    while (calls) {
        if (calls & 1u) {
            A = a * A;
            C = a * C + c;
        }
        c = (a + 1u) * c;
        a = a * a;
        calls >>= 1;
    }
    return A * seed + C;
}

}  // namespace

// dst[r + c n] = the front's diagonal block: mode 0 the full symmetric copy of
// its lower triangle (K^_ii before the level's in-place Cholesky), mode 1 the
// lower triangle with zeros above (the Cholesky factor L_ii afterwards).
__global__ void silSymCopyKernel(const SilCopyDesc* __restrict__ d, const TileRef* __restrict__ tiles) {
    const TileRef t = tiles[blockIdx.x];
    const SilCopyDesc D = d[t.desc];
    const int r = t.m0 + threadIdx.x, c0 = t.n0;
    if (r >= D.n) return;
    for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
        const int c = c0 + cc;
        if (c >= D.n) break;
        const double v = (r >= c) ? D.src[r + (int64_t)c * D.ld]
                                  : (D.mode == 0 ? D.src[c + (int64_t)r * D.ld] : 0.0);
        D.dst[r + (int64_t)c * D.n] = v;
    }
}

cudaError_t launchSilSymCopy(const SilCopyDesc* d, const TileRef* tiles, int nTiles, cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    silSymCopyKernel<<<nTiles, dim3(32, 8), 0, s>>>(d, tiles);
    return cudaGetLastError();
}

// nonzero values of each block (one CTA per block; integer sums, exact)
__global__ void __launch_bounds__(256) silCountKernel(const SilCountDesc* __restrict__ d,
                                                      unsigned long long* __restrict__ count) {
    const SilCountDesc D = d[blockIdx.x];
    const int64_t nn = (int64_t)D.n * D.n;
    unsigned long long c = 0;
    for (int64_t q = threadIdx.x; q < nn; q += blockDim.x) {
        const int r = (int)(q % D.n), col = (int)(q / D.n);
        c += D.F[r + (int64_t)col * D.ld] != 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(count + blockIdx.x, c);
}

cudaError_t launchSilCountNonzero(const SilCountDesc* d, int nDesc, unsigned long long* count, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned long long) * (size_t)nDesc, s);
    if (e != cudaSuccess) return e;
    silCountKernel<<<nDesc, 256, 0, s>>>(d, count);
    return cudaGetLastError();
}

// One CTA per node: sigma from the largest |K^_jj| (A holds K^), then
// A <- A - sigma M^ (M^ from the M front's lower triangle).
__global__ void __launch_bounds__(256) silShiftKernel(const SilShiftDesc* __restrict__ d) {
    __shared__ double red[32];
    const SilShiftDesc D = d[blockIdx.x];
    const int n = D.n;
    double mx = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) mx = fmax(mx, fabs(D.A[j + (int64_t)j * n]));
    mx = blockMax(mx, red);
    const double sigma = -fmax(1e-10, 1e-9 * (mx > 0.0 ? mx : 1.0));
    if (threadIdx.x == 0) *D.sigma = sigma;
    const int64_t nn = (int64_t)n * n;
    for (int64_t q = threadIdx.x; q < nn; q += blockDim.x) {
        const int r = (int)(q % n), c = (int)(q / n);
        const double m = (r >= c) ? D.M[r + (int64_t)c * D.ldm] : D.M[c + (int64_t)r * D.ldm];
        D.A[q] -= sigma * m;
    }
}

cudaError_t launchSilShift(const SilShiftDesc* d, int nDesc, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    silShiftKernel<<<nDesc, 256, 0, s>>>(d);
    return cudaGetLastError();
}

// The Lanczos iteration (see the file comment).  Every node with
// active != 0 runs steps until state[0] (steps done) reaches `target` or a
// breakdown (beta < 1e-13) sets state[1].  A node with no step done first
// builds q_0 from the start vector.
//
// At the start of the launch and of every step each CTA reads the nodes'
// states once into a shared table: which nodes take part, their step j, and
// exclusive prefix sums of their row units (n) and basis units (j + 1).  A
// phase's units are numbered over the table and dealt round-robin to the
// grid's warps, which find their node by binary search in the prefix sums,
// so a phase costs O(log nodes) per unit instead of a scan of all nodes.
namespace {
struct SilTable {
    int* live;      // node takes part in this step (or, before the loop, is fresh)
    int* j;         // its step count
    int* rowPre;    // nDesc + 1: prefix of n over live nodes
    int* basPre;    // nDesc + 1: prefix of j + 1 over live nodes
};

// exclusive prefix sum of v[0..n) into pre[0..n] by one CTA (chunked per
// thread, then a scan of the per-thread totals through shared memory)
__device__ __forceinline__ void ctaScan(const int* v, int* pre, int n, int* tot) {
    const int t = threadIdx.x, T = blockDim.x;
    const int per = (n + T - 1) / T, b0 = min(n, t * per), b1 = min(n, b0 + per);
    int sum = 0;
    for (int i = b0; i < b1; ++i) sum += v[i];
    tot[t] = sum;
    __syncthreads();
    if (t == 0) {
        int run = 0;
        for (int k = 0; k < T; ++k) {
            const int x = tot[k];
            tot[k] = run;
            run += x;
        }
        pre[n] = run;
    }
    __syncthreads();
    int run = tot[t];
    for (int i = b0; i < b1; ++i) {
        pre[i] = run;
        run += v[i];
    }
    __syncthreads();
}

// last node b with pre[b] <= U (pre non-decreasing, pre[0] = 0 <= U < pre[n])
__device__ __forceinline__ int silFind(const int* pre, int n, int U) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= U) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class F>
__device__ __forceinline__ void forRows(const SilTable& T, int nDesc, int gw, int tw, F&& f) {
    const int total = T.rowPre[nDesc];
    for (int U = gw; U < total; U += tw) {
        const int b = silFind(T.rowPre, nDesc, U);
        f(b, U - T.rowPre[b], T.j[b]);
    }
}

template <class F>
__device__ __forceinline__ void forBasis(const SilTable& T, int nDesc, int gw, int tw, F&& f) {
    const int total = T.basPre[nDesc];
    for (int U = gw; U < total; U += tw) {
        const int b = silFind(T.basPre, nDesc, U);
        f(b, U - T.basPre[b], T.j[b]);
    }
}
}  // namespace

__global__ void __launch_bounds__(kSilThreads) silLanczosKernel(const SilDesc* __restrict__ D, int nDesc,
                                                                  int maxSteps) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ int silSm[];
    __shared__ double red[32];
    __shared__ int tot[kSilThreads];
    __shared__ int anyLive;
    SilTable T;
    T.live = silSm;
    T.j = silSm + nDesc;
    T.rowPre = silSm + 2 * nDesc;
    T.basPre = silSm + 3 * nDesc + 1;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kSilWarps + (threadIdx.x >> 5);
    const int tw = gridDim.x * kSilWarps;

    // the table from the nodes' states: mode 0 = fresh nodes (no step done),
    // mode 1 = nodes live in this step; row units in rowPre, basis units in
    // basPre (T.j doubles as the unit buffer for each scan in turn)
    auto buildTable = [&](int mode) {
        for (int b = threadIdx.x; b < nDesc; b += blockDim.x) {
            const SilDesc& d = D[b];
            const int s0 = __ldcg(d.state), s1 = __ldcg(d.state + 1);
            const bool on = mode == 0 ? (d.active && s0 == 0 && d.target > 0)
                                      : (d.active && s1 == 0 && s0 < d.target);
            T.live[b] = on ? 1 : 0;
            T.j[b] = on ? d.n : 0;          // row units, scanned first
        }
        __syncthreads();
        ctaScan(T.j, T.rowPre, nDesc, tot);
        for (int b = threadIdx.x; b < nDesc; b += blockDim.x)
            T.j[b] = T.live[b] ? __ldcg(D[b].state) + 1 : 0;   // basis units
        __syncthreads();
        ctaScan(T.j, T.basPre, nDesc, tot);
        for (int b = threadIdx.x; b < nDesc; b += blockDim.x) T.j[b] = __ldcg(D[b].state);
        if (threadIdx.x == 0) anyLive = T.rowPre[nDesc] > 0;
        __syncthreads();
    };

    // mw = M^ w for the table's nodes (warp per row)
    auto mprod = [&]() {
        forRows(T, nDesc, gw, tw, [&](int b, int u, int) {
            const SilDesc& d = D[b];
            double acc = 0.0;
            for (int e = d.mRow[u] + lane; e < d.mRow[u + 1]; e += 32)
                acc = fma(d.mBase[d.mOff[e]], __ldcg(d.w + d.mCol[e]), acc);
            acc = warpSum<32>(acc);
            if (lane == 0) d.mw[u] = acc;
        });
    };

    // ---- start vector for nodes with no step done ----
    buildTable(0);
    for (int b = 0; b < nDesc; ++b) {
        if (!T.live[b]) continue;
        const SilDesc& d = D[b];
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < d.n; r += gridDim.x * blockDim.x) {
            const uint32_t x = lcgState(12345u, (uint32_t)r + 1u);
            // Eigen 3.4 Random: -1 + 2 rand() / RAND_MAX, RAND_MAX = 0x7fff
            d.w[r] = -1.0 + 2.0 * (double)((x >> 16) & 0x7fffu) / 32767.0;
        }
    }
    grid.sync();
    mprod();
    grid.sync();
    for (int b = blockIdx.x; b < nDesc; b += gridDim.x) {
        if (!T.live[b]) continue;
        const SilDesc& d = D[b];
        double s2 = 0.0;
        for (int r = threadIdx.x; r < d.n; r += blockDim.x) s2 += __ldcg(d.w + r) * __ldcg(d.mw + r);
        s2 = blockSum(s2, red);
        const double inv = 1.0 / sqrt(fmax(s2, 1e-300));
        for (int r = threadIdx.x; r < d.n; r += blockDim.x) {
            const double q = __ldcg(d.w + r) * inv;
            d.Q[r] = q;
            d.QT[(int64_t)r * d.n] = q;
            d.MQ[r] = __ldcg(d.mw + r) * inv;
        }
    }
    grid.sync();

    for (int step = 0; step < maxSteps; ++step) {
        // the same table in every CTA (states read after the barrier)
        buildTable(1);
        if (!anyLive) break;
        // P1: w = B (M q_j)    (warp per row; B symmetric: row r = column r)
        forRows(T, nDesc, gw, tw, [&](int b, int u, int j) {
            const SilDesc& d = D[b];
            const double* bc = d.B + (int64_t)u * d.n;
            const double* mq = d.MQ + (int64_t)j * d.n;
            double acc = 0.0;
            for (int c = lane; c < d.n; c += 32) acc = fma(__ldg(bc + c), __ldcg(mq + c), acc);
            acc = warpSum<32>(acc);
            if (lane == 0) d.w[u] = acc;
        });
        grid.sync();
        for (int pass = 0; pass < 2; ++pass) {
            // P2/P4: coef_l = (M q_l)^T w, l = 0 .. j (warp per l); alpha_j from the first pass
            forBasis(T, nDesc, gw, tw, [&](int b, int u, int j) {
                const SilDesc& d = D[b];
                const double* mq = d.MQ + (int64_t)u * d.n;
                double acc = 0.0;
                for (int r = lane; r < d.n; r += 32) acc = fma(__ldcg(mq + r), __ldcg(d.w + r), acc);
                acc = warpSum<32>(acc);
                if (lane == 0) {
                    d.coef[u] = acc;
                    if (pass == 0 && u == j) d.alpha[j] = acc;
                }
            });
            grid.sync();
            // P3/P5: w -= Q coef (warp per row, contiguous over l in Q^T)
            forRows(T, nDesc, gw, tw, [&](int b, int u, int j) {
                const SilDesc& d = D[b];
                const double* qt = d.QT + (int64_t)u * d.n;
                double acc = 0.0;
                for (int l = lane; l <= j; l += 32) acc = fma(__ldcg(qt + l), __ldcg(d.coef + l), acc);
                acc = warpSum<32>(acc);
                if (lane == 0) d.w[u] = __ldcg(d.w + u) - acc;
            });
            grid.sync();
        }
        // P6: mw = M^ w
        mprod();
        grid.sync();
        // P7: beta_j = ||w||_M, q_{j+1} = w / beta_j (CTA per node)
        for (int b = blockIdx.x; b < nDesc; b += gridDim.x) {
            if (!T.live[b]) continue;
            const SilDesc& d = D[b];
            const int j = T.j[b];
            double s2 = 0.0;
            for (int r = threadIdx.x; r < d.n; r += blockDim.x) s2 += __ldcg(d.w + r) * __ldcg(d.mw + r);
            s2 = blockSum(s2, red);
            const double bj = sqrt(fmax(s2, 0.0));
            const bool brk = bj < 1e-13;
            if (!brk && j + 1 < d.n) {
                const double inv = 1.0 / bj;
                double* qn = d.Q + (int64_t)(j + 1) * d.n;
                double* mqn = d.MQ + (int64_t)(j + 1) * d.n;
                for (int r = threadIdx.x; r < d.n; r += blockDim.x) {
                    const double q = __ldcg(d.w + r) * inv;
                    qn[r] = q;
                    d.QT[j + 1 + (int64_t)r * d.n] = q;
                    mqn[r] = __ldcg(d.mw + r) * inv;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                d.beta[j] = brk ? 0.0 : bj;
                if (brk || j + 1 >= d.n) d.state[1] = 1;
                d.state[0] = j + 1;
            }
        }
        grid.sync();
    }
}

namespace {
// nodes per cooperative launch (the shared table holds 4 ints per node)
constexpr int kSilMaxDesc = 4096;

int silLanczosMaxCtas(size_t smem) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, silLanczosKernel, kSilThreads, smem);
    if (per > 4) per = 4;
    return per * sms;
}
}  // namespace

cudaError_t launchSilLanczos(const SilDesc* d, int nDesc, int maxSteps, cudaStream_t s) {
    // independent nodes: chunks of at most kSilMaxDesc, one launch each
    for (int b0 = 0; b0 < nDesc; b0 += kSilMaxDesc) {
        int nb = nDesc - b0 < kSilMaxDesc ? nDesc - b0 : kSilMaxDesc;
        const size_t smem = sizeof(int) * (4 * static_cast<size_t>(nb) + 2);
        if (smem > 48 * 1024) {
            const cudaError_t e = cudaFuncSetAttribute(silLanczosKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(smem));
            if (e != cudaSuccess) return e;
        }
        const int nCta = silLanczosMaxCtas(smem);
        if (nCta < 1) return cudaErrorCooperativeLaunchTooLarge;
        const SilDesc* dc = d + b0;
        void* args[] = {(void*)&dc, (void*)&nb, (void*)&maxSteps};
        const cudaError_t e = cudaLaunchCooperativeKernel((void*)silLanczosKernel, dim3(nCta), dim3(kSilThreads), args,
                                                          smem, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Count thresholds and Ritz scalings.  thr[b] = 1 / (hi_b - sigma_b): a Ritz
// value lambda = 1/nu + sigma is <= hi exactly when nu >= thr[b] (+inf when
// hi_b <= sigma_b: none is).
__global__ void silThresholdKernel(const double* __restrict__ sigma, int nDesc, const double* __restrict__ hi,
                                   double* __restrict__ thr) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nDesc) return;
    const double g = hi[b] - sigma[b];
    thr[b] = g > 0.0 ? 1.0 / g : INFINITY;
}

cudaError_t launchSilThreshold(const double* sigma, int nDesc, const double* hi, double* thr, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    silThresholdKernel<<<(nDesc + 127) / 128, 128, 0, s>>>(sigma, nDesc, hi, thr);
    return cudaGetLastError();
}

// Per selected Ritz pair t of node b (nu descending): lambda = 1/nu + sigma,
// rs[t] = lambda^-1/2 (scales of the engine's local vectors) and
// wEng[t] = 1/lambda (the engine's nu of the mode).
__global__ void silRitzScaleKernel(const SilRitzDesc* __restrict__ d, int nDesc) {
    const int b = blockIdx.x;
    const SilRitzDesc D = d[b];
    const int k = *D.kOut;
    for (int t = threadIdx.x; t < k; t += blockDim.x) {
        const double lam = 1.0 / D.nu[t] + *D.sigma;
        D.rs[t] = 1.0 / sqrt(lam);
        D.wEng[t] = 1.0 / lam;
    }
}

cudaError_t launchSilRitzScale(const SilRitzDesc* d, int nDesc, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    silRitzScaleKernel<<<nDesc, 128, 0, s>>>(d, nDesc);
    return cudaGetLastError();
}

}  // namespace amls_b200
