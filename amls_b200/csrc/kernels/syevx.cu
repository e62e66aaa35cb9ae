// FP64 symmetric eigensolver for selected eigenpairs, batched.
//
// This is the device replacement of LAPACK's dsygvx path used by the
// reference for every local and reduced eigenproblem
// (src/linalg/dense_eigensolver.cpp:44-133): after the pencil has been
// reduced to a standard symmetric matrix (see engine), the steps are the
// classical ones - Householder tridiagonalisation (dsytrd), bisection on
// Sturm counts for the selected eigenvalues (dstebz), inverse iteration with
// reorthogonalisation inside clusters (dstein) and back-transformation by
// the reflectors (dormtr) - each written for the GPU:
//   * tridiagSmall:  one CTA per matrix (batched), trailing matrix in L2;
//   * tridiagLarge:  cooperative launch, the grid split into CTA groups, one
//                    group per matrix, one grid barrier per column step;
//   * bisect:        multisection, one warp (32 Sturm counts per round) per
//                    wanted eigenvalue; division-free Sturm counts;
//   * inverseIter:   one warp-sized CTA per cluster, members solved in
//                    sequence, the tridiagonal LU/solve on one thread with
//                    its operands staged through shared memory, the
//                    reorthogonalisation and norms warp-parallel;
//   * backTransform: columns and the reflector in shared memory (n <= 384),
//                    blocked compact-WY GEMMs above (host/eig_wy.cpp).
#include <cooperative_groups.h>

#include <cfloat>

#include "common.cuh"
#include "launch.hpp"

namespace cg = cooperative_groups;

namespace amls_b200 {

namespace {
constexpr int kSmallThreads = 768;
constexpr int kSmallPerLane = (kTridiagSmallMax + 31) / 32;   // column loads per lane
}

// ------------------------------------------------------------------------
// Householder step helpers
// ------------------------------------------------------------------------
struct HouseholderScalars {
    double beta, tau, scale;  // v = [1, x[1:] * scale]
};

// dlarfg on x = A[k+1:n, k] (alpha = x[0], xnorm2 = |x[1:]|^2).
__device__ __forceinline__ HouseholderScalars makeReflector(double alpha, double xnorm2) {
    HouseholderScalars h;
    if (xnorm2 == 0.0) {
        h.beta = alpha;
        h.tau = 0.0;
        h.scale = 0.0;
    } else {
        const double nrm = sqrt(alpha * alpha + xnorm2);
        h.beta = alpha >= 0.0 ? -nrm : nrm;
        h.tau = (h.beta - alpha) / h.beta;
        h.scale = 1.0 / (alpha - h.beta);
    }
    return h;
}

// ------------------------------------------------------------------------
// tridiagonalisation, one CTA per matrix
// ------------------------------------------------------------------------
// The one-CTA form of the fused step of tridiagLargeKernel: per column one
// read-modify-write pass over the trailing matrix, in which each warp
// applies step k's rank-2 update to a whole column and dots it with the next
// reflector (p_{k+1}[j] directly, no atomics), and __syncthreads for the
// barrier.  n <= kTridiagSmallMax.
__global__ void __launch_bounds__(kSmallThreads) tridiagSmallKernel(const EigDesc* __restrict__ descs) {
    __shared__ double v0[kTridiagSmallMax], v1[kTridiagSmallMax], sw[kTridiagSmallMax];
    __shared__ double p0[kTridiagSmallMax], p1[kTridiagSmallMax];
    __shared__ double red[32];
    __shared__ double red2[64];
    const EigDesc D = descs[blockIdx.x];
    const int n = D.n;
    double* A = D.A;
    const int64_t lda = D.lda;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    const int bd = blockDim.x;
    double *vcur = v0, *vnext = v1, *p = p0, *pn = p1;
    if (n <= 2) {
        if (tid == 0) {
            if (n >= 1) D.d[0] = A[0];
            if (n == 2) {
                D.e[0] = A[1];
                D.tau[0] = 0.0;
                D.d[1] = A[1 + lda];
            }
        }
        return;
    }
    // reflector 0 and p_0 = tau_0 A22 v_0
    HouseholderScalars h;
    {
        const int m = n - 1;
        const double* col = A + 1;
        double part = 0.0;
        for (int i = 1 + tid; i < m; i += bd) part += col[i] * col[i];
        h = makeReflector(col[0], blockSum(part, red));
        for (int i = tid; i < m; i += bd) vcur[i] = (i == 0) ? 1.0 : col[i] * h.scale;
        __syncthreads();
        const double* A22 = A + 1 + lda;
        for (int j = wid; j < m; j += nw) {
            const double* cj = A22 + (int64_t)j * lda;
            double sum = 0.0;
            for (int i = lane; i < m; i += 32) sum += cj[i] * vcur[i];
            sum = warpSum<32>(sum);
            if (lane == 0) p[j] = h.tau * sum;
        }
        __syncthreads();
    }
    int par = 0;
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1, m1 = m - 1;
        double* B = A + (k + 1) + (int64_t)(k + 1) * lda;
        // w = p - tau/2 (p . v) v and the updated first column of B in the
        // registers of the thread owning each index (as tridiagLargeKernel)
        const double bFirst = B[0], bSecond = B[1];
        double pv = 0.0;
        for (int i = tid; i < m; i += bd) {
            pv += p[i] * vcur[i];
            if (i >= 2) vnext[i - 1] = B[i];
        }
        pv = blockSum1(pv, red2, par);
        const double a2 = -0.5 * h.tau * pv;
        const double w0 = p[0] + a2 * vcur[0];
        double part = 0.0;
        for (int i = tid; i < m; i += bd) {
            const double wi = p[i] + a2 * vcur[i];
            sw[i] = wi;
            if (i >= 2) {
                const double b = vnext[i - 1] - (vcur[i] * w0 + wi);
                vnext[i - 1] = b;
                part += b * b;
            }
        }
        const double w1 = p[1] + a2 * vcur[1];
        const double b00 = bFirst - (w0 + w0);
        const double alpha = bSecond - (vcur[1] * w0 + w1);
        HouseholderScalars hn{0.0, 0.0, 0.0};
        if (m1 >= 2) {
            // the reduction's barrier orders every vnext write before the scaling
            hn = makeReflector(alpha, blockSum1(part, red2, par));
            for (int i = 1 + tid; i < m1; i += bd) vnext[i] *= hn.scale;
            if (tid == 0) vnext[0] = 1.0;
        }
        __syncthreads();
        {
            double* col = A + (k + 1) + (int64_t)k * lda;
            for (int i = tid; i < m; i += bd) col[i] = vcur[i];
            if (tid == 0) {
                if (k == 0) D.d[0] = A[0];
                D.e[k] = h.beta;
                D.tau[k] = h.tau;
                D.d[k + 1] = b00;
                if (m1 < 2) {
                    D.e[k + 1] = alpha;
                    D.tau[k + 1] = 0.0;
                    D.d[k + 2] = B[1 + lda] - 2.0 * vcur[1] * w1;
                }
            }
        }
        if (m1 >= 2) {
            double* C = B + 1 + lda;
            const double* vp = vcur + 1;
            const double* wp = sw + 1;
            const bool upd = h.tau != 0.0;
            // one warp per column; the whole column (m1 <= 383) is loaded in
            // one batch of kSmallPerLane loads per lane
            for (int j = wid; j < m1; j += nw) {
                double* cj = C + (int64_t)j * lda;
                const double vj = vp[j], wj = wp[j];
                double cv[kSmallPerLane];
#pragma unroll
                for (int t = 0; t < kSmallPerLane; ++t) {
                    const int i = lane + 32 * t;
                    cv[t] = i < m1 ? cj[i] : 0.0;
                }
                double sum = 0.0;
#pragma unroll
                for (int t = 0; t < kSmallPerLane; ++t) {
                    const int i = lane + 32 * t;
                    if (i < m1) {
                        double c = cv[t];
                        if (upd) {
                            c -= vp[i] * wj + wp[i] * vj;
                            cj[i] = c;
                        }
                        sum += c * vnext[i];
                    }
                }
                sum = warpSum<32>(sum);
                if (lane == 0) pn[j] = hn.tau * sum;
            }
        }
        h = hn;
        double* t = vcur;
        vcur = vnext;
        vnext = t;
        t = p;
        p = pn;
        pn = t;
        __syncthreads();
    }
}

cudaError_t launchTridiagSmall(const EigDesc* d, int nDesc, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    tridiagSmallKernel<<<nDesc, kSmallThreads, 0, s>>>(d);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// tridiagonalisation, cooperative, grid split into groups (one per matrix)
// ------------------------------------------------------------------------
struct LargeArgs {
    const EigDesc* descs;     // device
    const int* groupOf;       // CTA -> group (matrix)
    const int* groupFirst;    // first CTA of each group
    const int* groupSize;     // CTAs in each group
    double* pbuf;             // per matrix kTridiagPBufs * n doubles (offsets kTridiagPBufs * pOff)
    const int64_t* pOff;
    int maxN;
};

// One grid barrier per column.  Entering step k every CTA of the group holds
// the reflector v_k (tau_k) in shared memory and p_k = tau_k A22 v_k is
// complete in global memory (A22 = the trailing matrix before step k's
// rank-2 update).  Each CTA then forms, redundantly and in the same order
// (so all CTAs agree bit for bit),
//   w_k = p_k - tau_k/2 (p_k . v_k) v_k,
//   the updated first column of A22 and from it the next reflector v_{k+1};
// after which units (column j, 256-row segment) of the next trailing matrix
// are updated in place (A -= v w^T + w v^T) and dotted with v_{k+1} in the
// same pass, accumulating p_{k+1} with atomics.  The trailing matrix is thus
// read and written once per column.  Three rotating p accumulators: step k
// reads p_k, adds into p_{k+1} and clears the buffer of p_{k+2}.  Output as
// the one-CTA kernel: d, e, tau and the reflectors below the subdiagonal.
__global__ void __launch_bounds__(kTridiagLargeThreads) tridiagLargeKernel(LargeArgs a) {
    extern __shared__ double sm[];   // vA (maxN), vB (maxN), w (maxN)
    __shared__ double red[32];
    __shared__ double red2[64];
    int par = 0;
    constexpr int SEG = 256;
    cg::grid_group grid = cg::this_grid();
    const int g = a.groupOf[blockIdx.x];
    const int rank = blockIdx.x - a.groupFirst[g];
    const int gsize = a.groupSize[g];
    const EigDesc D = a.descs[g];
    const int n = D.n;
    double* A = D.A;
    const int64_t lda = D.lda;
    double* pbase = a.pbuf + (int64_t)kTridiagPBufs * a.pOff[g];
    double* vcur = sm;
    double* vnext = sm + a.maxN;
    double* sw = sm + 2 * a.maxN;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    const int bd = blockDim.x;
    const int gw = rank * nw + wid, GW = gsize * nw;
    const int gt = rank * bd + tid, GT = gsize * bd;

    // accumulators cleared; reflector v_0 from column 0
    for (int i = gt; i < kTridiagPBufs * n; i += GT) pbase[i] = 0.0;
    HouseholderScalars h{0.0, 0.0, 0.0};
    if (n >= 3) {
        const int m = n - 1;
        const double* col = A + 1;
        double part = 0.0;
        for (int i = 1 + tid; i < m; i += bd) part += col[i] * col[i];
        h = makeReflector(col[0], blockSum(part, red));
        for (int i = tid; i < m; i += bd) vcur[i] = (i == 0) ? 1.0 : col[i] * h.scale;
    }
    grid.sync();
    // p_0 = tau_0 A22 v_0
    if (n >= 3 && h.tau != 0.0) {
        const int m = n - 1, segs = (m + SEG - 1) / SEG;
        const double* A22 = A + 1 + lda;
        for (int u = gw; u < m * segs; u += GW) {
            const int j = u / segs, s0 = (u % segs) * SEG;
            const int s1 = min(m, s0 + SEG);
            const double* cj = A22 + (int64_t)j * lda;
            double sum = 0.0;
#pragma unroll 4
            for (int i = s0 + lane; i < s1; i += 32) sum += cj[i] * vcur[i];
            sum = warpSum<32>(sum);
            if (lane == 0) atomicAdd(pbase + j, h.tau * sum);
        }
    }
    grid.sync();
    for (int k = 0; k + 2 < a.maxN; ++k) {
        if (k + 2 < n) {
            const int m = n - k - 1;        // order of the trailing matrix B = A22
            const int m1 = m - 1;           // order of the next one, C = B(1:, 1:)
            const double* p = pbase + (int64_t)(k % kTridiagPBufs) * n;
            double* B = A + (k + 1) + (int64_t)(k + 1) * lda;
            // p_k and the first column of B are loaded together; then, in the
            // registers of the thread owning each index, w = p - tau/2 (p . v) v
            // and the updated first column b0 = B(:,0) - v w0 - w v0 (v0 = 1),
            // from whose tail the next reflector is built.  Two one-barrier
            // reductions and one barrier per column inside the CTA.
            const double pFirst = p[0], pSecond = p[1], bFirst = B[0], bSecond = B[1];
            double pv = 0.0;
            for (int i = tid; i < m; i += bd) {
                const double pi = p[i];
                sw[i] = pi;
                pv += pi * vcur[i];
                if (i >= 2) vnext[i - 1] = B[i];
            }
            pv = blockSum1(pv, red2, par);
            const double a2 = -0.5 * h.tau * pv;
            const double v0 = vcur[0];
            const double w0 = pFirst + a2 * v0;
            double part = 0.0;
            for (int i = tid; i < m; i += bd) {
                const double wi = sw[i] + a2 * vcur[i];
                sw[i] = wi;
                if (i >= 2) {
                    const double b = vnext[i - 1] - (vcur[i] * w0 + wi * v0);
                    vnext[i - 1] = b;
                    part += b * b;
                }
            }
            const double w1 = pSecond + a2 * vcur[1];
            const double b00 = bFirst - (v0 * w0 + w0 * v0);
            const double alpha = bSecond - (vcur[1] * w0 + w1 * v0);
            HouseholderScalars hn{0.0, 0.0, 0.0};
            if (m1 >= 2) {
                // the reduction's barrier orders every vnext write before the scaling
                hn = makeReflector(alpha, blockSum1(part, red2, par));
                for (int i = 1 + tid; i < m1; i += bd) vnext[i] *= hn.scale;
                if (tid == 0) vnext[0] = 1.0;
            }
            __syncthreads();
            if (rank == 0) {
                // reflector k into column k; nothing else reads that column now
                double* col = A + (k + 1) + (int64_t)k * lda;
                for (int i = tid; i < m; i += bd) col[i] = vcur[i];
                if (tid == 0) {
                    if (k == 0) D.d[0] = A[0];
                    D.e[k] = h.beta;
                    D.tau[k] = h.tau;
                    D.d[k + 1] = b00;
                    if (m1 < 2) {           // last column step: the 2 x 2 tail
                        D.e[k + 1] = alpha;
                        D.tau[k + 1] = 0.0;
                        D.d[k + 2] = B[1 + lda] - (vcur[1] * w1 + w1 * vcur[1]);
                    }
                }
            }
            if (m1 >= 2) {
                const int segs = (m1 + SEG - 1) / SEG;
                double* C = B + 1 + lda;
                const double* vp = vcur + 1;
                const double* wp = sw + 1;
                double* pn = pbase + (int64_t)((k + 1) % kTridiagPBufs) * n;
                const bool upd = h.tau != 0.0;
                for (int u = gw; u < m1 * segs; u += GW) {
                    const int j = u / segs, s0 = (u % segs) * SEG;
                    const int s1 = min(m1, s0 + SEG);
                    double* cj = C + (int64_t)j * lda;
                    const double vj = vp[j], wj = wp[j];
                    double sum = 0.0;
                    // SEG / 32 = 8 loads per lane issued together
                    double cv[SEG / 32];
#pragma unroll
                    for (int t = 0; t < SEG / 32; ++t) {
                        const int i = s0 + lane + 32 * t;
                        cv[t] = i < s1 ? cj[i] : 0.0;
                    }
#pragma unroll
                    for (int t = 0; t < SEG / 32; ++t) {
                        const int i = s0 + lane + 32 * t;
                        if (i < s1) {
                            double c = cv[t];
                            if (upd) {
                                c -= vp[i] * wj + wp[i] * vj;
                                cj[i] = c;
                            }
                            sum += c * vnext[i];
                        }
                    }
                    sum = warpSum<32>(sum);
                    if (lane == 0 && hn.tau != 0.0) atomicAdd(pn + j, hn.tau * sum);
                }
            }
            // the accumulator of step k+2 (last read at step k-1)
            double* pc = pbase + (int64_t)((k + 2) % kTridiagPBufs) * n;
            for (int i = gt; i < n; i += GT) pc[i] = 0.0;
            h = hn;
            double* t = vcur;
            vcur = vnext;
            vnext = t;
        }
        grid.sync();
    }
    if (rank == 0 && tid == 0 && n <= 2) {
        D.d[0] = A[0];
        if (n == 2) {
            D.e[0] = A[1];
            D.tau[0] = 0.0;
            D.d[1] = A[1 + lda];
        }
    }
}

cudaError_t launchTridiagLargeGroups(const EigDesc* dDescs, const int* dGroupOf,
                                     const int* dGroupFirst, const int* dGroupSize, int nCta,
                                     double* dP, const int64_t* dPOff, int maxN, cudaStream_t s) {
    LargeArgs a{dDescs, dGroupOf, dGroupFirst, dGroupSize, dP, dPOff, maxN};
    void* args[] = {&a};
    const size_t smem = 3 * (size_t)maxN * sizeof(double);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(tridiagLargeKernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaLaunchCooperativeKernel((void*)tridiagLargeKernel, dim3(nCta),
                                       dim3(kTridiagLargeThreads), args, smem, s);
}

int tridiagLargeMaxCtas(int maxN) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = 3 * (size_t)maxN * sizeof(double);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(tridiagLargeKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tridiagLargeKernel, kTridiagLargeThreads, smem);
    if (per > 1) per = 1;
    return per * sms;
}

// ------------------------------------------------------------------------
// bisection (Sturm counts)
// ------------------------------------------------------------------------
// Number of eigenvalues of T below x: the sign changes of the Sturm
// sequence of leading principal minors
//   p_{-1} = 1, p_0 = d_0 - x, p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2},
// i.e. the ratios q_i = p_i / p_{i-1} = (d_i - x) - e_{i-1}^2 / q_{i-1} of
// LAPACK's dstebz counted negative, but without a division on the serial
// chain (one FMA and a guard per step).  T is scaled by s = 2^-k >= 1/|T|
// (exact), so |d_i - x| <= 4 and e^2 <= 1 after scaling; a ratio smaller
// than piv = max(s pivmin, 2^-100) in magnitude is replaced by -piv (dstebz's
// pivmin rule, moving d_i by at most 2^-100 |T|), which bounds |q| to
// [2^-100, 2^101] and lets (p_{i-1}, p_i) be rescaled by a power of two
// only every fourth step.
__device__ __forceinline__ int sturmLess(const double* __restrict__ d, const double* __restrict__ e, int n,
                                         double x, double pivmin, double tnorm) {
    int k = 0;
    frexp(tnorm > 0.0 ? tnorm : 1.0, &k);
    const double s = ldexp(1.0, -k), s2 = s * s;
    const double xs = x * s;
    const double piv = fmax(pivmin * s, 0x1p-100);
    double p2 = 1.0;                       // p_{i-2}
    double p1 = fma(d[0], s, -xs);         // p_{i-1}
    if (fabs(p1) < piv) p1 = -piv;
    int cnt = p1 < 0.0;
    for (int i = 1; i < n; ++i) {
        const double t = fma(d[i], s, -xs);
        const double c = e[i - 1] * e[i - 1] * s2;
        double pn = fma(t, p1, -c * p2);
        if (fabs(pn) < piv * fabs(p1)) pn = -piv * p1;
        cnt += (pn < 0.0) != (p1 < 0.0);
        p2 = p1;
        p1 = pn;
        if ((i & 3) == 0) {
            // rescale by 2^-(exponent of p1); |p2 / p1| lies in [2^-101, 2^100]
            const int ex = (__double2hiint(p1) >> 20) & 0x7ff;
            const double sc = __hiloint2double((2046 - ex) << 20, 0);
            p1 *= sc;
            p2 *= sc;
        }
    }
    return cnt;
}

__device__ void gershgorin(const double* d, const double* e, int n, double& lo, double& hi,
                           double& pivmin, double& tnorm) {
    lo = DBL_MAX;
    hi = -DBL_MAX;
    double emax2 = 0.0;
    tnorm = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
        lo = fmin(lo, d[i] - r);
        hi = fmax(hi, d[i] + r);
        tnorm = fmax(tnorm, fabs(d[i]) + r);
        if (i + 1 < n) emax2 = fmax(emax2, e[i] * e[i]);
    }
    pivmin = DBL_MIN * fmax(1.0, emax2);
    const double pad = 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + 2.0 * pivmin;
    lo -= pad;
    hi += pad;
}

// count kernel: kOut[b] for modes 0/2 (min(want, n, kcap)) and 1/3 (threshold)
__global__ void bisectCountKernel(const EigDesc* __restrict__ descs, int nDesc, int mode, int want,
                                  double thr, const double* __restrict__ thrArr) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nDesc) return;
    const EigDesc D = descs[b];
    const int n = D.n;
    int k;
    if (n <= 0) k = 0;
    else if (mode == 0 || mode == 2) k = min(want, n);
    else {
        double lo, hi, pivmin, tn;
        gershgorin(D.d, D.e, n, lo, hi, pivmin, tn);
        const int less = sturmLess(D.d, D.e, n, thrArr ? thrArr[b] : thr, pivmin, tn);
        k = (mode == 1) ? (n - less) : less;
    }
    *D.kOut = min(k, D.kcap);
}

__global__ void bisectKernel(const EigDesc* __restrict__ descs, int mode, int maxK) {
    const int b = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const EigDesc D = descs[b];
    const int k = *D.kOut;
    if (j >= k) return;
    const int n = D.n;
    // 1-based ascending index of the wanted eigenvalue
    const int t = (mode <= 1) ? (n - j) : (j + 1);
    double lo, hi, pivmin, tn;
    gershgorin(D.d, D.e, n, lo, hi, pivmin, tn);
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin || mid <= lo ||
            mid >= hi)
            break;
        // count(< mid) >= t  <=>  lambda_t < mid
        if (sturmLess(D.d, D.e, n, mid, pivmin, tn) >= t) hi = mid;
        else lo = mid;
    }
    D.w[j] = 0.5 * (lo + hi);
}

cudaError_t launchBisect(const EigDesc* d, int nDesc, int mode, int want, double thr, int maxK,
                         int*, cudaStream_t s, const double* thrArr) {
    if (nDesc <= 0) return cudaSuccess;
    bisectCountKernel<<<(nDesc + 127) / 128, 128, 0, s>>>(d, nDesc, mode, want, thr, thrArr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || maxK <= 0) return e;
    dim3 grid((maxK + 63) / 64, nDesc);
    bisectKernel<<<grid, 64, 0, s>>>(d, mode, maxK);
    return cudaGetLastError();
}

// count of eigenvalues >= thr[b] (descriptor b), capped by kcap
__global__ void countAboveKernel(const EigDesc* __restrict__ descs, int nDesc,
                                 const double* __restrict__ thr) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nDesc) return;
    const EigDesc D = descs[b];
    const int n = D.n;
    const double x = thr[b];
    int k = 0;
    if (n > 0 && x < INFINITY) {
        double lo, hi, pivmin, tn;
        gershgorin(D.d, D.e, n, lo, hi, pivmin, tn);
        k = n - sturmLess(D.d, D.e, n, x, pivmin, tn);
    }
    *D.kOut = min(k, D.kcap);
}

cudaError_t launchCountAbove(const EigDesc* d, int nDesc, const double* thr, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    countAboveKernel<<<(nDesc + 127) / 128, 128, 0, s>>>(d, nDesc, thr);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// inverse iteration (dlagtf / dlagts / dstein), one warp-sized CTA per cluster
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(32) inverseIterKernel(const EigDesc* __restrict__ descs,
                                                          int maxK) {
    constexpr int kIiChunk = 256;
    __shared__ double red[32];
    __shared__ double sh[4];
    __shared__ double sIn0[kIiChunk + 1], sIn1[kIiChunk + 1], sC[kIiChunk], sPiv[kIiChunk], sDd[kIiChunk],
        sB[kIiChunk], sInv[kIiChunk], sOut[kIiChunk];
    const int b = blockIdx.y;
    const int j = blockIdx.x;
    const EigDesc D = descs[b];
    const int k = *D.kOut;
    const int n = D.n;
    if (j >= k || n <= 0) return;
    const int tid = threadIdx.x;
    // T norm and cluster tolerance.  LAPACK's dstein groups eigenvalues
    // closer than 1e-3 |T|; that makes clusters of hundreds of the reduced
    // problem's eigenvalues and serialises them.  Vectors of eigenvalues
    // separated by g come out of inverse iteration orthogonal to about
    // eps |T| / g, so grouping only gaps below 1e-8 |T| keeps every pair
    // orthogonal to ~2e-8 while clusters stay rare and every vector runs
    // in parallel (one CTA each).  The inverted spectra (1 / lambda) of the
    // AMLS problems crowd their upper eigenvalues within 1e-6 |T| of each
    // other, which a wider tolerance would chain into long serial clusters.
    double lo, hi, pivmin, tnorm;
    gershgorin(D.d, D.e, n, lo, hi, pivmin, tnorm);
    const double ortol = 1e-8 * tnorm;
    // cluster start: j is a start if j == 0 or |w[j] - w[j-1]| > ortol
    if (j > 0 && fabs(D.w[j] - D.w[j - 1]) <= ortol) return;
    int jend = j + 1;
    while (jend < k && fabs(D.w[jend] - D.w[jend - 1]) <= ortol) ++jend;
    if (n == 1) {
        if (tid == 0) D.Y[0 + (int64_t)j * D.ldy] = 1.0;
        return;
    }
    // scratch: (unused), b(super), c(sub), dd(2nd super), 1/a (guarded), piv  (6n doubles)
    double* W = D.work + (int64_t)j * 6 * n;
    double* bs = W + n;
    double* c = W + 2 * n;
    double* dd = W + 3 * n;
    double* ainv = W + 4 * n;
    double* piv = W + 5 * n;
    const double eps = DBL_EPSILON;
    const double tol = fmax(eps * tnorm, DBL_MIN);
    double prevLam = 0.0;
    for (int jj = j; jj < jend; ++jj) {
        double lam = D.w[jj];
        if (jj > j) {
            // perturb away from the previous member (dstein pertol = 10 |eps * x|)
            const double pertol = 10.0 * fabs(eps * lam);
            const double dir = (D.w[jend - 1] >= D.w[j]) ? 1.0 : -1.0;  // ordering direction
            if (dir * (lam - prevLam) < pertol) lam = prevLam + dir * pertol;
        }
        prevLam = lam;
        double* x = D.Y + (int64_t)jj * D.ldy;
        // LU with partial pivoting of T - lam I (dlagtf).  The recurrence runs
        // on one thread and carries the current pivot row (ak, bk) in
        // registers; its inputs and outputs pass through shared memory in
        // chunks of kIiChunk that the whole CTA loads and stores, so the
        // serial chain never waits on global memory.  No interchange when
        // |c|/scale2 <= |a|/scale1 (compared without divisions; a zero row
        // a = b = 0 always interchanges).  ainv holds the guarded
        // reciprocals of the U diagonal.
        {
            double ak = 0.0, bk = 0.0;
            for (int k0 = 0; k0 + 1 < n; k0 += kIiChunk) {
                const int cnt = min(kIiChunk, n - 1 - k0);     // steps kk = k0 .. k0 + cnt - 1
                __syncthreads();
                for (int i = tid; i <= cnt; i += blockDim.x) {
                    const int kk = k0 + i;                      // e[kk], d[kk + 1] (i < cnt), e[kk + 1]
                    sIn0[i] = kk < n - 1 ? D.e[kk] : 0.0;
                    sIn1[i] = (i < cnt) ? D.d[kk + 1] : 0.0;
                }
                if (k0 == 0 && tid == 0) {
                    ak = D.d[0] - lam;
                    bk = D.e[0];
                }
                __syncthreads();
                if (tid == 0) {
                    // branch-free step: both pivot choices share one division
                    for (int i = 0; i < cnt; ++i) {
                        const int kk = k0 + i;
                        const double ck = sIn0[i];
                        const double a1 = sIn1[i] - lam;
                        const double b1 = (kk + 2 < n) ? sIn0[i + 1] : 0.0;
                        const double scale1 = fabs(ak) + fabs(bk);
                        const double scale2 = fabs(ck) + fabs(a1) + fabs(b1);
                        const bool keep = ck == 0.0 || scale2 == 0.0 ||
                                          (scale1 > 0.0 && fabs(ck) * scale1 <= fabs(ak) * scale2);
                        // keep: mult = c / a (0 when either is 0); swap: mult = a / c, c != 0
                        const double q = (keep ? ck : ak) / (keep ? ak : ck);
                        const double mult = (keep && (ck == 0.0 || ak == 0.0)) ? 0.0 : q;
                        const double ua = keep ? ak : ck;                       // stored U row kk
                        sPiv[i] = keep ? 0.0 : 1.0;
                        sC[i] = mult;
                        sB[i] = keep ? bk : a1;
                        sDd[i] = keep ? 0.0 : b1;
                        sInv[i] = 1.0 / (fabs(ua) < tol ? (ua >= 0.0 ? tol : -tol) : ua);
                        const double na = keep ? fma(-mult, bk, a1) : fma(-mult, a1, bk);   // carried row kk + 1
                        const double nb = keep ? b1 : -mult * b1;
                        ak = na;
                        bk = nb;
                    }
                    if (k0 + cnt == n - 1) ainv[n - 1] = 1.0 / (fabs(ak) < tol ? (ak >= 0.0 ? tol : -tol) : ak);
                }
                __syncthreads();
                for (int i = tid; i < cnt; i += blockDim.x) {
                    piv[k0 + i] = sPiv[i];
                    c[k0 + i] = sC[i];
                    dd[k0 + i] = sDd[i];
                    bs[k0 + i] = sB[i];
                    ainv[k0 + i] = sInv[i];
                }
            }
        }
        // deterministic start vector
        for (int i = tid; i < n; i += blockDim.x) {
            unsigned h = (unsigned)(i * 2654435761u) ^ (unsigned)(jj * 40503u + 12345u);
            h ^= h >> 13;
            h *= 0x5bd1e995u;
            h ^= h >> 15;
            x[i] = ((h & 0xffffff) / double(0x1000000)) - 0.5 + 1e-3;
        }
        __syncthreads();
        // three solves, as dstein takes once the growth test passes (one
        // solve reaches it from an eigenvalue accurate to eps |T|, then
        // EXTRA = 2 more)
        for (int it = 0; it < 3; ++it) {
            // apply L^-1 with interchanges, then U^-1 (dlagts, job -1): one
            // thread carries the running components in registers, the CTA
            // stages the operands and the results chunk by chunk
            double cur = 0.0;
            for (int k0 = 0; k0 + 1 < n; k0 += kIiChunk) {
                const int cnt = min(kIiChunk, n - 1 - k0);     // kk = k0 .. k0 + cnt - 1 reads x[kk + 1]
                __syncthreads();
                for (int i = tid; i < cnt; i += blockDim.x) {
                    sIn0[i] = x[k0 + i + 1];
                    sC[i] = c[k0 + i];
                    sPiv[i] = piv[k0 + i];
                }
                if (k0 == 0 && tid == 0) cur = x[0];
                __syncthreads();
                if (tid == 0) {
                    // branch-free, so that the shared-memory loads of later
                    // steps issue ahead of the dependent chain
#pragma unroll 8
                    for (int i = 0; i < cnt; ++i) {
                        const double nxt = sIn0[i], ci = sC[i];
                        const bool sw = sPiv[i] != 0.0;
                        sOut[i] = sw ? nxt : cur;
                        cur = sw ? fma(-ci, nxt, cur) : fma(-ci, cur, nxt);
                    }
                    if (k0 + cnt == n - 1) x[n - 1] = cur;
                }
                __syncthreads();
                for (int i = tid; i < cnt; i += blockDim.x) x[k0 + i] = sOut[i];
            }
            double x1 = 0.0, x2 = 0.0;     // x[kk + 1], x[kk + 2] of the result
            for (int k1 = n; k1 > 0; k1 -= kIiChunk) {
                const int k0 = max(0, k1 - kIiChunk), cnt = k1 - k0;
                __syncthreads();
                for (int i = tid; i < cnt; i += blockDim.x) {
                    const int kk = k0 + i;
                    sIn0[i] = x[kk];
                    sB[i] = kk + 1 < n ? bs[kk] : 0.0;       // U's superdiagonals end at n-2, n-3
                    sDd[i] = kk + 2 < n ? dd[kk] : 0.0;
                    sInv[i] = ainv[kk];
                }
                __syncthreads();
                if (tid == 0) {
#pragma unroll 8
                    for (int i = cnt - 1; i >= 0; --i) {
                        const double t = fma(-sB[i], x1, fma(-sDd[i], x2, sIn0[i]));
                        const double v = t * sInv[i];
                        sOut[i] = v;
                        x2 = x1;
                        x1 = v;
                    }
                }
                __syncthreads();
                for (int i = tid; i < cnt; i += blockDim.x) x[k0 + i] = sOut[i];
            }
            __syncthreads();
            // reorthogonalise against earlier members of the cluster (MGS)
            for (int q = j; q < jj; ++q) {
                const double* xq = D.Y + (int64_t)q * D.ldy;
                double part = 0.0;
                for (int i = tid; i < n; i += blockDim.x) part += xq[i] * x[i];
                const double dot = blockSum(part, red);
                for (int i = tid; i < n; i += blockDim.x) x[i] -= dot * xq[i];
                __syncthreads();
            }
            // normalise (2-norm), guard against overflow by max-scaling first
            double mx = 0.0;
            for (int i = tid; i < n; i += blockDim.x) mx = fmax(mx, fabs(x[i]));
            mx = blockMax(mx, red);
            const double inv = mx > 0.0 ? 1.0 / mx : 1.0;
            double ss = 0.0;
            for (int i = tid; i < n; i += blockDim.x) {
                const double t = x[i] * inv;
                ss += t * t;
            }
            ss = blockSum(ss, red);
            const double sc = inv / sqrt(fmax(ss, DBL_MIN));
            for (int i = tid; i < n; i += blockDim.x) x[i] *= sc;
            __syncthreads();
        }
        // sign convention: largest-magnitude component positive (dstein)
        double mx = 0.0;
        int imx = 0;
        if (tid == 0) {
            for (int i = 0; i < n; ++i)
                if (fabs(x[i]) > mx) {
                    mx = fabs(x[i]);
                    imx = i;
                }
            sh[0] = x[imx] < 0.0 ? -1.0 : 1.0;
        }
        __syncthreads();
        const double sg = sh[0];
        for (int i = tid; i < n; i += blockDim.x) x[i] *= sg;
        __syncthreads();
    }
}

cudaError_t launchInverseIter(const EigDesc* d, int nDesc, int maxK, int*, cudaStream_t s) {
    if (nDesc <= 0 || maxK <= 0) return cudaSuccess;
    dim3 grid(maxK, nDesc);
    // one warp per cluster: the serial recurrences run on one thread, so a
    // small CTA lets every wanted vector of a large problem run at once
    inverseIterKernel<<<grid, 32, 0, s>>>(d, maxK);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// back-transform Y <- H_0 ... H_{n-3} Y, one warp per column
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) backTransformKernel(const EigDesc* __restrict__ descs,
                                                            int maxK) {
    const int b = blockIdx.y;
    const int col = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const EigDesc D = descs[b];
    const int k = *D.kOut;
    if (col >= k) return;
    const int n = D.n;
    double* y = D.Y + (int64_t)col * D.ldy;
    for (int kk = n - 3; kk >= 0; --kk) {
        const double tau = D.tau[kk];
        if (tau == 0.0) continue;
        const double* v = D.A + (kk + 1) + (int64_t)kk * D.lda;   // v[0] = 1
        const int m = n - kk - 1;
        double s = 0.0;
        for (int i = lane; i < m; i += 32) s += v[i] * y[kk + 1 + i];
        s = warpSum<32>(s) * tau;
        for (int i = lane; i < m; i += 32) y[kk + 1 + i] -= s * v[i];
        __syncwarp();
    }
}

cudaError_t launchBackTransform(const EigDesc* d, int nDesc, int maxK, cudaStream_t s) {
    if (nDesc <= 0 || maxK <= 0) return cudaSuccess;
    dim3 grid((maxK + 7) / 8, nDesc);
    backTransformKernel<<<grid, 256, 0, s>>>(d, maxK);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// bisection with one warp per eigenvalue: each round evaluates 32 Sturm
// counts at equally spaced points of the current bracket (multisection),
// narrowing it 32-fold per round instead of 2-fold.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) bisectWarpKernel(const EigDesc* __restrict__ descs, int mode) {
    const int b = blockIdx.y;
    const int j = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const EigDesc D = descs[b];
    const int k = *D.kOut;
    if (j >= k) return;
    const int n = D.n;
    const int t = (mode <= 1) ? (n - j) : (j + 1);
    double lo, hi, pivmin, tn;
    gershgorin(D.d, D.e, n, lo, hi, pivmin, tn);
    for (int it = 0; it < 40; ++it) {
        if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin) break;
        const double x = lo + (hi - lo) * (lane + 1) / 33.0;
        const bool ge = sturmLess(D.d, D.e, n, x, pivmin, tn) >= t;   // lambda_t < x
        const unsigned m = __ballot_sync(0xffffffffu, ge);
        // first lane whose point is above lambda_t
        const int f = m ? __ffs(m) - 1 : 32;
        const double nlo = (f == 0) ? lo : lo + (hi - lo) * f / 33.0;
        const double nhi = (f == 32) ? hi : lo + (hi - lo) * (f + 1) / 33.0;
        if (!(nhi < hi || nlo > lo)) break;   // no progress at this resolution
        lo = nlo;
        hi = nhi;
    }
    if (lane == 0) D.w[j] = 0.5 * (lo + hi);
}

cudaError_t launchBisectWarp(const EigDesc* d, int nDesc, int mode, int want, double thr, int maxK,
                             cudaStream_t s, const double* thrArr) {
    if (nDesc <= 0) return cudaSuccess;
    bisectCountKernel<<<(nDesc + 127) / 128, 128, 0, s>>>(d, nDesc, mode, want, thr, thrArr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || maxK <= 0) return e;
    dim3 grid((maxK + 7) / 8, nDesc);
    bisectWarpKernel<<<grid, 256, 0, s>>>(d, mode);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// eigenvector back-transform with the columns and the reflector in shared
// memory: a CTA owns `cols` columns (one warp each); per reflector the CTA
// stages v_k once, each warp forms its dot product and update in shared
// memory.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) backTransformSmemKernel(const EigDesc* __restrict__ descs,
                                                                int cols, int maxN) {
    extern __shared__ double sb[];
    const int b = blockIdx.y;
    const EigDesc D = descs[b];
    const int n = D.n;
    if (n > maxN) return;             // larger matrices go through the blocked form
    const int k = *D.kOut;
    const int c0 = blockIdx.x * cols;
    if (c0 >= k) return;
    const int nc = min(cols, k - c0);
    double* sv = sb;                  // maxN
    double* sy = sb + maxN;           // cols x maxN
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int e = threadIdx.x; e < nc * n; e += blockDim.x) {
        const int c = e / n, i = e % n;
        sy[c * maxN + i] = D.Y[i + (int64_t)(c0 + c) * D.ldy];
    }
    for (int kk = n - 3; kk >= 0; --kk) {
        const double tau = D.tau[kk];
        if (tau == 0.0) continue;
        const int m = n - kk - 1;
        const double* v = D.A + (kk + 1) + (int64_t)kk * D.lda;
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) sv[i] = v[i];
        __syncthreads();
        for (int c = wid; c < nc; c += nw) {
            double* y = sy + c * maxN + kk + 1;
            double s = 0.0;
            for (int i = lane; i < m; i += 32) s += sv[i] * y[i];
            s = warpSum<32>(s) * tau;
            for (int i = lane; i < m; i += 32) y[i] -= s * sv[i];
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nc * n; e += blockDim.x) {
        const int c = e / n, i = e % n;
        D.Y[i + (int64_t)(c0 + c) * D.ldy] = sy[c * maxN + i];
    }
}

cudaError_t launchBackTransformSmem(const EigDesc* d, int nDesc, int maxK, int maxN, cudaStream_t s) {
    if (nDesc <= 0 || maxK <= 0 || maxN <= 0) return cudaSuccess;
    const int budget = 200 * 1024 / 8;                  // doubles of shared memory
    int cols = budget / maxN - 1;
    if (cols > 8) cols = 8;
    if (cols < 1) return launchBackTransform(d, nDesc, maxK, s);
    const size_t smem = sizeof(double) * (size_t)maxN * (cols + 1);
    cudaError_t e = cudaFuncSetAttribute(backTransformSmemKernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((maxK + cols - 1) / cols, nDesc);
    backTransformSmemKernel<<<grid, 256, smem, s>>>(d, cols, maxN);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// blocked (compact WY) back-transform, for the matrices above the one-CTA
// size: Q = H_0 ... H_{n-3} = B_0 ... B_last with B_j = I - V_j T_j V_j^T
// over 64 reflectors; the host applies the blocks with GEMMs.
// ------------------------------------------------------------------------
// zero A[i, j] for i <= j: the reflector columns become unit lower
// trapezoidal (v_k[0] = 1 at row k + 1) with zeros above
__global__ void zeroUpperKernel(const EigDesc* __restrict__ descs) {
    const EigDesc D = descs[blockIdx.y];
    for (int j = blockIdx.x; j < D.n; j += gridDim.x)
        for (int i = threadIdx.x; i <= j; i += blockDim.x) D.A[i + (int64_t)j * D.lda] = 0.0;
}

cudaError_t launchZeroUpper(const EigDesc* d, int nDesc, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    zeroUpperKernel<<<dim3(64, nDesc), 256, 0, s>>>(d);
    return cudaGetLastError();
}

// T (upper triangular, ld 64) of one block from S = V^T V (ld 64) and tau
// (LAPACK dlarft, forward, columnwise): T[i][i] = tau_i,
// T[0:i, i] = -tau_i T[0:i, 0:i] S[0:i, i].
__global__ void __launch_bounds__(64) wyTKernel(const WyBlock* __restrict__ blocks) {
    const WyBlock B = blocks[blockIdx.x];
    __shared__ double z[64];
    const int r = threadIdx.x, nb = B.nb;
    for (int e = r; e < 64 * 64; e += 64) B.T[e] = 0.0;
    __syncthreads();
    for (int i = 0; i < nb; ++i) {
        const double ti = B.tau[i];
        if (r < i) z[r] = -ti * B.S[r + 64 * i];
        __syncthreads();
        if (r < i) {
            double acc = 0.0;
            for (int q = r; q < i; ++q) acc += B.T[r + 64 * q] * z[q];
            B.T[r + 64 * i] = acc;
        }
        if (r == i) B.T[i + 64 * i] = ti;
        __syncthreads();
    }
}

cudaError_t launchWyT(const WyBlock* blocks, int nBlocks, cudaStream_t s) {
    if (nBlocks <= 0) return cudaSuccess;
    wyTKernel<<<nBlocks, 64, 0, s>>>(blocks);
    return cudaGetLastError();
}

}  // namespace amls_b200
