// Per-element eigenvalue sensitivities (adjoint form).
//
// For a pencil assembled as K = sum_e E_e Kbar_t(e), M = sum_e rho_e
// Mbar_t(e) (reference element pairs indexed by an element type t(e), with a
// per-element modulus and density scale) and M-normalised eigenvectors x_k:
//   d lambda_k / d E_e   =  x_{k,e}^T Kbar_t(e) x_{k,e}
//   d lambda_k / d rho_e = -lambda_k x_{k,e}^T Mbar_t(e) x_{k,e}
// (simple eigenvalues only; modes whose relative gap to a neighbour is below
// gapTol get weight 0 in the weighted sums and NaN in the per-mode output).
//
// One CTA per element at a time (persistent over elements): the element
// type's Kbar and Mbar in shared memory (reloaded when the type changes), the
// element's rows of X gathered 32 modes at a time, the two quadratic forms
// per mode as shared-memory matrix products.
#include <cmath>

#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
constexpr int kMaxDofE = 96;     // 27-node hex: 81
constexpr int kModes = 32;
}

__global__ void __launch_bounds__(256) sensitivityKernel(
    int64_t nelem, int nd, const int64_t* __restrict__ dofmap, const int32_t* __restrict__ elemType,
    const double* __restrict__ Kbar,
    const double* __restrict__ Mbar, const double* __restrict__ X, int64_t n, int nmodes,
    const double* __restrict__ lambda, const double* __restrict__ weight,
    double* __restrict__ gE, double* __restrict__ gRho, double* __restrict__ dE,
    double* __restrict__ dRho) {
    extern __shared__ double sm[];
    double* sK = sm;                          // nd x nd
    double* sM = sK + nd * nd;                // nd x nd
    double* sX = sM + nd * nd;                // nd x kModes
    __shared__ int64_t sDof[kMaxDofE];
    __shared__ double sA[kModes], sB[kModes];
    int loaded = -1;                          // element type held in sK / sM
    for (int64_t e = blockIdx.x; e < nelem; e += gridDim.x) {
        __syncthreads();
        const int ty = elemType ? elemType[e] : 0;
        if (ty != loaded) {
            const double* kb = Kbar + (int64_t)ty * nd * nd;
            const double* mb = Mbar + (int64_t)ty * nd * nd;
            for (int t = threadIdx.x; t < nd * nd; t += blockDim.x) {
                sK[t] = kb[t];
                sM[t] = mb[t];
            }
            loaded = ty;
        }
        for (int t = threadIdx.x; t < nd; t += blockDim.x) sDof[t] = dofmap[e * nd + t];
        double accE = 0.0, accR = 0.0;   // weighted sums (thread 0 keeps them)
        for (int k0 = 0; k0 < nmodes; k0 += kModes) {
            const int km = min(kModes, nmodes - k0);
            __syncthreads();
            for (int t = threadIdx.x; t < nd * kModes; t += blockDim.x) {
                const int r = t % nd, k = t / nd;
                const int64_t d = sDof[r];
                sX[t] = (k < km && d >= 0) ? X[d + (int64_t)(k0 + k) * n] : 0.0;
            }
            if (threadIdx.x < kModes) {
                sA[threadIdx.x] = 0.0;
                sB[threadIdx.x] = 0.0;
            }
            __syncthreads();
            // thread (k, rgroup): partial sums of x_k^T A x_k over rows r
            const int k = threadIdx.x % kModes, rg = threadIdx.x / kModes;   // 8 row groups
            const int ngroups = blockDim.x / kModes;
            double a = 0.0, b = 0.0;
            if (k < km) {
                const double* xk = sX + k * nd;
                for (int r = rg; r < nd; r += ngroups) {
                    double tk = 0.0, tm = 0.0;
                    for (int c = 0; c < nd; ++c) {
                        tk = fma(sK[r + c * nd], xk[c], tk);
                        tm = fma(sM[r + c * nd], xk[c], tm);
                    }
                    a = fma(xk[r], tk, a);
                    b = fma(xk[r], tm, b);
                }
            }
            atomicAdd(&sA[k], a);
            atomicAdd(&sB[k], b);
            __syncthreads();
            if (threadIdx.x < km) {
                const int kk = k0 + threadIdx.x;
                const double lam = lambda[kk];
                const double w = weight ? weight[kk] : 0.0;
                const double de = sA[threadIdx.x], dr = -lam * sB[threadIdx.x];
                if (dE) dE[e + (int64_t)kk * nelem] = (w == w) ? de : NAN;
                if (dRho) dRho[e + (int64_t)kk * nelem] = (w == w) ? dr : NAN;
                if (w == w) {   // NaN weight marks a non-simple eigenvalue
                    sA[threadIdx.x] = w * de;
                    sB[threadIdx.x] = w * dr;
                } else {
                    sA[threadIdx.x] = 0.0;
                    sB[threadIdx.x] = 0.0;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0)
                for (int q = 0; q < km; ++q) {
                    accE += sA[q];
                    accR += sB[q];
                }
        }
        if (threadIdx.x == 0) {
            if (gE) gE[e] = accE;
            if (gRho) gRho[e] = accR;
        }
    }
}

cudaError_t launchSensitivity(int64_t nelem, int nd, const int64_t* dofmap, const int32_t* elemType,
                              const double* Kbar,
                              const double* Mbar, const double* X, int64_t n, int nmodes,
                              const double* lambda, const double* weight, double* gE,
                              double* gRho, double* dE, double* dRho, cudaStream_t s) {
    if (nelem <= 0 || nmodes <= 0) return cudaSuccess;
    if (nd <= 0 || nd > kMaxDofE) return cudaErrorInvalidValue;
    const size_t smem = sizeof(double) * (2 * nd * nd + nd * kModes);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(sensitivityKernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = nelem < (int64_t)sms ? nelem : (int64_t)sms;
    sensitivityKernel<<<(int)grid, 256, smem, s>>>(nelem, nd, dofmap, elemType, Kbar, Mbar, X, n, nmodes,
                                                    lambda, weight, gE, gRho, dE, dRho);
    return cudaGetLastError();
}

}  // namespace amls_b200
