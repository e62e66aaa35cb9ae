// Pencil assembly on the GPU: isoparametric hexahedral elasticity elements
// (8-node trilinear or 27-node triquadratic) integrated by Gauss-Legendre
// quadrature (2 or 3 points per direction) and scattered into the values of
// a CSR pattern given by the host.  Stands in for the host assembly of the
// synthetic benchmark pencils (the reference reads its pencils from files;
// its generators are graph Laplacians, src/io/case_generator.cpp).
//
// Element e with nodal coordinates X_a (a < nn), modulus E_e, density rho_e,
// Poisson ratio nu (lambda = nu / ((1 + nu)(1 - 2 nu)), mu = 1 / (2 (1 + nu))
// per unit modulus), at Gauss point g with weight w_g and J = dX/dxi:
//   Ke[3a+i, 3b+j] = E_e sum_g w_g |J| (lambda N_a,i N_b,j + mu N_a,j N_b,i
//                                        + mu delta_ij sum_k N_a,k N_b,k)
//   Me[3a+i, 3b+j] = rho_e delta_ij sum_g w_g |J| N_a N_b
// (the B^T D B and N^T N forms in Voigt notation), local node a = a0 +
// (p+1) (a1 + (p+1) a2) for 1-D node indices along x, y, z, DOF 3a + i.
// One CTA per element: the shape-function gradients of all Gauss points in
// shared memory, one matrix entry per thread and step, atomic scatter into
// the CSR values at the position found by binary search in the row.
#include <cmath>

#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
constexpr int kMaxNn = 27;
constexpr int kMaxGp = 27;

__device__ __forceinline__ void lagrange1d(int p, double x, double* v, double* d) {
    // nodes -1, 0, 1 (p = 2) or -1, 1 (p = 1)
    if (p == 1) {
        v[0] = 0.5 * (1.0 - x);
        v[1] = 0.5 * (1.0 + x);
        d[0] = -0.5;
        d[1] = 0.5;
    } else {
        v[0] = 0.5 * x * (x - 1.0);
        v[1] = 1.0 - x * x;
        v[2] = 0.5 * x * (x + 1.0);
        d[0] = x - 0.5;
        d[1] = -2.0 * x;
        d[2] = x + 0.5;
    }
}

__device__ __forceinline__ int findCol(const int32_t* __restrict__ col, int64_t lo, int64_t hi, int32_t c) {
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (col[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return static_cast<int>(lo);
}
}  // namespace

__global__ void __launch_bounds__(256) hexAssembleKernel(HexAssembleArgs A) {
    __shared__ double sX[kMaxNn * 3];
    __shared__ double sN[kMaxGp * kMaxNn];
    __shared__ double sD[kMaxGp * kMaxNn * 3];     // dN/dx per Gauss point
    __shared__ double sW[kMaxGp];
    __shared__ int64_t sDof[kMaxNn * 3];
    const int p = A.order, n1 = p + 1, nn = n1 * n1 * n1, nd = 3 * nn, ng = n1 * n1 * n1;
    // Gauss-Legendre points and weights
    double gx[3], gw[3];
    if (n1 == 2) {
        gx[0] = -0.57735026918962576451;   // -1/sqrt(3)
        gx[1] = 0.57735026918962576451;
        gw[0] = gw[1] = 1.0;
    } else {
        gx[0] = -0.77459666924148337704;   // -sqrt(3/5)
        gx[1] = 0.0;
        gx[2] = 0.77459666924148337704;
        gw[0] = gw[2] = 5.0 / 9.0;
        gw[1] = 8.0 / 9.0;
    }
    const double nu = A.nu;
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 1.0 / (2.0 * (1.0 + nu));
    for (int64_t e = blockIdx.x; e < A.nelem; e += gridDim.x) {
        __syncthreads();
        for (int t = threadIdx.x; t < nn * 3; t += blockDim.x) {
            const int64_t node = A.enodes[e * nn + t / 3];
            sX[t] = A.coords[node * 3 + t % 3];
        }
        for (int t = threadIdx.x; t < nd; t += blockDim.x) sDof[t] = A.dofmap[e * nd + t];
        __syncthreads();
        // one thread per Gauss point: N, dN/dxi, J, J^-1, dN/dx, weight
        for (int g = threadIdx.x; g < ng; g += blockDim.x) {
            const int gi = g % n1, gj = (g / n1) % n1, gk = g / (n1 * n1);
            double vx[3], dx[3], vy[3], dy[3], vz[3], dz[3];
            lagrange1d(p, gx[gi], vx, dx);
            lagrange1d(p, gx[gj], vy, dy);
            lagrange1d(p, gx[gk], vz, dz);
            double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // J[r][c] = dX_r / dxi_c
            for (int a = 0; a < nn; ++a) {
                const int a0 = a % n1, a1 = (a / n1) % n1, a2 = a / (n1 * n1);
                const double d0 = dx[a0] * vy[a1] * vz[a2], d1 = vx[a0] * dy[a1] * vz[a2], d2 = vx[a0] * vy[a1] * dz[a2];
                for (int r = 0; r < 3; ++r) {
                    J[r][0] += sX[a * 3 + r] * d0;
                    J[r][1] += sX[a * 3 + r] * d1;
                    J[r][2] += sX[a * 3 + r] * d2;
                }
            }
            const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            double Ji[3][3];   // inverse of J
            Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
            Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
            Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
            Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
            Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
            Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
            Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
            Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
            Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
            sW[g] = gw[gi] * gw[gj] * gw[gk] * fabs(det);
            for (int a = 0; a < nn; ++a) {
                const int a0 = a % n1, a1 = (a / n1) % n1, a2 = a / (n1 * n1);
                const double dxi[3] = {dx[a0] * vy[a1] * vz[a2], vx[a0] * dy[a1] * vz[a2], vx[a0] * vy[a1] * dz[a2]};
                sN[g * nn + a] = vx[a0] * vy[a1] * vz[a2];
                // dN/dX_k = sum_c dN/dxi_c (J^-1)[c][k]
                for (int k = 0; k < 3; ++k)
                    sD[(g * nn + a) * 3 + k] = dxi[0] * Ji[0][k] + dxi[1] * Ji[1][k] + dxi[2] * Ji[2][k];
            }
        }
        __syncthreads();
        const double Ee = A.E[e], re = A.rho[e];
        for (int q = threadIdx.x; q < nd * nd; q += blockDim.x) {
            const int r = q % nd, c = q / nd;
            const int64_t dr = sDof[r], dc = sDof[c];
            if (dr < 0 || dc < 0) continue;
            const int a = r / 3, i = r % 3, b = c / 3, j = c % 3;
            double k = 0.0, m = 0.0;
            for (int g = 0; g < ng; ++g) {
                const double* Da = sD + (g * nn + a) * 3;
                const double* Db = sD + (g * nn + b) * 3;
                double t = lam * Da[i] * Db[j] + mu * Da[j] * Db[i];
                if (i == j) {
                    t += mu * (Da[0] * Db[0] + Da[1] * Db[1] + Da[2] * Db[2]);
                    m += sW[g] * sN[g * nn + a] * sN[g * nn + b];
                }
                k += sW[g] * t;
            }
            const int64_t lo = A.rowptr[dr], hi = A.rowptr[dr + 1];
            const int pos = findCol(A.col, lo, hi, static_cast<int32_t>(dc));
            if (pos >= hi || A.col[pos] != dc) {
                setStatus(A.status, kDevBadPattern, static_cast<int>(e));
                continue;
            }
            atomicAdd(A.kval + pos, Ee * k);
            if (i == j) atomicAdd(A.mval + pos, re * m);
        }
    }
}

cudaError_t launchHexAssemble(const HexAssembleArgs& a, cudaStream_t s) {
    if (a.nelem <= 0) return cudaSuccess;
    if (a.order != 1 && a.order != 2) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(a.kval, 0, sizeof(double) * (size_t)a.nnz, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.mval, 0, sizeof(double) * (size_t)a.nnz, s);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = a.nelem < 8LL * sms ? a.nelem : 8LL * sms;
    hexAssembleKernel<<<(int)grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace amls_b200
