// FP64 blocked partial Cholesky of node fronts and row-panel triangular
// solves.
//
// Partial Cholesky (the multifrontal form of the reference's factorNode_ +
// X = K^-1 K_{i,a} solves, gaussian_elimination.cpp:458-598): a front F_i of
// (n + s) x n holds [K^_ii ; K_{S,i}]; after the call its top n x n lower
// triangle is L_ii and its bottom s x n block is L_Si = K_{S,i} L_ii^-T.
// Left-looking over 32-wide column blocks, two launches per block:
//   cholDiag:  D = F[J,J] - F[J,:J] F[J,:J]^T, D = chol(D)   (one CTA/front)
//   cholPanel: F[R,J] = (F[R,J] - F[R,:J] F[J,:J]^T) L_JJ^-T (CTA per 32 rows)
// A non-positive or NaN pivot sets the status word (code, node) and the
// front's factorisation continues with a unit pivot so no NaN spreads; the
// host turns the status into AMLS_ERR_NOT_SPD (reference P10 check,
// sparse_direct.cpp:17-22, 48-53).
#include "common.cuh"
#include "launch.hpp"

namespace amls_b200 {

namespace {
constexpr int NB = kCholBlock;  // 32
constexpr int NT = 256;
constexpr int TR = kTrsmRows;   // 32 rows per CTA
}

// acc[r][c] (32x32, thread owns 4 entries: col = tid/8, rows = tid%8 + 8*i)
// -= sum_{k in [k0,k1)} X(r, k) * Y(c, k), X and Y given by accessors.
template <class FX, class FY>
__device__ __forceinline__ void accumulateNT(double (&acc)[4], int k0, int k1, FX X, FY Y,
                                             double (*Xs)[NB + 1], double (*Ys)[NB + 1]) {
    const int tid = threadIdx.x;
    const int col = tid / 8, rsub = tid % 8;
    for (int kb = k0; kb < k1; kb += NB) {
        const int kn = min(NB, k1 - kb);
        __syncthreads();
        for (int e = tid; e < NB * NB; e += NT) {
            const int r = e % NB, k = e / NB;
            Xs[k][r] = (k < kn) ? X(r, kb + k) : 0.0;
            Ys[k][r] = (k < kn) ? Y(r, kb + k) : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < kn; ++k) {
            const double y = Ys[k][col];
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[i] = fma(-Xs[k][rsub + 8 * i], y, acc[i]);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(NT) cholDiagKernel(const FrontDesc* __restrict__ descs, int jb,
                                                     int* status) {
    __shared__ double Xs[NB][NB + 1], Ys[NB][NB + 1], Dm[NB][NB + 1];
    __shared__ int bad;
    const FrontDesc F = descs[blockIdx.x];
    const int j0 = jb * NB;
    if (j0 >= F.n) return;
    const int nb = min(NB, F.n - j0);
    const int tid = threadIdx.x, col = tid / 8, rsub = tid % 8;
    double acc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = rsub + 8 * i;
        acc[i] = (r < nb && col < nb) ? F.F[(j0 + r) + (int64_t)(j0 + col) * F.ld] : 0.0;
    }
    auto XJ = [&](int r, int k) -> double {
        return r < nb ? F.F[(j0 + r) + (int64_t)k * F.ld] : 0.0;
    };
    accumulateNT(acc, 0, j0, XJ, XJ, Xs, Ys);
#pragma unroll
    for (int i = 0; i < 4; ++i) Dm[rsub + 8 * i][col] = acc[i];
    if (tid == 0) bad = 0;
    __syncthreads();
    // unblocked right-looking Cholesky of Dm (lower)
    for (int k = 0; k < nb; ++k) {
        if (tid == 0) {
            double d = Dm[k][k];
            if (!(d > 0.0) || !isfinite(d)) {
                bad = 1;
                d = 1.0;
            }
            Dm[k][k] = sqrt(d);
        }
        __syncthreads();
        const double dk = Dm[k][k];
        for (int r = k + 1 + tid; r < nb; r += NT) Dm[r][k] /= dk;
        __syncthreads();
        for (int e = tid; e < nb * nb; e += NT) {
            const int r = e % nb, c = e / nb;
            if (c > k && r >= c) Dm[r][c] -= Dm[r][k] * Dm[c][k];
        }
        __syncthreads();
    }
    if (bad && tid == 0) setStatus(status, kDevNotSpd, F.node);
    for (int e = tid; e < nb * nb; e += NT) {
        const int r = e % nb, c = e / nb;
        F.F[(j0 + r) + (int64_t)(j0 + c) * F.ld] = (r >= c) ? Dm[r][c] : 0.0;
    }
}

__global__ void __launch_bounds__(NT) cholPanelKernel(const FrontDesc* __restrict__ descs, int jb,
                                                      int maxRowTiles) {
    __shared__ double Xs[NB][NB + 1], Ys[NB][NB + 1], Ls[NB][NB + 1], Out[TR][NB + 1];
    const FrontDesc F = descs[blockIdx.x / maxRowTiles];
    const int tile = blockIdx.x % maxRowTiles;
    const int j0 = jb * NB;
    if (j0 >= F.n) return;
    const int nb = min(NB, F.n - j0);
    const int j1 = j0 + nb;
    const int r0 = j1 + tile * TR;
    if (r0 >= F.rows) return;
    const int nr = min(TR, F.rows - r0);
    const int tid = threadIdx.x, col = tid / 8, rsub = tid % 8;
    double acc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = rsub + 8 * i;
        acc[i] = (r < nr && col < nb) ? F.F[(r0 + r) + (int64_t)(j0 + col) * F.ld] : 0.0;
    }
    auto XR = [&](int r, int k) -> double {
        return r < nr ? F.F[(r0 + r) + (int64_t)k * F.ld] : 0.0;
    };
    auto YJ = [&](int c, int k) -> double {
        return c < nb ? F.F[(j0 + c) + (int64_t)k * F.ld] : 0.0;
    };
    accumulateNT(acc, 0, j0, XR, YJ, Xs, Ys);
#pragma unroll
    for (int i = 0; i < 4; ++i) Out[rsub + 8 * i][col] = acc[i];
    for (int e = tid; e < NB * NB; e += NT) {
        const int r = e % NB, c = e / NB;
        Ls[r][c] = (r < nb && c < nb) ? F.F[(j0 + r) + (int64_t)(j0 + c) * F.ld] : 0.0;
    }
    __syncthreads();
    // x L_JJ^T = out : x_j = (out_j - sum_{c<j} x_c L[j][c]) / L[j][j]
    if (tid < nr) {
        for (int j = 0; j < nb; ++j) {
            double v = Out[tid][j];
            for (int c = 0; c < j; ++c) v -= Out[tid][c] * Ls[j][c];
            Out[tid][j] = v / Ls[j][j];
        }
    }
    __syncthreads();
    for (int e = tid; e < TR * NB; e += NT) {
        const int r = e % TR, c = e / TR;
        if (r < nr && c < nb) F.F[(r0 + r) + (int64_t)(j0 + c) * F.ld] = Out[r][c];
    }
}

cudaError_t launchCholDiag(const FrontDesc* d, int nDesc, int jb, int* status, cudaStream_t s) {
    if (nDesc <= 0) return cudaSuccess;
    cholDiagKernel<<<nDesc, NT, 0, s>>>(d, jb, status);
    return cudaGetLastError();
}

cudaError_t launchCholPanel(const FrontDesc* d, int nDesc, int jb, int maxRowTiles,
                            cudaStream_t s) {
    if (nDesc <= 0 || maxRowTiles <= 0) return cudaSuccess;
    cholPanelKernel<<<nDesc * maxRowTiles, NT, 0, s>>>(d, jb, maxRowTiles);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// row-panel TRSM: X (r x n) <- X L^-T (forward) or X L^-1 (backward)
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) trsmRowsKernel(const TrsmDesc* __restrict__ descs,
                                                     const TileRef* __restrict__ tiles) {
    __shared__ double Xs[NB][NB + 1], Ys[NB][NB + 1], Ls[NB][NB + 1], Out[TR][NB + 1];
    const TileRef t = tiles[blockIdx.x];
    const TrsmDesc D = descs[t.desc];
    const int r0 = t.m0;
    const int nr = min(TR, D.r - r0);
    if (nr <= 0) return;
    const int tid = threadIdx.x, col = tid / 8, rsub = tid % 8;
    const int nblk = (D.n + NB - 1) / NB;
    for (int bi = 0; bi < nblk; ++bi) {
        const int jb = D.backward ? (nblk - 1 - bi) : bi;
        const int j0 = jb * NB, nb = min(NB, D.n - j0), j1 = j0 + nb;
        double acc[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = rsub + 8 * i;
            acc[i] = (r < nr && col < nb) ? D.X[(r0 + r) + (int64_t)(j0 + col) * D.ldx] : 0.0;
        }
        auto XR = [&](int r, int k) -> double {
            return r < nr ? D.X[(r0 + r) + (int64_t)k * D.ldx] : 0.0;
        };
        if (!D.backward) {
            // acc -= X[:, :j0] L[J, :j0]^T
            auto YJ = [&](int c, int k) -> double {
                return c < nb ? D.L[(j0 + c) + (int64_t)k * D.ldl] : 0.0;
            };
            accumulateNT(acc, 0, j0, XR, YJ, Xs, Ys);
        } else {
            // acc -= X[:, j1:] L[j1:, J]
            auto YJ = [&](int c, int k) -> double {
                return c < nb ? D.L[k + (int64_t)(j0 + c) * D.ldl] : 0.0;
            };
            accumulateNT(acc, j1, D.n, XR, YJ, Xs, Ys);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) Out[rsub + 8 * i][col] = acc[i];
        for (int e = tid; e < NB * NB; e += NT) {
            const int r = e % NB, c = e / NB;
            Ls[r][c] = (r < nb && c < nb) ? D.L[(j0 + r) + (int64_t)(j0 + c) * D.ldl] : 0.0;
        }
        __syncthreads();
        if (tid < nr) {
            if (!D.backward) {
                for (int j = 0; j < nb; ++j) {
                    double v = Out[tid][j];
                    for (int c = 0; c < j; ++c) v -= Out[tid][c] * Ls[j][c];
                    Out[tid][j] = v / Ls[j][j];
                }
            } else {
                // x L = out: x_j = (out_j - sum_{c>j} x_c L[c][j]) / L[j][j]
                for (int j = nb - 1; j >= 0; --j) {
                    double v = Out[tid][j];
                    for (int c = j + 1; c < nb; ++c) v -= Out[tid][c] * Ls[c][j];
                    Out[tid][j] = v / Ls[j][j];
                }
            }
        }
        __syncthreads();
        for (int e = tid; e < TR * NB; e += NT) {
            const int r = e % TR, c = e / TR;
            if (r < nr && c < nb) D.X[(r0 + r) + (int64_t)(j0 + c) * D.ldx] = Out[r][c];
        }
        __syncthreads();
    }
}

cudaError_t launchTrsmRows(const TrsmDesc* d, const TileRef* dTiles, int nTiles, cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    trsmRowsKernel<<<nTiles, NT, 0, s>>>(d, dTiles);
    return cudaGetLastError();
}


// ------------------------------------------------------------------------
// right-looking blocked partial Cholesky, 64-wide column blocks: per block J
// this kernel factors the (already updated) diagonal block in place and
// writes its inverse; the panel solve (in place, times inv^T) and the
// trailing SYRK update are batched GEMMs issued by the host.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) cholDiag64Kernel(const FrontDesc* __restrict__ fronts,
                                                       const TrsmDesc* __restrict__ invd, int J,
                                                       int* status) {
    extern __shared__ double cdSmem[];
    double (*D)[65] = reinterpret_cast<double (*)[65]>(cdSmem);            // block, then L
    double (*X)[65] = reinterpret_cast<double (*)[65]>(cdSmem + 64 * 65);  // L^-1
    __shared__ double piv[64];
    __shared__ int bad;
    const FrontDesc F = fronts[blockIdx.x];
    const int j0 = J * 64;
    if (j0 >= F.n) return;
    const int nb = min(64, F.n - j0);
    const int tid = threadIdx.x;
    for (int e = tid; e < 64 * 64; e += NT) {
        const int r = e % 64, c = e / 64;
        D[r][c] = (r < nb && c < nb) ? F.F[(j0 + r) + (int64_t)(j0 + c) * F.ld] : (r == c ? 1.0 : 0.0);
        X[r][c] = (r == c) ? 1.0 : 0.0;
    }
    if (tid == 0) bad = 0;
    __syncthreads();
    // right-looking on the unscaled block, one barrier per column: with
    // d_k = D[k][k] (a non-positive or NaN pivot counts as 1, as in the
    // left-looking kernel), D[r][c] -= D[r][k] D[c][k] / d_k for k < c <= r;
    // thread (r = tid % 64, columns c = tid / 64 + 4 j)
    const int tr = tid & 63, tc = tid >> 6;
    for (int k = 0; k < nb; ++k) {
        double dk = D[k][k];
        if (!(dk > 0.0) || !isfinite(dk)) {
            if (tid == 0) bad = 1;
            dk = 1.0;
        }
        if (tid == 0) piv[k] = sqrt(dk);
        const double rinv = 1.0 / dk;
        if (tr < nb) {
            // operands staged in registers first: the stores cannot then
            // serialise the loads of the next columns
            const double lr = D[tr][k] * rinv;
            double a[16], b[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = k + 1 + tc + 4 * j;
                if (c <= tr) {
                    a[j] = D[c][k];
                    b[j] = D[tr][c];
                }
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = k + 1 + tc + 4 * j;
                if (c <= tr) D[tr][c] = b[j] - lr * a[j];
            }
        }
        __syncthreads();
    }
    if (bad && tid == 0) setStatus(status, kDevNotSpd, F.node);
    // scale: L[r][c] = D[r][c] / piv[c] (r > c), L[c][c] = piv[c]
    for (int e = tid; e < nb * nb; e += NT) {
        const int r = e % nb, c = e / nb;
        if (r > c) D[r][c] /= piv[c];
        else if (r == c) D[r][c] = piv[c];
    }
    __syncthreads();
    for (int e = tid; e < nb * nb; e += NT) {
        const int r = e % nb, c = e / nb;
        F.F[(j0 + r) + (int64_t)(j0 + c) * F.ld] = (r >= c) ? D[r][c] : 0.0;
    }
    // X = L^-1 of the identity-padded block, right-looking on unscaled rows:
    // X[r][c] -= L[r][k] X[k][c] / L[k][k] for r > k, c <= k; rows scaled last
    for (int k = 0; k < nb; ++k) {
        const double rinv = 1.0 / D[k][k];
        if (tr > k && tr < nb) {
            const double lr = D[tr][k] * rinv;
            double a[16], b[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = tc + 4 * j;
                if (c <= k) {
                    a[j] = X[k][c];
                    b[j] = X[tr][c];
                }
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = tc + 4 * j;
                if (c <= k) X[tr][c] = b[j] - lr * a[j];
            }
        }
        __syncthreads();
    }
    double* out = invd[blockIdx.x].inv + (int64_t)J * 4096;
    for (int e = tid; e < 64 * 64; e += NT) {
        const int r = e % 64, c = e / 64;
        out[r + 64 * c] = (r < nb && c <= r) ? X[r][c] / D[r][r] : (r == c ? 1.0 : 0.0);
    }
}

cudaError_t launchCholDiag64(const FrontDesc* fronts, const TrsmDesc* invd, int nFront, int J,
                             int* status, cudaStream_t s) {
    if (nFront <= 0) return cudaSuccess;
    constexpr size_t smem = sizeof(double) * 2 * 64 * 65;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(cholDiag64Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    cholDiag64Kernel<<<nFront, NT, smem, s>>>(fronts, invd, J, status);
    return cudaGetLastError();
}

// X[J*64 + r, J*64 + c] = inv[J][r + 64 c] for r, c < the block's size: the
// diagonal blocks of L^-1 (X n x n, ld ldx), the start of its doubling
// construction.  One CTA per (descriptor, block).
__global__ void __launch_bounds__(256) placeDiagInvKernel(const TrsmDesc* __restrict__ descs,
                                                          const TileRef* __restrict__ tiles) {
    const TileRef t = tiles[blockIdx.x];
    const TrsmDesc D = descs[t.desc];
    const int J = t.m0;
    const int j0 = J * 64, nb = min(64, D.n - j0);
    const double* in = D.inv + (int64_t)J * 4096;
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
        const int r = e % 64, c = e / 64;
        if (r < nb && c < nb) D.X[(j0 + r) + (int64_t)(j0 + c) * D.ldx] = in[r + 64 * c];
    }
}

cudaError_t launchPlaceDiagInv(const TrsmDesc* d, const TileRef* tiles, int nTiles, cudaStream_t s) {
    if (nTiles <= 0) return cudaSuccess;
    placeDiagInvKernel<<<nTiles, 256, 0, s>>>(d, tiles);
    return cudaGetLastError();
}

}  // namespace amls_b200
