// Host-side launch interface of the AMLS kernels.  Plain structs shared with
// the device code; every launcher enqueues on the given stream and returns
// the cudaError_t of the launch.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace amls_b200 {

// Device status word codes written by kernels (read back by the host):
// status[0] = code of the first failure, status[1] = where (node / matrix).
enum DevStatus : int {
    kDevOk = 0,
    kDevNotSpd = 1,      // non-positive or NaN pivot
    kDevIterCap = 2,     // iteration cap reached
    kDevTimeout = 3,     // a bounded wait on the tensor cores ran out
    kDevBadPattern = 4,  // an element entry missing from the given CSR pattern
};

// ---------------------------------------------------------------- GEMM --
// C(MxN) = alpha * op(A)(MxK) * op(B)(KxN) [+ beta*C], column-major, FP64.
enum GemmFlags : int32_t {
    kTransA = 1,        // op(A)[i,k] = A[k + i*lda]
    kTransB = 2,        // op(B)[k,j] = B[j + k*ldb]
    kScatter = 4,       // output address = C + colOff[j] + rowIdx[i]
    kAtomic = 8,        // accumulate with atomicAdd (scatter only)
    kGatherA = 16,      // op(A)[i,k] = A[i + aMap[k]*lda]   (no transA)
    kRowScale = 32,     // multiply result row i by rowScale[i]
    kColScale = 64,     // multiply result column j by colScale[j]
    kAccumulate = 128,  // dense: C = alpha*AB + beta*C ; scatter: *dst += alpha*AB
    kTriKUpTo = 256,    // op(B) upper triangular: column j uses k <= j only
    kTriKFrom = 512,    // op(B) lower triangular: column j uses k >= j only
    kTriAUpTo = 1024,   // op(A) lower triangular: row i uses k <= i only
};

struct GemmDesc {
    int32_t M, N, K, flags;
    const double* A;
    int64_t lda;
    const double* B;
    int64_t ldb;
    double* C;
    int64_t ldc;
    double alpha, beta;
    const int32_t* rowIdx;
    const int64_t* colOff;
    const int32_t* aMap;
    const double* rowScale;
    const double* colScale;
    int32_t kChunk;        // > 0: split-K, tile's TileRef.pad = chunk index, dense C
    int32_t pad0;          // accumulated with atomics (caller zeroes C first)
};

struct TileRef {
    int32_t desc, m0, n0, pad;
};

// Tile size of the batched GEMM (host builds TileRef tables with it).  One
// descriptor table per launch may mix layouts (kTransA / kTransB / kGatherA).
constexpr int kGemmTile = 64;

cudaError_t launchGemmBatched(const GemmDesc* dDescs, const TileRef* dTiles, int nTiles,
                              cudaStream_t s);
// Mixed precision (gemm_mixed.cu): the same descriptors on tcgen05 with the
// operands split into BF16 pairs (3 products, FP32 accumulation, relative
// error ~2^-16), 128 x 128 tiles (TileRef m0/n0 multiples of 128).
constexpr int kGemmTileMixed = 128;
cudaError_t launchGemmBatchedMixed(const GemmDesc* dDescs, const TileRef* dTiles, int nTiles,
                                   int* status, cudaStream_t s);

// Extend-add update of one eliminated front (multifrontal form of the
// reference's Schur + congruence updates):
//   UK = A A^T, UM = A B^T + B A^T  (s x s), A = L_Si, B = R_i^T (s x n each)
// entry (p, q) with p >= pmin[q] is subtracted (atomically) from
//   kPool[colOff[q] + rowIdx[rowBase[q] + p]]  and  mPool[same offset].
struct FrontUpdDesc {
    int32_t s, n;          // update order s, inner dimension n
    int32_t tilesM, pad;   // number of 64-row tiles
    const double* A;       // s x n, ld
    const double* B;
    int64_t ld;
    const int32_t* pmin;   // per column q
    const int64_t* colOff; // per column q (element offset in pools)
    const int32_t* rowIdx; // row target offsets
    const int32_t* rowBase;// per column q, index base into rowIdx
};
cudaError_t launchFrontUpdate(const FrontUpdDesc* dDescs, const TileRef* dTiles, int nTiles,
                              double* kPool, double* mPool, cudaStream_t s);

// -------------------------------------------------------- factorisation --
// Batched blocked partial Cholesky of fronts F_i ((n+s) x n, ld = n+s):
// L_ii = chol(F_ii), L_Si = F_Si L_ii^-T, in place.  One call per column
// block jb; descs list the fronts of one tree level.
struct FrontDesc {
    double* F;             // front (column-major)
    int64_t ld;            // n + s
    int32_t n, rows;       // n pivots, rows = n + s
    int32_t node, pad;
};
constexpr int kCholBlock = 32;
cudaError_t launchCholDiag(const FrontDesc* d, int nDesc, int jb, int* status, cudaStream_t s);
cudaError_t launchCholPanel(const FrontDesc* d, int nDesc, int jb, int maxRowTiles,
                            cudaStream_t s);

// Batched row-panel triangular solve with a factored front's L (n x n):
//   forward  (backward=0):  X <- X L^-T   (X: r x n, ld ldx)
//   backward (backward=1):  X <- X L^-1
struct TrsmDesc {
    const double* L;
    int64_t ldl;
    double* X;
    int64_t ldx;
    int32_t n, r;
    int32_t rowTiles, backward;
    double* inv;            // inverses of the 64x64 diagonal blocks (cholDiag64, placeDiagInv)
};
constexpr int kTrsmRows = 32;
cudaError_t launchTrsmRows(const TrsmDesc* d, const TileRef* dTiles, int nTiles, cudaStream_t s);
// Right-looking variant, 64-wide blocks: factor the diagonal block J of each
// front in place (fronts[i]) and write its inverse to invd[i].inv + 4096 J
// (identity-padded to 64 x 64); panel and trailing update are GEMMs.
cudaError_t launchCholDiag64(const FrontDesc* fronts, const TrsmDesc* invd, int nFront, int J,
                             int* status, cudaStream_t s);
// X (n x n, ld ldx) diagonal 64 x 64 blocks <- inv blocks (TileRef.m0 = J);
// the rest of X is left as it is (the caller zeroes it).
cudaError_t launchPlaceDiagInv(const TrsmDesc* d, const TileRef* dTiles, int nTiles, cudaStream_t s);

// ------------------------------------------------------- eigensolver ----
// Symmetric tridiagonalisation (Householder), in place.  A (n x n, full
// symmetric, ld) is overwritten: v_k stored in A[k+1:n, k] (v_k[0] = 1);
// d[n], e[n-1], tau[n-1].
struct EigDesc {
    double* A;
    int64_t lda;
    double* d;
    double* e;
    double* tau;
    int32_t n, id;
    // selection and outputs
    double* w;          // selected eigenvalues (of the tridiagonal/symmetric matrix)
    double* Y;          // n x kcap eigenvectors, ld = ldy
    int64_t ldy;
    int32_t kcap;       // capacity (columns of Y)
    int32_t* kOut;      // number selected (device)
    double* work;       // per-matrix scratch (>= 8n doubles)
};
// One CTA per matrix, n <= kTridiagSmallMax.
constexpr int kTridiagSmallMax = 384;
cudaError_t launchTridiagSmall(const EigDesc* d, int nDesc, cudaStream_t s);
// Cooperative multi-CTA tridiagonalisation of a batch of large matrices: the
// grid is split into CTA groups, group g (CTAs groupFirst[g] ..
// + groupSize[g]) works on descs[g]; p accumulators at
// dP + kTridiagPBufs * dPOff[g] (kTridiagPBufs * n doubles per matrix: dP must
// hold kTridiagPBufs * sum n).  One CTA of kTridiagLargeThreads per SM.
constexpr int kTridiagPBufs = 3;
constexpr int kTridiagLargeThreads = 1024;
cudaError_t launchTridiagLargeGroups(const EigDesc* dDescs, const int* dGroupOf,
                                     const int* dGroupFirst, const int* dGroupSize, int nCta,
                                     double* dP, const int64_t* dPOff, int maxN, cudaStream_t s);
// Co-resident CTA count for the cooperative kernel at a given maxN.
int tridiagLargeMaxCtas(int maxN);
// Select eigenvalues of T: mode 0 = the k largest (k = want), mode 1 = all
// >= thr (thrArr[b] per descriptor when given); mode 2 = the k smallest,
// mode 3 = all <= thr; each count capped by the descriptor's kcap.
// Bisection.  Selected values are written in "wanted" order (largest first
// for modes 0/1, smallest first for modes 2/3).
cudaError_t launchBisect(const EigDesc* d, int nDesc, int mode, int want, double thr,
                         int maxN, int* status, cudaStream_t s, const double* thrArr = nullptr);
// Inverse iteration for the selected eigenvalues (clusters reorthogonalised).
cudaError_t launchInverseIter(const EigDesc* d, int nDesc, int maxK, int* status,
                              cudaStream_t s);
// Y <- Q Y with Q = H_0 ... H_{n-3} (back-transform of tridiagonal vectors).
cudaError_t launchBackTransform(const EigDesc* d, int nDesc, int maxK, cudaStream_t s);
// Same with columns and reflectors staged in shared memory; matrices with
// n > maxN are skipped (they go through the blocked form below).
cudaError_t launchBackTransformSmem(const EigDesc* d, int nDesc, int maxK, int maxN, cudaStream_t s);
// Blocked back-transform pieces (matrices with n > kTridiagSmallMax): zero
// the upper triangle (diagonal included) of each A so its reflector columns
// form a unit lower trapezoidal V; T factors of 64-reflector blocks.
struct WyBlock {
    const double* tau;     // first tau of the block
    const double* S;       // V^T V, 64 x 64 (ld 64)
    double* T;             // out: 64 x 64 upper triangular (ld 64)
    int32_t nb, pad;       // reflectors in the block (<= 64)
};
cudaError_t launchZeroUpper(const EigDesc* d, int nDesc, cudaStream_t s);
cudaError_t launchWyT(const WyBlock* blocks, int nBlocks, cudaStream_t s);
// Bisection with one warp per eigenvalue (32-point multisection per round).
cudaError_t launchBisectWarp(const EigDesc* d, int nDesc, int mode, int want, double thr, int maxK,
                             cudaStream_t s, const double* thrArr = nullptr);

// Count of the eigenvalues of T >= thr[b] per descriptor (Sturm counts),
// written to kOut (capped by kcap); thr[b] = +inf counts none.
cudaError_t launchCountAbove(const EigDesc* d, int nDesc, const double* thr, cudaStream_t s);

// ------------------------------------------- shift-invert Lanczos (sil.cu) --
// Copy of a front's diagonal block: mode 0 the full symmetric matrix from
// its lower triangle, mode 1 the lower triangle with zeros above.
struct SilCopyDesc {
    const double* src;     // front diagonal block, ld
    int64_t ld;
    double* dst;           // n x n, ld n
    int32_t n, mode;
};
cudaError_t launchSilSymCopy(const SilCopyDesc* d, const TileRef* tiles, int nTiles, cudaStream_t s);
// count[b] = number of nonzero values of the n x n block F (ld) of descriptor b
struct SilCountDesc {
    const double* F;
    int64_t ld;
    int32_t n, pad;
};
cudaError_t launchSilCountNonzero(const SilCountDesc* d, int nDesc, unsigned long long* count, cudaStream_t s);
// sigma = -max(1e-10, 1e-9 max_j |A_jj|), then A <- A - sigma M (M: lower
// triangle of the M front's diagonal block, ld ldm).  One CTA per node.
struct SilShiftDesc {
    double* A;             // n x n, K^_ii on entry
    const double* M;
    int64_t ldm;
    double* sigma;
    int32_t n, pad;
};
cudaError_t launchSilShift(const SilShiftDesc* d, int nDesc, cudaStream_t s);
// Lanczos state of one node (all n x n arrays ld n).
struct SilDesc {
    int32_t n, target, active, pad;
    int32_t* state;        // [0] steps done, [1] stopped (breakdown or full)
    const double* B;       // (K^ - sigma M^)^-1
    double* Q;             // basis q_l (columns)
    double* MQ;            // M^ q_l
    double* QT;            // Q^T
    double* w;
    double* mw;
    double* coef;
    double* alpha;         // T diagonal
    double* beta;          // T off-diagonal (beta[j] couples j, j+1)
    const int32_t* mRow;   // local CSR of M^_ii (n + 1)
    const int32_t* mCol;
    const int64_t* mOff;   // value offsets into mBase (lower triangle)
    const double* mBase;
};
cudaError_t launchSilLanczos(const SilDesc* d, int nDesc, int maxSteps, cudaStream_t s);
// thr[b] = 1 / (hi[b] - sigma[b]) (+inf when hi[b] <= sigma[b])
cudaError_t launchSilThreshold(const double* sigma, int nDesc, const double* hi, double* thr, cudaStream_t s);
// lambda_t = 1/nu_t + sigma; rs[t] = lambda_t^-1/2, wEng[t] = 1/lambda_t (t < *kOut)
struct SilRitzDesc {
    const int32_t* kOut;
    const double* nu;
    const double* sigma;
    double* rs;
    double* wEng;
};
cudaError_t launchSilRitzScale(const SilRitzDesc* d, int nDesc, cudaStream_t s);

// --------------------------------------------------------------- misc ---
// Zero a list of (pointer, count) ranges.
cudaError_t launchZero(double* p, int64_t count, cudaStream_t s);
// Scatter permuted CSR entries into the fronts: entry e -> pool[dst[e]]
// (dst < 0: skipped).
cudaError_t launchScatterAdd(const double* vals, const int64_t* dst, int64_t nnz, double scale,
                             double* pool, cudaStream_t s);
// C[j + j*p] = w[j], j < p.
cudaError_t launchSetDiagonal(double* C, const double* w, int64_t p, cudaStream_t s);
// Symmetrise a batch of square blocks: A = (A + A^T)/2.
cudaError_t launchSymmetrize(const FrontDesc* d, int nDesc, cudaStream_t s);
// Symmetrise 32x32 tile pairs listed in tiles (desc, bi, bj with bi >= bj):
// A = (A + A^T)/2, or with mirror the upper triangle from the lower.
cudaError_t launchSymmetrizeTiles(const FrontDesc* d, const TileRef* tiles, int nTiles,
                                  cudaStream_t s, bool mirror = false);
// Transpose-copy: out(c x r) = in(r x c)^T  for a batch.
struct CopyDesc {
    const double* in;
    int64_t ldin;
    double* out;
    int64_t ldout;
    int32_t r, c;
};
cudaError_t launchTransposeBatched(const CopyDesc* d, const TileRef* tiles, int nTiles,
                                   cudaStream_t s);
// Z[perm[d] + j*n] = zt[j + d*ldz] / sqrt(norms[q * m + j]), j < m, with q
// = pencil[d] (permuted row d; null: one pencil).
cudaError_t launchUnpermute(const double* zt, int64_t ldz, int m, int64_t n, const int64_t* perm,
                            const double* norms, double* Z, cudaStream_t s,
                            const int32_t* pencil = nullptr);
// Products with M in the transposed layout over super-rows (see misc.cu):
// rows row0 .. row0 + rows - 1 (original order, rows <= kSpmmSuperRows) with
// the union column pattern ucols[colOff .. colOff + len) and the dense block
// vals[valOff + t * kSpmmSuperRows + r].
constexpr int kSpmmSuperRows = 12;
struct SpmmSuper {
    int64_t row0, colOff, valOff;
    int32_t rows, len;
    int32_t pencil, pad;   // pencil of the rows (batches of independent pencils)
};
// Rt[j + inv[o]*ld] = sum_c M[o, c] Qt[j + inv[c]*ld] for j < m <= ld (also
// into Rt2 when given).
cudaError_t launchSpmmSuperT(const SpmmSuper* sup, int64_t nsup, const int32_t* ucols, const double* vals,
                             const int64_t* inv, const double* Qt, int m, int64_t ld, double* Rt,
                             cudaStream_t s, double* Rt2 = nullptr);
// M-norms of the columns of X held transposed in permuted order:
// norms[q * m + j] = x_j^T M_q x_j over the rows of pencil q (the super-row's
// pencil), x[o, j] = zt[j + inv[o]*ld], j < m <= ld; norms holds
// pencils * m doubles.
cudaError_t launchMNormSuper(const SpmmSuper* sup, int64_t nsup, const int32_t* ucols, const double* vals,
                             const int64_t* inv, const double* zt, int m, int64_t ld, double* norms,
                             int pencils, cudaStream_t s);
// Per-element eigenvalue sensitivities of the M-normalised eigenvectors X
// (n x nmodes, original order): see sensitivity.cu.  elemType[e] (null: all
// 0) selects element e's matrices Kbar/Mbar + type * nd * nd.  weight[k] NaN
// marks a non-simple eigenvalue.  Any of gE/gRho/dE/dRho may be null.
cudaError_t launchSensitivity(int64_t nelem, int nd, const int64_t* dofmap, const int32_t* elemType,
                              const double* Kbar,
                              const double* Mbar, const double* X, int64_t n, int nmodes,
                              const double* lambda, const double* weight, double* gE,
                              double* gRho, double* dE, double* dRho, cudaStream_t s);
// Hex elasticity assembly on the GPU (assemble.cu): element matrices of
// isoparametric 8-node (order 1) or 27-node (order 2) hexahedra scaled by
// E[e] / rho[e] and summed into the CSR values kval / mval (nnz each, zeroed
// first) of the pattern rowptr / col (device arrays, sorted columns).
struct HexAssembleArgs {
    int32_t order, pad;
    int64_t nelem;
    const double* coords;      // node coordinates (3 per node)
    const int64_t* enodes;     // nelem x nn node ids
    const int64_t* dofmap;     // nelem x 3 nn global DOFs (-1 constrained)
    const double* E;
    const double* rho;
    double nu;
    const int64_t* rowptr;
    const int32_t* col;
    int64_t nnz;
    double* kval;
    double* mval;
    int* status;               // kDevBadPattern when an entry is missing
};
cudaError_t launchHexAssemble(const HexAssembleArgs& a, cudaStream_t s);

// Graph of |K| + |M| without self loops (graph.cu), neighbour lists sorted:
// cnt[v] = degree, then with xadj = prefix sums of cnt, the lists in adj.
cudaError_t launchGraphCount(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp, const int32_t* mc,
                             int64_t* cnt, cudaStream_t s);
cudaError_t launchGraphFill(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp, const int32_t* mc,
                            const int64_t* xadj, int64_t* adj, cudaStream_t s);

// out = a*x + b*y + c*z (z may be null), elementwise over n doubles.
cudaError_t launchAxpby3(int64_t n, double a, const double* x, double b, const double* y,
                         double c, const double* z, double* out, cudaStream_t s);

}  // namespace amls_b200
