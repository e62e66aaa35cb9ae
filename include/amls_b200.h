/* amls_b200.h - C ABI of the B200 AMLS eigensolver (libamls_b200.so).
 *
 * Solves K x = lambda M x for the lowest eigenpairs of a sparse symmetric
 * positive-definite pencil by automated multilevel substructuring (AMLS),
 * with nested dissection on the host (METIS) and every numeric phase
 * (block elimination, congruence updates, local eigensolves, projection,
 * reduced eigensolve, back-transform) in hand-written sm_100a kernels.
 *
 * Conventions (same as the reference, src/core/types.hpp:11-28):
 *   - sparse input is CSR with int64 row pointers, int32 column indices
 *     sorted within each row, float64 values; K and M symmetric (both
 *     triangles stored);
 *   - dense output is column-major;
 *   - perm[new] = old.
 * Every entry point returns an int status (AMLS_OK = 0).  No C++ exception
 * crosses this boundary; amls_last_error() gives the message of the last
 * failure on the calling thread.  A handle owns one CUDA stream and its
 * device memory; calls on one handle must not overlap.
 */
#ifndef AMLS_B200_H
#define AMLS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define AMLS_OK 0
#define AMLS_ERR_INVALID_ARGUMENT 1 /* reference: std::invalid_argument           */
#define AMLS_ERR_NOT_SPD 2          /* non-positive or NaN pivot (sparse_direct.cpp:17-22, 48-53) */
#define AMLS_ERR_ITERATION 3        /* an iterative kernel hit its iteration cap  */
#define AMLS_ERR_TIMEOUT 4          /* a bounded device-side wait expired         */
#define AMLS_ERR_OOM 5              /* device allocation failed                   */
#define AMLS_ERR_CUDA 6             /* other CUDA runtime error                   */
#define AMLS_ERR_NUMERIC 7          /* reference: std::runtime_error (solver.cpp:107-111, 148-149, 254-256) */
#define AMLS_ERR_PARTITION 8        /* METIS failure (metis_partitioner.cpp:95-96, 103-104) */
#define AMLS_ERR_NO_DEVICE 9        /* no usable CUDA device                      */

/* Options: the fields and defaults of AmlsOptions (src/amls/solver.hpp:18-30). */
typedef struct amls_options {
    int32_t nLevels;            /* 6    */
    int32_t twoPass;            /* 1    */
    int64_t leafSize;           /* 500  */
    double thresholdFactor;     /* 2.0  (eta) */
    int64_t fixedKeep;          /* 0    */
    int64_t nev;                /* 100  */
    int64_t denseProjectedMax;  /* 5000 (warning only, as in solver.cpp:285-288) */
    double shift;               /* 0.0  K <- K + shift*M */
    int32_t numThreads;         /* 0    host threads (partition/analysis)  */
    int32_t recoverVectors;     /* 1    */
    int32_t verbosity;          /* 1    */
    /* FP64 refinement of the AMLS eigenpairs (no counterpart in the
     * reference, which stops at the AMLS Ritz pairs): subspace iteration
     * with T = K^-1 M applied through the exact block factorisation of K
     * that the elimination produced (AMLS-SIMb,
     * papers/Improving_eigenpairs...md:288-420), Chebyshev-filtered, with a
     * Rayleigh-Ritz step per outer iteration.  refine = 0: off; refine = k:
     * each outer iteration applies T k times (a degree k-1 Chebyshev filter
     * on the unwanted interval [0, 1/theta_max] followed by one T step). */
    int32_t refine;             /* 0    */
    int32_t refineMaxIter;      /* 60   outer iterations */
    int32_t refineExtra;        /* extra subspace vectors beyond nev; -1 = nev/2 + 16 */
    double refineTol;           /* 1e-9: target relative eigenvalue error, estimated
                                   from the geometric contraction of the Ritz values */
    /* Arithmetic of the M-side products of the AMLS approximation (no
     * counterpart in the reference, which is FP64 throughout):
     * AMLS_PRECISION_FP64 (0): every product in FP64 on the FP64 tensor
     * cores; AMLS_PRECISION_MIXED (1): the M congruence (G L^-T, C, R), the
     * projection and the back-transform products on the BF16 tensor cores
     * with each FP64 operand split into two BF16 parts (three products, FP32
     * accumulation, relative error ~2^-16).  The factorisation of K, its
     * Schur updates, the eigensolvers and the refinement stay FP64, so the
     * refined eigenpairs reach the same accuracy. */
    int32_t precision;          /* 0    */
    /* Local eigensolver choice per node, the reference's
     * EigenpairSolver::silMode (src/amls/eigenpair_solver.hpp:28-29, 68-82):
     * 0 = automatic (shift-invert Lanczos when nnz(K^_ii) < 0.15 n_i^2 and
     * n_i >= 200, the nonzeros counted from the sparsity structure after
     * fill), 1 = shift-invert Lanczos for every node, -1 = dense for every
     * node.  Index requests with k >= 4 n_i / 5 and Lanczos runs that return
     * fewer pairs than asked (index) or none (interval) fall back to the
     * dense solver, as in the reference (:38-63). */
    int32_t silMode;            /* 0    */
} amls_options;

#define AMLS_PRECISION_FP64 0
#define AMLS_PRECISION_MIXED 1

/* slots of the timing array filled by amls_solve (seconds) */
#define AMLS_T_PARTITION 0     /* METIS + permutation + symbolic analysis (host) */
#define AMLS_T_UPLOAD 1        /* host -> device copies of the pencil            */
#define AMLS_T_ELIMINATION 2   /* front assembly, factorisation, Schur/congruence */
#define AMLS_T_CONDENSE 3      /* local eigensolves + projection (both passes)   */
#define AMLS_T_REDUCED 4       /* reduced eigensolve(s)                          */
#define AMLS_T_BACKTRANSFORM 5 /* back-transform, refinement, un-permute, M-normalise */
#define AMLS_T_TOTAL 6         /* host wall clock of the call                    */
#define AMLS_T_DEVICE 7        /* CUDA-event time of the numeric solve on the handle's stream */
#define AMLS_T_SLOTS 8

typedef struct amls_handle_s* amls_handle;

/* Fill *opt with the reference defaults. */
int amls_options_default(amls_options* opt);

/* Create a solver handle on CUDA device `device` (one stream, lazily grown
 * device arena).  Replaces constructing AmlsSolver (src/amls/solver.hpp:32). */
int amls_create(int device, amls_handle* out);
int amls_destroy(amls_handle h);

/* Message of the last failure on this thread ("" if none). */
const char* amls_last_error(void);

/* Nested dissection of the graph of |K|+|M| (host only, no GPU needed).
 * Replaces MetisPartitioner::recursiveBisection
 * (src/partition/metis_partitioner.cpp:110-179).  All output arrays are
 * caller-owned with capacity n (idx_ptr: n+1):
 *   perm[n]            perm[new] = old
 *   *n_nodes           number of tree nodes N
 *   parent[N]          parent id, -1 for the root
 *   role[N]            0 leaf, 1 separator, 2 root
 *   left[N], right[N]  children ids, -1 for leaves
 *   idx_ptr[N+1], idx[n]  node index lists (original indices) by node id */
int amls_partition(int64_t n, const int64_t* k_rowptr, const int32_t* k_col,
                   const int64_t* m_rowptr, const int32_t* m_col, int32_t nLevels,
                   int64_t leafSize, int64_t* perm, int64_t* n_nodes, int64_t* parent,
                   int32_t* role, int64_t* left, int64_t* right, int64_t* idx_ptr,
                   int64_t* idx);

/* Matrix Market input (host only).  Replaces readMatrixMarket
 * (src/io/matrix_market.cpp:48-97): coordinate format, real / double /
 * integer / pattern fields (pattern entries 1.0), general or symmetric
 * (mirrored), comments and empty lines skipped, duplicates summed.  The
 * matrix must be square.  Two calls: with rowptr/col/val NULL it sets *n and
 * *nnz; then with arrays of n+1 / nnz / nnz entries it fills the CSR (sorted
 * columns). */
int amls_mm_read(const char* path, int64_t* n, int64_t* nnz, int64_t* rowptr, int32_t* col,
                 double* val);
/* Matrix Market output of a symmetric CSR matrix: the lower triangle as
 * "real symmetric" with 17 significant digits (writeMatrixMarket,
 * src/io/matrix_market.cpp:99-115; the size line counts the entries
 * written). */
int amls_mm_write(const char* path, int64_t n, const int64_t* rowptr, const int32_t* col,
                  const double* val);

/* CSR pattern of an element mesh (host only): the union over elements of
 * the cliques of their free DOFs (dofmap[nelem * ndofe], -1 constrained),
 * columns sorted.  Two calls: with rowptr / col NULL it sets *nnz; then with
 * arrays of n+1 / nnz entries it fills them. */
int amls_element_pattern(int64_t n, int64_t nelem, int32_t ndofe, const int64_t* dofmap, int64_t* nnz,
                         int64_t* rowptr, int32_t* col);

/* Hex elasticity pencil assembled on the GPU (no counterpart in the
 * reference, whose pencils come from files or graph-Laplacian generators):
 * isoparametric 8-node (order 1) or 27-node (order 2) hexahedra with nodal
 * coordinates coords[nnodes * 3] and node ids enodes[nelem * (order+1)^3]
 * (local node a0 + (order+1)(a1 + (order+1) a2) along x, y, z), isotropic
 * elasticity with modulus E[e] and Poisson ratio nu, consistent mass with
 * density rho[e], Gauss-Legendre quadrature with order + 1 points per
 * direction; DOF 3 a + component mapped by dofmap[nelem * 3 nn] (-1
 * constrained).  The values of K and M in the CSR pattern rowptr / col (host
 * arrays, e.g. from amls_element_pattern) are written to k_val / m_val:
 * device arrays of nnz doubles with outputs_on_device = 1 (ready for
 * amls_solve_values), host arrays otherwise. */
int amls_hex_assemble(amls_handle h, int32_t order, int64_t nelem, int64_t nnodes, const double* coords,
                      const int64_t* enodes, const int64_t* dofmap, const double* E, const double* rho,
                      double nu, int64_t n, const int64_t* rowptr, const int32_t* col, double* k_val,
                      double* m_val, int32_t outputs_on_device);

/* Whole AMLS solve from host CSR arrays.  Replaces AmlsSolver::solve
 * (src/amls/solver.cpp:100-319): optional shift, partition + permutation,
 * two-pass truncation (k0 = max(4, ceil(3 nev / N)), lambda_cut = eta *
 * lambda_hat) or fixedKeep, reduced eigensolve, back-transform, un-permute
 * and M-normalisation.  Outputs (host, caller-owned):
 *   theta[nev]      ascending Ritz values (nev clamped to n)
 *   Z[n * nev]      M-normalised vectors, column-major, original ordering;
 *                   may be NULL (or recoverVectors = 0) to skip recovery
 *   *p_out          size of the final reduced problem
 *   timing[AMLS_T_SLOTS] phase seconds, may be NULL */
int amls_solve(amls_handle h, int64_t n, const int64_t* k_rowptr, const int32_t* k_col,
               const double* k_val, const int64_t* m_rowptr, const int32_t* m_col,
               const double* m_val, const amls_options* opt, double* theta, double* Z,
               int64_t* p_out, double* timing);

/* Split form of amls_solve for callers that reuse one sparsity pattern:
 * amls_analyze runs the host phase (partition, permutation, symbolic fill,
 * device plan) for a pattern; amls_solve_values then runs the numeric solve
 * for values given either as host arrays (values_on_device = 0) or as device
 * arrays of nnz(K), nnz(M) float64 already resident in HBM
 * (values_on_device = 1).  Outputs as for amls_solve; with
 * outputs_on_device = 1, theta and Z are device pointers. */
int amls_analyze(amls_handle h, int64_t n, const int64_t* k_rowptr, const int32_t* k_col,
                 const int64_t* m_rowptr, const int32_t* m_col, const amls_options* opt);
int amls_solve_values(amls_handle h, const double* k_val, const double* m_val,
                      int32_t values_on_device, double* theta, double* Z,
                      int32_t outputs_on_device, int64_t* p_out, double* timing);

/* Batch of independent pencils in one launch sequence (no counterpart in
 * the reference, which solves one pencil per AmlsSolver::solve call,
 * src/amls/solver.cpp:100-319): every pencil gets the reference's own solve
 * (its own nested dissection, two-pass truncation and reduced eigenproblem),
 * while the numeric phases run level by level over all pencils' tree nodes
 * at once.  The pencils come as one block-diagonal CSR over
 * n = pencil_off[batch] rows: pencil b owns rows and columns pencil_off[b]
 * .. pencil_off[b+1] (pencil_off[0] = 0) and has no entry outside its
 * block.  Options as for amls_solve (refine must be 0).  Outputs (host,
 * caller-owned):
 *   theta[batch * nev]  pencil b's ascending Ritz values at theta + b * nev
 *                       (nev = min(opt->nev, n))
 *   m[batch]            values per pencil (min(nev, rows of the pencil))
 *   Z[n * nev]          M-normalised vectors, column-major: pencil b's
 *                       vectors in its own rows, columns beyond m[b] zero;
 *                       may be NULL
 *   timing[AMLS_T_SLOTS] as for amls_solve, may be NULL */
int amls_solve_batch(amls_handle h, int32_t batch, const int64_t* pencil_off,
                     const int64_t* k_rowptr, const int32_t* k_col, const double* k_val,
                     const int64_t* m_rowptr, const int32_t* m_col, const double* m_val,
                     const amls_options* opt, double* theta, int64_t* m, double* Z,
                     double* timing);
/* Split form of amls_solve_batch (pattern analysis once, numeric solves on
 * host or device values, as amls_analyze / amls_solve_values). */
int amls_analyze_batch(amls_handle h, int32_t batch, const int64_t* pencil_off,
                       const int64_t* k_rowptr, const int32_t* k_col, const int64_t* m_rowptr,
                       const int32_t* m_col, const amls_options* opt);
int amls_solve_values_batch(amls_handle h, const double* k_val, const double* m_val,
                            int32_t values_on_device, double* theta, int64_t* m, double* Z,
                            int32_t outputs_on_device, double* timing);

/* Stage-by-stage numeric solve of an analysed single pencil, at the seams
 * of the reference's pipeline, so that a caller can drive its own
 * truncation policy (every stage runs on the GPU; state stays on the
 * handle):
 *   amls_eliminate      GaussianElimination::run (gaussian_elimination.cpp:
 *                       828-1088): values in (host or device arrays of
 *                       nnz(K), nnz(M)), fronts assembled, elimination and
 *                       congruence updates, shift-invert factorisations
 *   amls_condense       SubspaceCondensation::run (subspace_condensation.cpp:
 *                       18-36) with FixedCountTruncation(k) (mode 0) or
 *                       ThresholdTruncation(lambda_cut) (mode 1,
 *                       spectral_truncation.hpp:35-88): local eigensolves of
 *                       every node (dense or shift-invert by silMode) and the
 *                       projection; *p = reduced size
 *   amls_pass_modes     the pass's kept count per tree node k_node[N] and
 *                       local eigenvalues mu[p] (node-id order)
 *   amls_reduced_eig    solveProjected (solver.cpp:145-161): the lowest
 *                       min(want, p) theta of the reduced pencil; vectors = 1
 *                       keeps its eigenvectors for the back-transform
 *   amls_backtransform  backtransform + un-permute + M-normalise
 *                       (subspace_condensation.cpp:263-319, solver.cpp:
 *                       302-311): Z (n x m, column-major, m = *m)
 *   amls_refine         FP64 refinement of the back-transformed basis
 *                       (amls_options.refine / refineTol / refineMaxIter of
 *                       the analysis) to the lowest nev eigenpairs
 * amls_tree gives the analysed forest's node count, parents, sizes and
 * levels (node ids as in k_node; arrays NULL to skip). */
int amls_eliminate(amls_handle h, const double* k_val, const double* m_val, int32_t values_on_device);
int amls_condense(amls_handle h, int32_t mode, int64_t k, double lambda_cut, int64_t* p);
int amls_pass_modes(amls_handle h, int32_t* k_node, double* mu);
int amls_reduced_eig(amls_handle h, int64_t want, int32_t vectors, double* theta, int64_t* m);
int amls_backtransform(amls_handle h, double* Z, int32_t outputs_on_device, int64_t* m);
int amls_refine(amls_handle h, int64_t nev, double* theta, double* Z, int32_t outputs_on_device,
                int64_t* iters);
int amls_tree(amls_handle h, int64_t* n_nodes, int64_t* parent, int64_t* size, int32_t* level);

/* Diagnostics of the last analysis/solve on the handle:
 *   info[0] tree nodes, [1] levels, [2] p of pass A, [3] p of the final pass,
 *   [4] sum of front sizes (doubles), [5] device bytes in use,
 *   [6] kernel launches in the last numeric solve,
 *   [7] refinement iterations, [8] refinement subspace size,
 *   [9] order n of the analysed pencil, [10] nodes taking the shift-invert
 *   Lanczos branch (silMode), [11] nodes it served in the last pass (the
 *   others fell back to the dense solver) */
#define AMLS_INFO_SLOTS 16
int amls_info(amls_handle h, int64_t* info);

/* Permutation of the last analysis on the handle (amls_solve or
 * amls_analyze): perm[n] with perm[new] = old, the post-order concatenation
 * of the separator tree's node index lists (the reference's
 * IPartitioner::Result::perm, src/partition/metis_partitioner.cpp:168-175). */
int amls_permutation(amls_handle h, int64_t* perm);

/* Algorithmic work of the last numeric solve, from the host ledger built
 * from the tree and the symbolic fronts (independent of the kernels):
 *   work[0] fp64 flops, elimination      [1] bytes, elimination
 *   work[2] fp64 flops, condensation     [3] bytes, condensation
 *   work[4] fp64 flops, reduced          [5] bytes, reduced
 *   work[6] fp64 flops, back-transform   [7] bytes, back-transform */
#define AMLS_WORK_SLOTS 8
int amls_work(amls_handle h, double* work);

/* Kernel profiling: when on, every kernel launch of the handle is bracketed
 * by CUDA events on its stream and the times are summed per category:
 *   0 Cholesky (diag+panel) 1 TRSM 2 batched GEMM 3 front extend-add
 *   4 tridiagonalisation 5 bisection 6 inverse iteration 7 eigenvector
 *   back-transform 8 other (assembly, transposes, norms)
 * amls_kernel_times returns milliseconds and launch counts accumulated since
 * the last amls_set_profiling call. */
#define AMLS_PROF_CATS 9
int amls_set_profiling(amls_handle h, int32_t on);
int amls_kernel_times(amls_handle h, double* ms, int64_t* launches);
/* Algorithmic work of the last numeric solve per kernel category (same
 * categories): FP64 flops and the minimum bytes each category must move,
 * from the host ledger (tree + symbolic fronts), not from counters. */
int amls_category_work(amls_handle h, double* flops, double* bytes);

/* Batched dense generalized symmetric-definite eigensolver on the GPU,
 * lowest eigenpairs of (K_b, M_b) for b = 0..batch-1.  Replaces
 * LapackDenseEigensolver::solveIndex / solveInterval
 * (src/linalg/dense_eigensolver.cpp:44-133: dsygvx, itype 1, uplo 'L',
 * abstol 0): mode 0 = index range [il, iu] (1-based, il must be 1),
 * mode 1 = value interval (lo, hi].  Host arrays, column-major, K_b and M_b
 * of order n[b] at offsets mat_off[b] (doubles); on return
 * w[w_off[b] ...] holds m[b] ascending eigenvalues and
 * V[v_off[b] ...] the n[b] x m[b] M-orthonormal eigenvectors (capacity
 * n[b] * cap[b] doubles, cap[b] = max vectors accepted).  K and M are not
 * modified. */
int amls_sygvx_batched(amls_handle h, int32_t batch, const int64_t* n, const int64_t* mat_off,
                       const double* K, const double* M, int32_t mode, int64_t il, int64_t iu,
                       double lo, double hi, const int64_t* cap, const int64_t* w_off,
                       double* w, const int64_t* v_off, double* V, int64_t* m);

/* Per-element eigenvalue sensitivities of the last amls_solve /
 * amls_solve_values on the handle (no counterpart in the reference).  For a
 * pencil assembled from reference element pairs with per-element scales,
 * K = sum_e E_e Kbar_t(e), M = sum_e rho_e Mbar_t(e) (t(e) the element's
 * type), and the solve's M-normalised eigenvectors x_k (kept on the device):
 *   dlambda_k/dE_e = x_{k,e}^T Kbar_t(e) x_{k,e},
 *   dlambda_k/drho_e = -lambda_k x_{k,e}^T Mbar_t(e) x_{k,e}
 * (adjoint form, simple eigenvalues only).  Inputs (host):
 *   dofmap[nelem * ndofe]   global DOF of each element DOF, -1 = constrained
 *   ntypes, elemType[nelem] element types 0 .. ntypes-1 (elemType NULL: one
 *                           type, ntypes must be 1)
 *   Kbar, Mbar [ntypes * ndofe^2]  column-major element matrices per type
 *                           (ndofe <= 96)
 *   weights[nev] or NULL     w_k of the weighted sum sum_k w_k lambda_k
 *   gapTol                   modes with relative gap <= gapTol are not simple
 * Outputs (host, NULL to skip): gE[nelem], gRho[nelem] the gradient of
 * sum_k w_k lambda_k over the simple modes; dE, dRho [nelem * nev]
 * (column-major, NaN for non-simple modes); simple[nev] 1/0. */
int amls_sensitivities(amls_handle h, int64_t nelem, int32_t ndofe, const int64_t* dofmap,
                       int32_t ntypes, const int32_t* elemType, const double* Kbar,
                       const double* Mbar, const double* weights, double gapTol, double* gE,
                       double* gRho, double* dE, double* dRho, int32_t* simple);

/* Allocation-free dense generalized eigensolver (no counterpart in the
 * reference).  For callers that cannot allocate device memory: a host
 * application whose own memory pool owns every device allocation, or a
 * real-time loop that must never enter the driver's allocator.  Lowest k
 * eigenpairs of one dense pencil (K, M), M positive definite, of order
 * n <= AMLS_NOALLOC_MAX_N: same semantics as amls_sygvx_batched in index
 * mode (il = 1, iu = k).
 *   K, M   device pointers, n x n column-major (read only)
 *   w      device pointer, k eigenvalues ascending
 *   V      device pointer, n x k M-orthonormal eigenvectors, column-major
 *   *m     host: number of eigenpairs returned
 *   stream CUDA stream (cudaStream_t) or NULL for the default stream
 * No handle, and no cudaMalloc/cudaFree or other allocating call: every
 * intermediate lives in a fixed-size device array inside the library
 * (about 1.5 MB, held on each GPU that loads the library until exit).  The
 * first call on a device (and the first after its context is re-created)
 * looks up that array's device address.  The call is synchronous: it reads
 * a status word back and synchronises `stream` before returning.  Calls
 * share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  Sizes beyond the limit return
 * AMLS_ERR_INVALID_ARGUMENT; an M that is not positive definite returns
 * AMLS_ERR_NOT_SPD. */
#define AMLS_NOALLOC_MAX_N 128
int amls_sygvx_lowest_noalloc(int64_t n, const double* K, const double* M, int64_t k,
                              double* w, double* V, int64_t* m, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AMLS_B200_H */
