// AMLS engine: host analysis + device numeric pipeline for one handle.
//
// Algorithm (the reference's AmlsSolver::solve, src/amls/solver.cpp:100-319,
// re-designed for one B200):
//   analysis (host):  shift pattern, METIS nested dissection, post-order
//     offsets, symbolic fill of every node's coupling set S_i (the rows of
//     ancestors coupled to node i after elimination; the reference's
//     symbolicFill_ column masks, gaussian_elimination.cpp:221-270), front
//     layout and extend-add maps, per-level launch tables.
//   elimination (device, once per solve; the reference runs it per pass):
//     per tree level, partial Cholesky of the K fronts (L_ii, L_Si), G_i <- G_i
//     L_ii^-T on the M fronts, C_i = L_ii^-1 M^_ii L_ii^-T, R_i = Q_i - C_i
//     L_Si^T / 2, and the extend-add of UK = L_Si L_Si^T and UM = L_Si R_i^T +
//     R_i L_Si^T into the ancestors' fronts.  This is the reference's Schur
//     and congruence update (K^_aa -= K_ai X_a, M^_ab -= K_ai Y_b + (K_bi
//     Y_a)^T - K_ai WX_b, gaussian_elimination.cpp:678-826) in factored form.
//   condensation (per pass): local eigenpairs of (K^_ii, M^_ii) as the largest
//     eigenvalues nu = 1/mu of C_i (tridiagonalised once), truncation (index
//     [1, k0] in pass A, mu <= lambda_cut in pass B), and the projection of
//     subspace_condensation.cpp:129-261 on per-node panels.
//   reduced eigensolve: the largest eigenvalues of Kp^-1/2 Mp Kp^-1/2.
//   back-transform z = L^-T S q (subspace_condensation.cpp:263-319),
//     un-permutation and M-normalisation (solver.cpp:302-311).
#pragma once
#include <array>
#include <chrono>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "amls_b200.h"
#include "host/devmem.hpp"
#include "host/tree.hpp"
#include "kernels/launch.hpp"

namespace amls_b200 {

class Engine {
public:
    explicit Engine(int device);
    ~Engine();

    void analyze(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp,
                 const int32_t* mc, const amls_options& opt);
    // P independent pencils as one block-diagonal CSR (pencil b: rows and
    // columns pOff[b] .. pOff[b+1]), each partitioned on its own
    void analyzeBatch(int P, const int64_t* pOff, const int64_t* kp, const int32_t* kc,
                      const int64_t* mp, const int32_t* mc, const amls_options& opt);
    int pencils() const { return nPencils_; }
    // stage-by-stage numeric solve of one analysed pencil, at the reference's
    // seams: GaussianElimination::run, SubspaceCondensation::run with
    // FixedCount(k) (mode 0) or Threshold(lambda_cut) (mode 1),
    // solveProjected, backtransform + un-permute + M-normalise, and the FP64
    // refinement
    void stageEliminate(const double* kv, const double* mv, bool onDevice);
    void stageCondense(int mode, int k, double lambdaCut, int64_t* pOut);
    void stageModes(int32_t* kNode, double* mu) const;
    void stageReduced(int want, bool vectors, double* theta, int64_t* mOut);
    void stageBacktransform(double* Z, bool onDevice, int64_t* mOut);
    void stageRefine(int nev, double* theta, double* Z, bool onDevice, int64_t* iters);
    void tree(int64_t* nNodes, int64_t* parent, int64_t* size, int32_t* level) const;
    // theta: one pencil theta[nev]; a batch theta[q * nev + j] with
    // mOut[q] values per pencil.  Z: n x (nev or fewer for one pencil).
    void solveValues(const double* kv, const double* mv, bool valuesOnDevice, double* theta,
                     double* Z, bool outputsOnDevice, int64_t* pOut, double* timing,
                     int64_t* mOut = nullptr);
    // dense batched generalized eigensolver (amls_sygvx_batched)
    void sygvxBatched(int batch, const int64_t* n, const int64_t* matOff, const double* K,
                      const double* M, int mode, int64_t il, int64_t iu, double lo, double hi,
                      const int64_t* cap, const int64_t* wOff, double* w, const int64_t* vOff,
                      double* V, int64_t* m);

    // per-element sensitivities of the last solve's eigenpairs
    void sensitivities(int64_t nelem, int nd, const int64_t* dofmap, int32_t ntypes,
                       const int32_t* elemType, const double* Kbar,
                       const double* Mbar, const double* weights, double gapTol, double* gE,
                       double* gRho, double* dE, double* dRho, int32_t* simple);
    // hex elasticity pencil values assembled on the GPU (assemble.cu)
    void assembleHex(int order, int64_t nelem, int64_t nnodes, const double* coords, const int64_t* enodes,
                     const int64_t* dofmap, const double* E, const double* rho, double nu, int64_t n,
                     const int64_t* rowptr, const int32_t* col, double* kval, double* mval, bool outputsOnDevice);
    void info(int64_t* out) const;
    // permutation of the last analysis (perm[new] = old, n entries)
    void permutation(int64_t* out) const;
    int64_t size() const { return n_; }
    // per-category kernel timing with CUDA events on the engine stream
    static constexpr int kProfCats = 9;
    void setProfiling(bool on);
    void kernelTimes(double* ms, int64_t* counts) const;
    // algorithmic flops / bytes of the last numeric solve per kernel category
    void categoryWork(double* flops, double* bytes) const;
    void work(double* out) const;
    bool analyzed() const { return analyzed_; }

private:
    struct Node {
        int64_t off = 0, n = 0;      // permuted offset and size
        int level = 0;
        int parent = -1;
        std::vector<int> anc;        // parent .. root
        std::vector<int32_t> S;      // coupling set (permuted indices, sorted)
        int64_t ld = 0;              // n + |S|
        int64_t frontOff = 0;        // doubles into the front pools
        int64_t eigOff = 0;          // doubles into the eig matrix pool (n*n)
        int64_t vecOff = 0;          // doubles into d/e/tau pools (n)
        int64_t pathPrefix = 0;      // sum of ancestor sizes (panel rows)
        int64_t invOff = 0;          // doubles into invPool_ (64x64 diagonal-block inverses)
        // extend-add maps (offsets into the static int arrays)
        int64_t mapCol = 0;          // pmin/colOff/rowBase start (|S| entries)
        int64_t rowS = 0;            // panel row index of each S entry (|S| entries)
    };

    // pass-dependent state
    struct Pass {
        std::vector<int32_t> k;      // kept modes per node
        std::vector<int64_t> projOff;   // first mode of each node over all pencils (node-id order)
        std::vector<int64_t> localOff;  // first mode of each node in its pencil's reduced problem
        std::vector<int64_t> pp;        // reduced size per pencil
        std::vector<int64_t> credOff;   // per pencil: doubles into credPool_ (pp x pp, ld pp)
        int64_t credTotal = 0;
        int64_t p = 0;                  // modes over all pencils
        std::vector<std::vector<double>> theta;   // per pencil: reduced eigenvalues ascending
        std::vector<int> got;           // per pencil: eigenpairs of the last reduced solve
        std::vector<int64_t> vOff;      // per pencil: its eigenvectors at redY_ + vOff (ld pp)
        int mMax = 0;                   // largest got
    };

    using Clock = std::chrono::steady_clock;
    Clock::time_point numericElimination(const double* kv, const double* mv, bool valuesOnDevice, cudaStream_t s);
    void extractGraphDevice(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp, const int32_t* mc,
                            std::vector<int64_t>& xadj, std::vector<int64_t>& adj);
    void buildStatic();
    void eliminate(cudaStream_t s);
    void eliminateLaunches(cudaStream_t s);
    void dropGraphs();
    void tridiagonalizeAll(cudaStream_t s);
    void tridiagLargeAll(const std::vector<EigDesc>& large, DevBuf& pbuf, DevBuf& blob, cudaStream_t s);
    // per pencil b: mode 0 index [1, wantP[b]]; mode 1 interval nu >= thrP[b]
    // (mu <= hiP[b] = 1 / thrP[b])
    void condense(int mode, const std::vector<int>& wantP, const std::vector<double>& thrP,
                  const std::vector<double>& hiP, Pass& P, cudaStream_t s);
    // per pencil the largest wantP[b] eigenpairs of its reduced matrix: fills
    // P.theta, P.got, P.vOff, P.mMax
    void reducedSolve(Pass& P, const std::vector<int>& wantP, cudaStream_t s, bool vectors = true);
    // z^T (m x n, permuted order) into ztPool_
    void backtransform(const Pass& P, int m, cudaStream_t s);
    // M-normalise the first m rows of zt (ld ldz) and un-permute into zOut_
    void finalizeVectors(const double* zt, int64_t ldz, int m, cudaStream_t s);
    void denseGenEigDev(double* K, double* M, int n, int want, double* w, double* V, int64_t ldv,
                        cudaStream_t s);
    // Y <- Q Y for the matrices of `descs` with n > kTridiagSmallMax (k[i]
    // vectors each) by compact-WY blocks (eig_wy.cpp)
    void backTransformBig(const std::vector<EigDesc>& descs, const std::vector<int>& k, cudaStream_t s);
    int refine(double* Q, int nq, int nev, std::vector<double>& theta, bool vectors, cudaStream_t s);
    void checkStatus(const char* phase);
    bool mixed() const { return opt_.precision == AMLS_PRECISION_MIXED; }
    int mTile() const { return mixed() ? kGemmTileMixed : kGemmTile; }
    cudaError_t launchGemmM(const GemmDesc* d, const TileRef* t, int n, cudaStream_t s);
    // generic selected-eigenpair driver over prepared EigDesc tables
    void selectEigen(std::vector<EigDesc>& descs, int mode, int want, double thr, bool tridiag,
                     cudaStream_t s);
    double elapsed(cudaEvent_t a, cudaEvent_t b);
    int profBegin(const char* text);
    void profEnd(int cat);
    void profCollect();

    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    int sms_ = 148;
    bool analyzed_ = false;
    amls_options opt_{};

    // problem (a batch of nPencils_ independent pencils as one block-diagonal
    // pencil; one pencil for amls_solve)
    int64_t n_ = 0, nnzK_ = 0, nnzM_ = 0;
    int nPencils_ = 1;
    std::vector<int64_t> pOff_;                    // DOF offsets of the pencils (P + 1)
    std::vector<int> pencilOf_;                    // node -> pencil
    std::vector<int> pNodes_;                      // tree nodes per pencil
    DevBuf pencilDev_;                             // pencil of each permuted DOF (batches)
    std::vector<int64_t> perm_, inv_;
    std::vector<Node> nodes_;
    std::vector<int> order_;                       // post-order
    std::vector<std::vector<int>> byLevel_;
    int maxLevel_ = 0;
    std::vector<int32_t> owner_;                   // permuted index -> node
    int64_t frontTotal_ = 0, eigTotal_ = 0, vecTotal_ = 0, invTotal_ = 0;

    // static device data
    DevBuf kPool_, mPool_, eigPool_, dPool_, ePool_, tauPool_, invPool_;
    DevBuf gPool_;                                 // G L^-T of every front (R in its lower block)
    DevBuf linvPool_, linvScratch_;                // L_ii^-1 per node (eig layout), doubling scratch
    DevBuf kVal_, mVal_, kDst_, mDst_;             // CSR values and their front destinations
    DevBuf mRp_, mCi_, invDev_, permDev_;          // original M CSR pattern, maps
    DevBuf supDesc_, supCols_, supDst_, supVal_;   // super-rows of M (SpMM, M-norms)
    int64_t nSup_ = 0, supValTotal_ = 0;
    DevBuf staticInts_;                            // extend-add and panel maps
    DevBuf staticBlob_;                            // level launch tables
    DevBuf status_;
    Blob sblob_;
    // offsets into sblob_ for level tables
    struct GemmBatch {                          // one batched GEMM launch
        size_t desc = 0, tiles = 0;
        int nTiles = 0;
    };
    static GemmBatch addBatch(Blob& b, const std::vector<GemmDesc>& d, const std::vector<TileRef>& t);
    // Batched right-looking partial Cholesky with the diagonal-block inverses
    // and L^-1 (cholesky.cpp).  linv must be zero above the diagonal.
    struct CholItem {
        double* F;             // (ld x n) front, factored in place
        int64_t ld, n;
        double* inv;           // ceil(n / 64) x 4096 diagonal-block inverses
        double* linv;          // n x n, ld n: L^-1
        double* scratch;       // n x n, ld n
        int node;              // reported with a non-positive pivot
    };
    struct CholPlan {
        size_t fronts = 0, invd = 0, invTiles = 0;
        int nFront = 0, nInvTiles = 0, nChol = 0;
        std::vector<GemmBatch> panel, trail, dbl;
    };
    static CholPlan buildCholPlan(Blob& b, const std::vector<CholItem>& items);
    void runCholPlan(const Blob& b, const CholPlan& P, cudaStream_t s);
    struct LevelPlan {
        CholPlan chol;                             // partial Cholesky and L_ii^-1 of the fronts
        GemmBatch w;                               // W = G L^-T (all rows of the front)
        GemmBatch c;                               // C = W_ii^T L^-T
        size_t symDesc = 0, symTiles = 0;          // symmetrize eig matrices
        int nSymTiles = 0;
        size_t rDesc = 0, rTiles = 0;              // R = Q - L C / 2
        int nRTiles = 0;
        size_t uDesc = 0, uTiles = 0;              // extend-add
        int nUTiles = 0;
    };
    std::vector<LevelPlan> levelPlans_;
    std::vector<int64_t> hostKDst_, hostMDst_;

    // eigen
    bool tridiagDone_ = false;

    // ---- shift-invert Lanczos nodes (the reference's SIL, sil.cpp) ----
    struct SilNode {
        int node = -1;
        int64_t mat = 0;                           // doubles into the n^2 pools
        int64_t vec = 0;                           // doubles into silVec_ (5 n)
        int64_t inv = 0;                           // doubles into silInv_
        int64_t csr = 0;                           // row pointers of M^_ii in silMRow_ (n + 1, node-relative)
        int64_t ent = 0;                           // first entry in silMCol_ / silMOff_
    };
    struct SilLevelCopy {
        size_t desc = 0, tiles = 0;
        int nTiles = 0;
    };
    void silAnalyze(const int64_t* kp, const int32_t* kc, const int64_t* mp, const int32_t* mc);
    void silBuildStatic();                         // separator copies and leaf counts (into sblob_)
    void silChoose(cudaStream_t s);                // per solve, after front assembly: the SIL node set
    void silPlan(const std::vector<int>& set);     // buffers and tables of a SIL node set
    void silPrepare(cudaStream_t s);               // per solve: sigma, factor, (K^ - sigma M^)^-1
    // Lanczos runs and Ritz selection of one pass (mode 0 index [1, want],
    // mode 1 interval (-inf, hi]): kSel[node] = kept pairs, -1 = dense solver
    void silSelect(int mode, const std::vector<int>& wantP, const std::vector<double>& hiP,
                   std::vector<int>& kSel, cudaStream_t s);
    // Ritz vectors of the selected pairs into the engine's local form (Y, nu,
    // C Y) at the pass's offsets
    void silVectors(const std::vector<int>& kSel, const std::vector<int64_t>& projOff, cudaStream_t s);
    std::vector<int> silSep_;                      // separators picked at analysis (structure)
    std::map<int, int64_t> silSepOff_;             // their K^_ii copies in silSepK_
    int64_t silSepTotal_ = 0;
    std::vector<int> silLeafCand_;                 // leaves decided per solve
    std::vector<std::vector<int32_t>> silMPat_;    // leaf M_ii patterns (row-major keys r n + c)
    std::vector<SilCountDesc> silCountDescH_;
    size_t silCountDesc_ = 0;
    DevBuf silSepK_, silCount_, silBlobBuf_;
    Blob silBlob_;                                 // tables of the current SIL node set
    std::vector<int> silPlanSet_;
    bool silPlanned_ = false;
    size_t silLeafCopyDesc_ = 0, silLeafCopyTiles_ = 0, silSepCopyDesc_ = 0, silSepCopyTiles_ = 0;
    int silLeafCopyNTiles_ = 0, silSepCopyNTiles_ = 0;
    // stage-by-stage state
    Pass stage_;
    int stageLevel_ = 0;          // 1 eliminated, 2 condensed, 3 reduced (with vectors: 4), 5 back-transformed
    std::vector<SilNode> sil_;
    std::vector<int> silOf_;                       // node -> index into sil_ (-1)
    std::vector<int32_t> silMRowH_, silMColH_;
    std::vector<int64_t> silMOffH_;
    int64_t silMatTotal_ = 0, silVecTotal_ = 0, silInvTotal_ = 0;
    DevBuf silA_, silL_, silLinv_, silScratch_, silInv_, silB_, silQ_, silMQ_, silQT_, silVec_;
    DevBuf silState_, silSigma_, silMRow_, silMCol_, silMOff_, silRunBlob_, silThr_;
    DevBuf silS_, silX_, silP_, silYt_, silCY_, silNu_, silRs_, silWork_, silKOut_, silEigBlob_;
    CholPlan silChol_;
    GemmBatch silBGemm_;
    size_t silShiftDesc_ = 0, silLowerDesc_ = 0, silLowerTiles_ = 0;
    int silLowerNTiles_ = 0;
    std::vector<SilLevelCopy> silCopy_;            // per level: K^_ii before the in-place Cholesky
    std::vector<const double*> silCYPtr_;          // per node: C_i Y_i of the pass (SIL nodes)
    // per SIL node after silSelect: Lanczos steps and T eigen offsets of the pass
    std::vector<int> silM_;
    std::vector<int64_t> silSOff_, silNuOff_;
    int64_t silServed_ = 0;                        // nodes served by shift-invert Lanczos in the last pass

    // per-pass device buffers
    DevBuf yPool_, wPool_, kOutDev_, iiWork_, panelPool_, wtPool_, credPool_;
    DevBuf redY_, redW_, redWork_, redD_, redE_, redTau_, redK_, redP_;
    DevBuf ztPool_, zTmp_, zOut_, norms_, sqrtTheta_, passBlob_, tlBlob_, redBlob_, idxBlob_, tlLargeBlob_;
    const int32_t* sIdxDev_ = nullptr;              // S_i lists (device, static)
    const int32_t* rowSDev_ = nullptr;             // panel rows of S_i (device, static)
    std::vector<int64_t> panelOff_;                // per node (doubles), -1 none
    std::vector<int64_t> yOff_;                    // per node (doubles into yPool_)

    // refinement and the device dense eigensolver
    DevBuf dgE_, dgY_, dgT_, dgLinv_, dgD_, dgWork_, dgK_, dgBlob_, dgP_, dgInv_;
    DevBuf refR_, refX_, refMX_, refKc_, refMc_, refV_, refW_, refIdx_, refBlob_, refY1_, refY2_;
    DevBuf refT_, refMQ_, refKQ_;
    DevBuf wyS_, wyW_, wyBlob_;                    // blocked back-transform
    int refineIters_ = 0, refineNq_ = 0;
    std::vector<double> lastTheta_;                // eigenvalues of the last solve
    bool lastHasVectors_ = false;
    DevBuf senDof_, senEl_, senOut_, senType_;
    DevBuf asmCoords_, asmEnodes_, asmDof_, asmE_, asmRho_, asmRp_, asmCol_, asmK_, asmM_;

    // kernel profiling
    bool profiling_ = false;
    cudaGraphExec_t elimExec_ = nullptr;            // captured elimination schedule
    int64_t elimLaunches_ = 0;                      // kernels in it
    int elimEagerRuns_ = 0;                         // eager eliminations since the analysis
    // the refinement's K^-1 M applications (an M product and the forward and
    // backward sweeps over the tree levels), captured per (locked rows,
    // operand and output buffers) from the second refinement of an analysis
    // on and replayed after: graph and the kernels in it
    std::map<std::array<uintptr_t, 10>, std::pair<cudaGraphExec_t, int64_t>> applyGraphs_;
    int refineEagerRuns_ = 0;                       // eager refinements since the analysis
    std::vector<cudaEvent_t> evPool_;
    size_t evUsed_ = 0;
    std::vector<int> evCat_;
    std::vector<const char*> evText_;
    double profMs_[kProfCats] = {0};
    int64_t profCount_[kProfCats] = {0};
    cudaEvent_t evSolve0_ = nullptr, evSolve1_ = nullptr;
    // device buffers of the graph extraction for the partition (kept across analyses)
    DevBuf grKp_, grKc_, grMp_, grMc_, grCnt_, grAdj_;
    // pinned double buffer of the device -> host result copy (copyToHost)
    static constexpr size_t kPinChunk = size_t(16) << 20;
    char* pinRing_ = nullptr;
    cudaEvent_t pinEv_[2] = {nullptr, nullptr};
    void copyToHost(double* dst, const double* src, size_t count, cudaStream_t s);

    // diagnostics / ledger
    int64_t pA_ = 0, pFinal_ = 0, launches_ = 0;
    double work_[AMLS_WORK_SLOTS] = {0};
    double catF_[kProfCats] = {0}, catB_[kProfCats] = {0};
    double elimCatF_[kProfCats] = {0}, elimCatB_[kProfCats] = {0};
};

}  // namespace amls_b200
