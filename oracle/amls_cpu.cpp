// C++ restatement of the reference AMLS algorithm on the CPU (test
// infrastructure: the oracle's timed CPU baseline, never part of the
// product).  It follows the same reference code as oracle/amls_ref.py, in the
// reference's own language and parallel scheme: BLAS single-threaded, the
// nodes of one tree level processed by a pool of host threads
// (src/amls/thread_pool.hpp:16-43, src/amls/solver.cpp:140-143), with per-
// target locks on the shared ancestor blocks
// (src/amls/gaussian_elimination.cpp:438-448).
//
//   solve            src/amls/solver.cpp:100-319 (shift, permutation, two-pass
//                    truncation k0 = max(4, ceil(3 nev / N)), lambda_cut =
//                    eta * lambda_hat, elimination re-run per pass as
//                    runFused does (:196-209), reduced problem, back-transform,
//                    un-permute, M-normalise)
//   elimination      src/amls/gaussian_elimination.cpp:458-826 (factorNode_,
//                    solveXYAnc_ over the nonzero coupling rows, makeWX_, the
//                    K Schur and M congruence updates)
//   condensation     src/amls/subspace_condensation.cpp:45-319 (dense local
//                    eigensolves dsygvx 'I' / 'V', truncation, projectNode_,
//                    finalize, backtransform)
//   dense eigen      src/linalg/dense_eigensolver.cpp:11-133 (dsygvd, dsygvx
//                    itype 1, uplo 'L', abstol 0)
//
// LAPACK and BLAS come from the OpenBLAS build that scipy ships (LP64,
// symbols prefixed "scipy_"), opened at run time from a path the caller
// gives.  The local eigensolver follows the reference's choice: shift-invert
// Lanczos (src/amls/shift_invert_lanczos.hpp:32-203, with a dense Cholesky of
// K - sigma M in place of the sparse LDL^T and the start vector of Eigen 3.4's
// Random over the Microsoft C runtime's rand()) when nnz(K^_ii) < 0.15 n^2
// and n >= 200 (src/amls/eigenpair_solver.hpp:38-82), dense dsygvx otherwise.
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;
double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

// ---------------------------------------------------------------- LAPACK --
typedef void (*dgemm_t)(const char*, const char*, const int*, const int*, const int*, const double*,
                        const double*, const int*, const double*, const int*, const double*, double*,
                        const int*, size_t, size_t);
typedef void (*dpotrf_t)(const char*, const int*, double*, const int*, int*, size_t);
typedef void (*dpotrs_t)(const char*, const int*, const int*, const double*, const int*, double*,
                         const int*, int*, size_t);
typedef void (*dsygvx_t)(const int*, const char*, const char*, const char*, const int*, double*, const int*,
                         double*, const int*, const double*, const double*, const int*, const int*,
                         const double*, int*, double*, double*, const int*, double*, const int*, int*, int*,
                         int*, size_t, size_t, size_t);
typedef void (*dsygvd_t)(const int*, const char*, const char*, const int*, double*, const int*, double*,
                         const int*, double*, double*, const int*, int*, const int*, int*, size_t, size_t);
typedef void (*setthreads_t)(int);

struct Lapack {
    dgemm_t dgemm = nullptr;
    dpotrf_t dpotrf = nullptr;
    dpotrs_t dpotrs = nullptr;
    dsygvx_t dsygvx = nullptr;
    dsygvd_t dsygvd = nullptr;
    setthreads_t setThreads = nullptr;
    void* h = nullptr;
    void open(const char* path) {
        if (h) return;
        h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!h) throw std::runtime_error(std::string("dlopen failed: ") + dlerror());
        auto sym = [&](const char* n) {
            void* f = dlsym(h, n);
            if (!f) throw std::runtime_error(std::string("missing symbol ") + n);
            return f;
        };
        dgemm = reinterpret_cast<dgemm_t>(sym("scipy_dgemm_"));
        dpotrf = reinterpret_cast<dpotrf_t>(sym("scipy_dpotrf_"));
        dpotrs = reinterpret_cast<dpotrs_t>(sym("scipy_dpotrs_"));
        dsygvx = reinterpret_cast<dsygvx_t>(sym("scipy_dsygvx_"));
        dsygvd = reinterpret_cast<dsygvd_t>(sym("scipy_dsygvd_"));
        setThreads = reinterpret_cast<setthreads_t>(sym("scipy_openblas_set_num_threads"));
    }
};
Lapack L;

struct NotSpd : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// column-major dense matrix
struct Mat {
    int r = 0, c = 0;
    std::vector<double> a;
    Mat() = default;
    Mat(int r_, int c_) : r(r_), c(c_), a(static_cast<size_t>(r_) * c_, 0.0) {}
    double& operator()(int i, int j) { return a[static_cast<size_t>(i) + static_cast<size_t>(j) * r]; }
    double operator()(int i, int j) const { return a[static_cast<size_t>(i) + static_cast<size_t>(j) * r]; }
    double* data() { return a.data(); }
    const double* data() const { return a.data(); }
};

// C (m x n) = alpha op(A) op(B) + beta C
void gemm(char ta, char tb, int m, int n, int k, double alpha, const double* A, int lda, const double* B, int ldb,
          double beta, double* C, int ldc) {
    if (m <= 0 || n <= 0) return;
    if (k <= 0) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < m; ++i) C[i + static_cast<size_t>(j) * ldc] *= beta;
        return;
    }
    L.dgemm(&ta, &tb, &m, &n, &k, &alpha, A, &lda, B, &ldb, &beta, C, &ldc, 1, 1);
}

// sparse block in CSC (rows x cols), local indices
struct Csc {
    int rows = 0, cols = 0;
    std::vector<int64_t> cp;
    std::vector<int> ri;
    std::vector<double> v;
    Mat dense() const {
        Mat d(rows, cols);
        for (int j = 0; j < cols; ++j)
            for (int64_t e = cp[j]; e < cp[j + 1]; ++e) d(ri[e], j) += v[e];
        return d;
    }
};

// coupling block: sparse (leaf node, original entries) or dense (target)
struct Coup {
    const Csc* s = nullptr;
    const Mat* d = nullptr;
    int rows() const { return s ? s->rows : d->r; }
    int cols() const { return s ? s->cols : d->c; }
    // rows with a nonzero (the reference solves only for those columns of K_{i,a})
    std::vector<int> nonzeroRows() const {
        std::vector<char> f(static_cast<size_t>(rows()), 0);
        if (s) {
            for (size_t e = 0; e < s->ri.size(); ++e)
                f[static_cast<size_t>(s->ri[e])] = 1;   // stored entries (the sparse structure)
        } else {
            for (int j = 0; j < d->c; ++j)
                for (int i = 0; i < d->r; ++i)
                    if ((*d)(i, j) != 0.0) f[static_cast<size_t>(i)] = 1;
        }
        std::vector<int> out;
        for (int i = 0; i < rows(); ++i)
            if (f[static_cast<size_t>(i)]) out.push_back(i);
        return out;
    }
    // B^T restricted to rows idx: out (cols x |idx|) = B[idx, :]^T
    Mat rowsT(const std::vector<int>& idx) const {
        Mat out(cols(), static_cast<int>(idx.size()));
        if (s) {
            std::vector<int> pos(static_cast<size_t>(rows()), -1);
            for (size_t t = 0; t < idx.size(); ++t) pos[static_cast<size_t>(idx[t])] = static_cast<int>(t);
            for (int j = 0; j < s->cols; ++j)
                for (int64_t e = s->cp[j]; e < s->cp[j + 1]; ++e) {
                    const int p = pos[static_cast<size_t>(s->ri[e])];
                    if (p >= 0) out(j, p) += s->v[e];
                }
        } else {
            for (size_t t = 0; t < idx.size(); ++t)
                for (int j = 0; j < d->c; ++j) out(j, static_cast<int>(t)) = (*d)(idx[t], j);
        }
        return out;
    }
    // out (rows x n) = B X, X (cols x n)
    Mat mul(const Mat& X) const {
        Mat out(rows(), X.c);
        if (s) {
            for (int c = 0; c < X.c; ++c)
                for (int j = 0; j < s->cols; ++j) {
                    const double x = X(j, c);
                    if (x == 0.0) continue;
                    for (int64_t e = s->cp[j]; e < s->cp[j + 1]; ++e) out(s->ri[e], c) += s->v[e] * x;
                }
        } else {
            gemm('N', 'N', d->r, X.c, d->c, 1.0, d->data(), d->r, X.data(), X.r, 0.0, out.data(), out.r);
        }
        return out;
    }
    // out (cols x n) = B^T X, X (rows x n)
    Mat mulT(const Mat& X) const {
        Mat out(cols(), X.c);
        if (s) {
            for (int c = 0; c < X.c; ++c)
                for (int j = 0; j < s->cols; ++j) {
                    double acc = 0.0;
                    for (int64_t e = s->cp[j]; e < s->cp[j + 1]; ++e) acc += s->v[e] * X(s->ri[e], c);
                    out(j, c) = acc;
                }
        } else {
            gemm('T', 'N', d->c, X.c, d->r, 1.0, d->data(), d->r, X.data(), X.r, 0.0, out.data(), out.r);
        }
        return out;
    }
};

// the node-level thread pool of one parallel-for
void parallelFor(int count, int threads, const std::function<void(int)>& f) {
    if (threads <= 1 || count <= 1) {
        for (int i = 0; i < count; ++i) f(i);
        return;
    }
    std::atomic<int> next(0);
    std::exception_ptr err;
    std::mutex em;
    std::vector<std::thread> th;
    for (int t = 0; t < std::min(threads, count); ++t)
        th.emplace_back([&] {
            for (;;) {
                const int i = next++;
                if (i >= count) break;
                try {
                    f(i);
                } catch (...) {
                    std::lock_guard<std::mutex> lk(em);
                    if (!err) err = std::current_exception();
                }
            }
        });
    for (auto& x : th) x.join();
    if (err) std::rethrow_exception(err);
}

struct Problem {
    int N = 0;
    std::vector<int> parent, order, level, off, size;
    std::vector<std::vector<int>> children, anc, byLevel;
    int maxLevel = 0;
    std::vector<char> leaf;
    std::vector<Mat> origK, origM;                       // node diagonal blocks
    std::map<std::pair<int, int>, Csc> origKc, origMc;   // (ancestor, node) couplings
};

struct Elim {
    const Problem* P = nullptr;
    std::vector<Mat> kdiag, mdiag;                       // separator targets
    std::vector<char> kdiagSet, mdiagSet;
    std::map<std::pair<int, int>, Mat> kcoup, mcoup;
    std::vector<Mat> fact;                               // Cholesky factors (lower)
    std::vector<std::unique_ptr<std::mutex>> lockDiag;
    std::map<std::pair<int, int>, std::unique_ptr<std::mutex>> lockCoup;
    std::mutex mapMu;

    void reset() {
        const int N = P->N;
        kdiag.assign(static_cast<size_t>(N), Mat());
        mdiag.assign(static_cast<size_t>(N), Mat());
        kdiagSet.assign(static_cast<size_t>(N), 0);
        mdiagSet.assign(static_cast<size_t>(N), 0);
        kcoup.clear();
        mcoup.clear();
        fact.assign(static_cast<size_t>(N), Mat());
        lockDiag.clear();
        for (int i = 0; i < N; ++i) lockDiag.emplace_back(new std::mutex);
        lockCoup.clear();
        for (const auto& kv : P->origKc) lockCoup[kv.first].reset(new std::mutex);
        // every (hi, lo) ancestor pair of a node gets a target lock
        for (int i = 0; i < N; ++i) {
            const auto& a = P->anc[static_cast<size_t>(i)];
            for (size_t p = 0; p < a.size(); ++p)
                for (size_t q = p + 1; q < a.size(); ++q)
                    if (!lockCoup.count({a[q], a[p]})) lockCoup[{a[q], a[p]}].reset(new std::mutex);
        }
    }
    // targets (created from the original block on first use)
    Mat& kdiagT(int a) {
        if (!kdiagSet[static_cast<size_t>(a)]) {
            kdiag[static_cast<size_t>(a)] = P->origK[static_cast<size_t>(a)];
            kdiagSet[static_cast<size_t>(a)] = 1;
        }
        return kdiag[static_cast<size_t>(a)];
    }
    Mat& mdiagT(int a) {
        if (!mdiagSet[static_cast<size_t>(a)]) {
            mdiag[static_cast<size_t>(a)] = P->origM[static_cast<size_t>(a)];
            mdiagSet[static_cast<size_t>(a)] = 1;
        }
        return mdiag[static_cast<size_t>(a)];
    }
    Mat& coupT(std::map<std::pair<int, int>, Mat>& tab, const std::map<std::pair<int, int>, Csc>& orig, int hi,
               int lo) {
        std::lock_guard<std::mutex> lk(mapMu);
        auto it = tab.find({hi, lo});
        if (it == tab.end()) it = tab.emplace(std::make_pair(hi, lo), orig.at({hi, lo}).dense()).first;
        return it->second;
    }
    const Mat& khat(int i) const {
        return P->leaf[static_cast<size_t>(i)] ? P->origK[static_cast<size_t>(i)] : kdiag[static_cast<size_t>(i)];
    }
    const Mat& mhat(int i) const {
        return P->leaf[static_cast<size_t>(i)] ? P->origM[static_cast<size_t>(i)] : mdiag[static_cast<size_t>(i)];
    }
    Coup kcpl(int a, int i) {
        Coup c;
        if (P->leaf[static_cast<size_t>(i)]) c.s = &P->origKc.at({a, i});
        else c.d = &coupT(kcoup, P->origKc, a, i);
        return c;
    }
    Coup mcpl(int a, int i) {
        Coup c;
        if (P->leaf[static_cast<size_t>(i)]) c.s = &P->origMc.at({a, i});
        else c.d = &coupT(mcoup, P->origMc, a, i);
        return c;
    }
    // X <- K^_ii^-1 X
    void solve(int i, Mat& X) const {
        const Mat& F = fact[static_cast<size_t>(i)];
        const int n = F.r, nrhs = X.c;
        if (n == 0 || nrhs == 0) return;
        int info = 0;
        L.dpotrs("L", &n, &nrhs, F.data(), &n, X.data(), &n, &info, 1);
        if (info != 0) throw std::runtime_error("dpotrs failed");
    }

    void factor(int i) {
        Mat A = P->leaf[static_cast<size_t>(i)] ? P->origK[static_cast<size_t>(i)] : kdiagT(i);
        const int n = A.r;
        int info = 0;
        if (n > 0) L.dpotrf("L", &n, A.data(), &n, &info, 1);
        if (info != 0) throw NotSpd("non-positive pivot");
        fact[static_cast<size_t>(i)] = std::move(A);
    }

    // factorNode_ + solveXYAnc_ + makeWX_ + the Schur / congruence tasks
    void eliminate(int i) {
        factor(i);
        const auto& anc = P->anc[static_cast<size_t>(i)];
        if (anc.empty()) return;
        const Mat& W = mhat(i);
        const size_t na = anc.size();
        std::vector<Coup> Kc(na), Mc(na);
        std::vector<std::vector<int>> xi(na), yi(na);
        std::vector<Mat> X(na), Y(na), WX(na);
        for (size_t q = 0; q < na; ++q) {
            Kc[q] = kcpl(anc[q], i);
            Mc[q] = mcpl(anc[q], i);
            xi[q] = Kc[q].nonzeroRows();
            yi[q] = Mc[q].nonzeroRows();
            if (!xi[q].empty()) {
                X[q] = Kc[q].rowsT(xi[q]);
                solve(i, X[q]);
                Mat t(W.r, X[q].c);
                gemm('N', 'N', W.r, X[q].c, W.c, 1.0, W.data(), W.r, X[q].data(), X[q].r, 0.0, t.data(), t.r);
                solve(i, t);
                WX[q] = std::move(t);
            }
            if (!yi[q].empty()) {
                Y[q] = Mc[q].rowsT(yi[q]);
                solve(i, Y[q]);
            }
        }
        // K Schur: K^_aa[:, xi] -= K_ai X_a ; K^_{hi,lo}[:, xi_lo] -= K_{hi,i} X_lo
        for (size_t q = 0; q < na; ++q) {
            if (xi[q].empty()) continue;
            const Mat U = Kc[q].mul(X[q]);
            std::lock_guard<std::mutex> lk(*lockDiag[static_cast<size_t>(anc[q])]);
            Mat& T = kdiagT(anc[q]);
            for (size_t t = 0; t < xi[q].size(); ++t)
                for (int r = 0; r < T.r; ++r) T(r, xi[q][t]) -= U(r, static_cast<int>(t));
        }
        for (size_t p = 0; p < na; ++p)
            for (size_t q = p + 1; q < na; ++q) {
                const int hi = anc[q], lo = anc[p];
                if (xi[p].empty()) continue;
                const Mat U = Kc[q].mul(X[p]);
                std::lock_guard<std::mutex> lk(*lockCoup.at({hi, lo}));
                Mat& T = coupT(kcoup, P->origKc, hi, lo);
                for (size_t t = 0; t < xi[p].size(); ++t)
                    for (int r = 0; r < T.r; ++r) T(r, xi[p][t]) -= U(r, static_cast<int>(t));
            }
        // M congruence (diagonal and coupling targets)
        for (size_t q = 0; q < na; ++q) {
            const int a = anc[q];
            Mat U1, U2;
            if (!yi[q].empty()) U1 = Kc[q].mul(Y[q]);
            if (!xi[q].empty()) U2 = Kc[q].mul(WX[q]);
            std::lock_guard<std::mutex> lk(*lockDiag[static_cast<size_t>(a)]);
            Mat& T = mdiagT(a);
            for (size_t t = 0; t < yi[q].size(); ++t)
                for (int r = 0; r < T.r; ++r) T(r, yi[q][t]) -= U1(r, static_cast<int>(t));
            for (size_t t = 0; t < yi[q].size(); ++t)
                for (int r = 0; r < T.r; ++r) T(yi[q][t], r) -= U1(r, static_cast<int>(t));
            for (size_t t = 0; t < xi[q].size(); ++t)
                for (int r = 0; r < T.r; ++r) T(r, xi[q][t]) += U2(r, static_cast<int>(t));
        }
        for (size_t p = 0; p < na; ++p)
            for (size_t q = p + 1; q < na; ++q) {
                const int hi = anc[q], lo = anc[p];
                Mat U1, U2, U3;
                if (!yi[p].empty()) U1 = Kc[q].mul(Y[p]);     // K_{hi,i} Y_lo
                if (!yi[q].empty()) U2 = Kc[p].mul(Y[q]);     // K_{lo,i} Y_hi
                if (!xi[p].empty()) U3 = Kc[q].mul(WX[p]);    // K_{hi,i} WX_lo
                std::lock_guard<std::mutex> lk(*lockCoup.at({hi, lo}));
                Mat& T = coupT(mcoup, P->origMc, hi, lo);
                for (size_t t = 0; t < yi[p].size(); ++t)
                    for (int r = 0; r < T.r; ++r) T(r, yi[p][t]) -= U1(r, static_cast<int>(t));
                for (size_t t = 0; t < yi[q].size(); ++t)
                    for (int c = 0; c < T.c; ++c) T(yi[q][t], c) -= U2(c, static_cast<int>(t));
                for (size_t t = 0; t < xi[p].size(); ++t)
                    for (int r = 0; r < T.r; ++r) T(r, xi[p][t]) += U3(r, static_cast<int>(t));
            }
    }

    void run(int threads) {
        reset();
        for (int l = 0; l <= P->maxLevel; ++l) {
            const auto& nodes = P->byLevel[static_cast<size_t>(l)];
            parallelFor(static_cast<int>(nodes.size()), threads, [&](int t) { eliminate(nodes[static_cast<size_t>(t)]); });
        }
    }
};

// dsygvx on copies: index [1, iu] (mode 0) or interval (lo, hi] (mode 1)
void sygvx(const Mat& K0, const Mat& M0, int mode, int iu, double lo, double hi, std::vector<double>& w, Mat& V) {
    const int n = K0.r;
    w.clear();
    V = Mat(n, 0);
    if (n == 0) return;
    if (mode == 0 && iu < 1) return;
    if (mode == 1 && !(hi > lo)) return;
    Mat A = K0, B = M0;
    const int itype = 1;
    const char jobz = 'V', range = mode == 0 ? 'I' : 'V', uplo = 'L';
    const int il = 1, iuu = std::min(iu, n);
    const double abstol = 0.0;
    int m = 0, info = 0;
    std::vector<double> ww(static_cast<size_t>(n));
    Mat Z(n, n);
    std::vector<int> iwork(static_cast<size_t>(5 * n)), ifail(static_cast<size_t>(n));
    int lwork = -1;
    double wq = 0;
    L.dsygvx(&itype, &jobz, &range, &uplo, &n, A.data(), &n, B.data(), &n, &lo, &hi, &il, &iuu, &abstol, &m,
             ww.data(), Z.data(), &n, &wq, &lwork, iwork.data(), ifail.data(), &info, 1, 1, 1);
    lwork = std::max(1, static_cast<int>(wq));
    std::vector<double> work(static_cast<size_t>(lwork));
    L.dsygvx(&itype, &jobz, &range, &uplo, &n, A.data(), &n, B.data(), &n, &lo, &hi, &il, &iuu, &abstol, &m,
             ww.data(), Z.data(), &n, work.data(), &lwork, iwork.data(), ifail.data(), &info, 1, 1, 1);
    if (info != 0) throw std::runtime_error("dsygvx failed, info=" + std::to_string(info));
    w.assign(ww.begin(), ww.begin() + m);
    V = Mat(n, m);
    std::memcpy(V.data(), Z.data(), sizeof(double) * static_cast<size_t>(n) * m);
}

void sygvd(const Mat& K0, const Mat& M0, std::vector<double>& w, Mat& V) {
    const int n = K0.r;
    Mat A = K0, B = M0;
    const int itype = 1;
    int info = 0, lwork = -1, liwork = -1, iq = 0;
    double wq = 0;
    w.assign(static_cast<size_t>(n), 0.0);
    L.dsygvd(&itype, "V", "L", &n, A.data(), &n, B.data(), &n, w.data(), &wq, &lwork, &iq, &liwork, &info, 1, 1);
    lwork = std::max(1, static_cast<int>(wq));
    liwork = std::max(1, iq);
    std::vector<double> work(static_cast<size_t>(lwork));
    std::vector<int> iwork(static_cast<size_t>(liwork));
    L.dsygvd(&itype, "V", "L", &n, A.data(), &n, B.data(), &n, w.data(), work.data(), &lwork, iwork.data(), &liwork,
             &info, 1, 1);
    if (info != 0) throw std::runtime_error("dsygvd failed");
    V = std::move(A);
}

// ---------------------------------------------------- shift-invert Lanczos --
// M-inner-product Lanczos on C = (K - sigma M)^-1 M (shift_invert_lanczos.hpp:32-122)
struct Sil {
    int n = 0, m = 0;
    double shift = 0;
    Mat F, Md;                 // Cholesky factor of K - sigma M; M
    std::vector<std::vector<double>> Q;
    std::vector<double> alpha, beta, nu;
    Mat S;
    Sil(const Mat& K, const Mat& M, double sigma) : n(K.r), shift(sigma), F(K), Md(M) {
        // sparseView(1e-14): |x| > 1e-14 * 1e-12 kept
        for (double& x : Md.a)
            if (std::fabs(x) <= 1e-26) x = 0.0;
        for (size_t e = 0; e < F.a.size(); ++e) {
            const double k = std::fabs(F.a[e]) > 1e-26 ? F.a[e] : 0.0;
            F.a[e] = k - sigma * Md.a[e];
        }
        int info = 0;
        L.dpotrf("L", &n, F.data(), &n, &info, 1);
        if (info != 0) throw NotSpd("SIL: factorisation failed");
        buildSparseM();
    }
    // M as a sparse matrix (the reference's M_ = Md.sparseView), by columns
    std::vector<int> mcp, mri;
    std::vector<double> mv;
    void buildSparseM() {
        mcp.assign(static_cast<size_t>(n) + 1, 0);
        for (int j = 0; j < n; ++j) {
            for (int i = 0; i < n; ++i)
                if (Md(i, j) != 0.0) {
                    mri.push_back(i);
                    mv.push_back(Md(i, j));
                }
            mcp[static_cast<size_t>(j) + 1] = static_cast<int>(mri.size());
        }
    }
    void mulM(const double* x, double* y) const {
        for (int i = 0; i < n; ++i) y[i] = 0.0;
        for (int j = 0; j < n; ++j) {
            const double xj = x[j];
            for (int e = mcp[static_cast<size_t>(j)]; e < mcp[static_cast<size_t>(j) + 1]; ++e)
                y[mri[static_cast<size_t>(e)]] += mv[static_cast<size_t>(e)] * xj;
        }
    }
    double dotM(const std::vector<double>& a, const std::vector<double>& b) const {
        std::vector<double> mb(static_cast<size_t>(n));
        mulM(b.data(), mb.data());
        double s = 0;
        for (int i = 0; i < n; ++i) s += a[static_cast<size_t>(i)] * mb[static_cast<size_t>(i)];
        return s;
    }
    void applyC(const std::vector<double>& x, std::vector<double>& y) const {
        y.assign(static_cast<size_t>(n), 0.0);
        mulM(x.data(), y.data());
        const int one = 1;
        int info = 0;
        L.dpotrs("L", &n, &one, F.data(), &n, y.data(), &n, &info, 1);
    }
    int iterate(int ncv) {
        ncv = std::min(ncv, n);
        alpha.assign(static_cast<size_t>(ncv), 0.0);
        beta.assign(static_cast<size_t>(ncv), 0.0);
        Q.assign(static_cast<size_t>(ncv), {});
        // std::srand(12345); Vec::Random(n): -1 + 2 rand() / RAND_MAX
        std::vector<double> q0(static_cast<size_t>(n));
        uint32_t x = 12345u;
        for (int i = 0; i < n; ++i) {
            x = x * 214013u + 2531011u;
            q0[static_cast<size_t>(i)] = -1.0 + 2.0 * static_cast<double>((x >> 16) & 0x7fffu) / 32767.0;
        }
        const double mq = std::sqrt(std::max(dotM(q0, q0), 1e-300));
        for (double& v : q0) v /= mq;
        Q[0] = q0;
        int mm = 0;
        for (int j = 0; j < ncv; ++j) {
            std::vector<double> w;
            applyC(Q[static_cast<size_t>(j)], w);
            alpha[static_cast<size_t>(j)] = dotM(Q[static_cast<size_t>(j)], w);
            for (int t = 0; t < 2; ++t)
                for (int l = 0; l <= j; ++l) {
                    const double c = dotM(Q[static_cast<size_t>(l)], w);
                    for (int i = 0; i < n; ++i) w[static_cast<size_t>(i)] -= c * Q[static_cast<size_t>(l)][static_cast<size_t>(i)];
                }
            const double bj = std::sqrt(std::max(dotM(w, w), 0.0));
            mm = j + 1;
            if (bj < 1e-13 || mm == ncv) break;
            beta[static_cast<size_t>(j)] = bj;
            for (double& v : w) v /= bj;
            Q[static_cast<size_t>(j + 1)] = std::move(w);
        }
        m = mm;
        // eigenpairs of T (ascending): dense symmetric, dsygvd with B = I
        Mat T(m, m), I(m, m);
        for (int j = 0; j < m; ++j) {
            T(j, j) = alpha[static_cast<size_t>(j)];
            I(j, j) = 1.0;
            if (j + 1 < m) T(j, j + 1) = T(j + 1, j) = beta[static_cast<size_t>(j)];
        }
        sygvd(T, I, nu, S);
        return m;
    }
    double lambda(int j) const { return 1.0 / nu[static_cast<size_t>(j)] + shift; }
    double res(int j) const { return std::fabs((m > 1 ? beta[static_cast<size_t>(m - 1)] : 0.0) * S(m - 1, j)); }
    void ritz(int j, double* x) const {
        for (int i = 0; i < n; ++i) x[i] = 0.0;
        for (int l = 0; l < m; ++l)
            for (int i = 0; i < n; ++i) x[i] += S(l, j) * Q[static_cast<size_t>(l)][static_cast<size_t>(i)];
    }
};

double diagScale(const Mat& K) {
    double s = 0.0;
    for (int j = 0; j < K.r; ++j) s = std::max(s, std::fabs(K(j, j)));
    return s;
}

void silInterval(const Mat& K, const Mat& M, double lo, double hi, std::vector<double>& w, Mat& V, double tol = 1e-9) {
    const int n = K.r;
    const double scale = diagScale(K);
    const double loSane = lo > -1e100 ? lo : 0.0;
    const double sigma = std::min(0.0, loSane) - std::max(1e-10, 1e-9 * (scale > 0.0 ? scale : 1.0));
    Sil lz(K, M, sigma);
    int ncv = std::min(n, 96);
    const int cap = std::min(n, 1536);
    for (;;) {
        const int m = lz.iterate(ncv);
        int cnt = 0;
        for (int j = 0; j < m; ++j) cnt += lz.lambda(j) <= hi;
        if (cnt < m && cnt > 0 && lz.res(cnt - 1) <= tol * std::max(1.0, lz.nu[static_cast<size_t>(m - 1)])) break;
        if (ncv >= cap || m < ncv) break;
        ncv = std::min(cap, ncv * 2);
    }
    std::vector<int> pick;
    for (int j = 0; j < lz.m; ++j) {
        const double lam = lz.lambda(j);
        if (lam > hi || lam <= lo) continue;
        if (lz.res(j) > 100 * tol * std::max(1.0, lz.nu[static_cast<size_t>(lz.m - 1)])) continue;
        pick.push_back(j);
    }
    w.clear();
    V = Mat(n, static_cast<int>(pick.size()));
    for (size_t t = 0; t < pick.size(); ++t) {
        w.push_back(lz.lambda(pick[t]));
        lz.ritz(pick[t], V.data() + t * static_cast<size_t>(n));
    }
}

void silIndex(const Mat& K, const Mat& M, int k, std::vector<double>& w, Mat& V, double tol = 1e-10) {
    const int n = K.r;
    const double scale = diagScale(K);
    const double sigma = -std::max(1e-10, 1e-9 * (scale > 0.0 ? scale : 1.0));
    Sil lz(K, M, sigma);
    const int cap = std::min(n, 1536);
    int ncv = std::min(n, std::max(4 * k + 16, 48));
    for (;;) {
        const int m = lz.iterate(ncv);
        const int want = std::min(k, m);
        bool ok = true;
        for (int t = 0; t < want; ++t)
            if (lz.res(m - 1 - t) > tol * std::max(1.0, lz.nu[static_cast<size_t>(m - 1)])) ok = false;
        if (ok || ncv >= cap || m < ncv) break;
        ncv = std::min(cap, ncv * 2);
    }
    const int m = lz.m, kk = std::min(k, m);
    w.clear();
    V = Mat(n, kk);
    for (int t = 0; t < kk; ++t) {
        w.push_back(lz.lambda(m - 1 - t));
        lz.ritz(m - 1 - t, V.data() + static_cast<size_t>(t) * n);
    }
}

// EigenpairSolver::useSil_ (eigenpair_solver.hpp:68-82) with silMode 0
bool useSil(const Mat& K) {
    const int n = K.r;
    if (n < 200) return false;
    int64_t nnz = 0;
    for (double x : K.a) nnz += x != 0.0;
    return static_cast<double>(nnz) < 0.15 * static_cast<double>(n) * static_cast<double>(n);
}

struct Cond {
    int p = 0;
    std::vector<int> k, projOff;
    std::vector<std::vector<double>> mu;
    std::vector<Mat> Z;
    struct Blk {
        int r, c;
        Mat b;
    };
    std::vector<Blk> blocks;
};

// SubspaceCondensation::run with a truncation: mode 0 FixedCount(kfix), mode 1 Threshold(cut)
Cond condense(const Problem& P, Elim& E, int mode, int kfix, double cut, int threads) {
    const int N = P.N;
    Cond R;
    R.k.assign(static_cast<size_t>(N), 0);
    R.mu.assign(static_cast<size_t>(N), {});
    R.Z.assign(static_cast<size_t>(N), Mat());
    // spectral levels (:45-100)
    for (int l = 0; l <= P.maxLevel; ++l) {
        const auto& nodes = P.byLevel[static_cast<size_t>(l)];
        parallelFor(static_cast<int>(nodes.size()), threads, [&](int t) {
            const int i = nodes[static_cast<size_t>(t)];
            std::vector<double> w;
            Mat V;
            const Mat& Kh = E.khat(i);
            const Mat& Mh = E.mhat(i);
            const int n = Kh.r;
            const bool sil = useSil(Kh);
            if (mode == 1) {                              // solveLocalInterval (:38-47)
                if (sil) silInterval(Kh, Mh, -1e300, cut, w, V);
                if (!sil || w.empty()) sygvx(Kh, Mh, 1, 0, -1e300, cut, w, V);
            } else {                                      // solveLocalIndex (:51-63)
                bool done = false;
                if (sil && kfix < (n * 4) / 5) {
                    silIndex(Kh, Mh, kfix, w, V);
                    done = static_cast<int>(w.size()) == kfix;
                }
                if (!done) sygvx(Kh, Mh, 0, kfix, 0.0, 0.0, w, V);
            }
            int ki = 0;
            if (mode == 0) ki = std::min<int>(kfix, static_cast<int>(w.size()));
            else
                while (ki < static_cast<int>(w.size()) && w[static_cast<size_t>(ki)] <= cut) ++ki;
            R.k[static_cast<size_t>(i)] = ki;
            if (ki > 0) {
                R.mu[static_cast<size_t>(i)].assign(w.begin(), w.begin() + ki);
                Mat Z(V.r, ki);
                std::memcpy(Z.data(), V.data(), sizeof(double) * static_cast<size_t>(V.r) * ki);
                R.Z[static_cast<size_t>(i)] = std::move(Z);
            }
        });
    }
    // projection levels (projectNode_, :129-261)
    std::map<std::pair<int, int>, Mat> mbar;
    std::vector<std::vector<int>> mbarRow(static_cast<size_t>(N));
    std::mutex mu;
    for (int l = 0; l <= P.maxLevel; ++l) {
        const auto& nodes = P.byLevel[static_cast<size_t>(l)];
        parallelFor(static_cast<int>(nodes.size()), threads, [&](int t) {
            const int i = nodes[static_cast<size_t>(t)];
            const auto& anc = P.anc[static_cast<size_t>(i)];
            const int ki = R.k[static_cast<size_t>(i)];
            std::vector<int> rowKK;
            {
                std::lock_guard<std::mutex> lk(mu);
                rowKK = mbarRow[static_cast<size_t>(i)];
            }
            if (!anc.empty()) {
                if (!rowKK.empty()) {
                    int cols = 0;
                    std::vector<Mat*> blk;
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        for (int kk : rowKK) blk.push_back(&mbar.at({i, kk}));
                    }
                    for (Mat* b : blk) cols += b->c;
                    Mat RHS(P.size[static_cast<size_t>(i)], cols);
                    int o = 0;
                    for (Mat* b : blk) {
                        std::memcpy(RHS.data() + static_cast<size_t>(o) * RHS.r, b->data(), sizeof(double) * b->a.size());
                        o += b->c;
                    }
                    E.solve(i, RHS);
                    o = 0;
                    for (size_t q = 0; q < rowKK.size(); ++q) {
                        const int kc = blk[q]->c;
                        Mat Vk(RHS.r, kc);
                        std::memcpy(Vk.data(), RHS.data() + static_cast<size_t>(o) * RHS.r, sizeof(double) * Vk.a.size());
                        for (int a : anc) {
                            const Mat U = E.kcpl(a, i).mul(Vk);
                            Mat* tgt;
                            {
                                std::lock_guard<std::mutex> lk(mu);
                                tgt = &mbar.at({a, rowKK[q]});
                            }
                            for (size_t e = 0; e < U.a.size(); ++e) tgt->a[e] -= U.a[e];
                        }
                        o += kc;
                    }
                }
                if (ki > 0) {
                    const Mat& Zi = R.Z[static_cast<size_t>(i)];
                    const Mat& Mh = E.mhat(i);
                    Mat WMz(Mh.r, ki);
                    gemm('N', 'N', Mh.r, ki, Mh.c, 1.0, Mh.data(), Mh.r, Zi.data(), Zi.r, 0.0, WMz.data(), WMz.r);
                    E.solve(i, WMz);
                    for (int a : anc) {
                        Mat proj = E.mcpl(a, i).mul(Zi);
                        const Mat U = E.kcpl(a, i).mul(WMz);
                        for (size_t e = 0; e < proj.a.size(); ++e) proj.a[e] -= U.a[e];
                        std::lock_guard<std::mutex> lk(mu);
                        mbar[{a, i}] = std::move(proj);
                        mbarRow[static_cast<size_t>(a)].push_back(i);
                    }
                }
            }
            if (ki > 0) {
                for (int kk : rowKK) {
                    const Mat* b;
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        b = &mbar.at({i, kk});
                    }
                    const Mat& Zi = R.Z[static_cast<size_t>(i)];
                    Mat blk(ki, b->c);
                    gemm('T', 'N', ki, b->c, Zi.r, 1.0, Zi.data(), Zi.r, b->data(), b->r, 0.0, blk.data(), blk.r);
                    std::lock_guard<std::mutex> lk(mu);
                    R.blocks.push_back({i, kk, std::move(blk)});
                }
            }
            std::lock_guard<std::mutex> lk(mu);
            for (int kk : rowKK) mbar.erase({i, kk});
            mbarRow[static_cast<size_t>(i)].clear();
        });
    }
    R.projOff.assign(static_cast<size_t>(N), 0);
    int acc = 0;
    for (int i = 0; i < N; ++i) {
        R.projOff[static_cast<size_t>(i)] = acc;
        acc += R.k[static_cast<size_t>(i)];
    }
    R.p = acc;
    return R;
}

// solveProjected (solver.cpp:145-161)
void solveProjected(const Cond& R, int want, std::vector<double>& w, Mat& Q) {
    if (R.p <= 0) throw std::runtime_error("reduced problem is empty");
    Mat Mp(R.p, R.p), Kp(R.p, R.p);
    for (int i = 0; i < R.p; ++i) Mp(i, i) = 1.0;
    for (const auto& b : R.blocks) {
        const int r0 = R.projOff[static_cast<size_t>(b.r)], c0 = R.projOff[static_cast<size_t>(b.c)];
        for (int j = 0; j < b.b.c; ++j)
            for (int i = 0; i < b.b.r; ++i) {
                Mp(r0 + i, c0 + j) = b.b(i, j);
                Mp(c0 + j, r0 + i) = b.b(i, j);
            }
    }
    for (size_t i = 0; i < R.k.size(); ++i)
        for (int j = 0; j < R.k[i]; ++j) Kp(R.projOff[i] + j, R.projOff[i] + j) = R.mu[i][static_cast<size_t>(j)];
    want = std::min(want, R.p);
    if (want < R.p) sygvx(Kp, Mp, 0, want, 0.0, 0.0, w, Q);
    else sygvd(Kp, Mp, w, Q);
}

}  // namespace

extern "C" {

// K, M: CSR (n, int64 row pointers, int32 columns, both triangles) in the
// original ordering; the tree: N nodes, parent[N] (-1 root), left/right[N]
// (-1 for leaves), idx_ptr[N+1] / idx[n] the original indices per node.
// Outputs: theta[nev], Z[n * nev] (column-major, may be NULL), *p_out,
// *pA_out, timing[6] = permutation, elimination (both passes), condensation,
// reduced, back-transform, total.  Returns 0, or 1 on an error (message in
// err, capacity errcap).
int amls_cpu_solve(const char* blasPath, int threads, int64_t n, const int64_t* kp, const int32_t* kc,
                   const double* kv, const int64_t* mp, const int32_t* mc, const double* mv, int N,
                   const int64_t* parent, const int64_t* left, const int64_t* right, const int64_t* idx_ptr,
                   const int64_t* idx, int nev, double eta, int fixedKeep, int rerunElimination, double* theta,
                   double* Z, int64_t* p_out, int64_t* pA_out, double* timing, char* err, int errcap) {
    try {
        L.open(blasPath);
        L.setThreads(1);                 // BLAS single-threaded, parallel over nodes (solver.cpp:140-143)
        const auto t0 = Clock::now();
        Problem P;
        P.N = N;
        P.parent.assign(parent, parent + N);
        P.children.assign(static_cast<size_t>(N), {});
        for (int i = 0; i < N; ++i)
            if (left[i] >= 0) P.children[static_cast<size_t>(i)] = {static_cast<int>(left[i]), static_cast<int>(right[i])};
        int root = -1;
        for (int i = 0; i < N; ++i)
            if (parent[i] < 0) root = i;
        // post-order: children then self
        std::function<void(int)> post = [&](int v) {
            for (int c : P.children[static_cast<size_t>(v)]) post(c);
            P.order.push_back(v);
        };
        post(root);
        P.off.assign(static_cast<size_t>(N), 0);
        P.size.assign(static_cast<size_t>(N), 0);
        std::vector<int64_t> perm;
        int acc = 0;
        for (int i : P.order) {
            P.off[static_cast<size_t>(i)] = acc;
            P.size[static_cast<size_t>(i)] = static_cast<int>(idx_ptr[i + 1] - idx_ptr[i]);
            acc += P.size[static_cast<size_t>(i)];
            for (int64_t e = idx_ptr[i]; e < idx_ptr[i + 1]; ++e) perm.push_back(idx[e]);
        }
        if (acc != n) throw std::runtime_error("tree does not cover the matrix");
        P.level.assign(static_cast<size_t>(N), 0);
        for (int i : P.order)
            for (int c : P.children[static_cast<size_t>(i)])
                P.level[static_cast<size_t>(i)] = std::max(P.level[static_cast<size_t>(i)], P.level[static_cast<size_t>(c)] + 1);
        P.maxLevel = 0;
        for (int i = 0; i < N; ++i) P.maxLevel = std::max(P.maxLevel, P.level[static_cast<size_t>(i)]);
        P.byLevel.assign(static_cast<size_t>(P.maxLevel) + 1, {});
        for (int i : P.order) P.byLevel[static_cast<size_t>(P.level[static_cast<size_t>(i)])].push_back(i);
        P.anc.assign(static_cast<size_t>(N), {});
        P.leaf.assign(static_cast<size_t>(N), 0);
        for (int i = 0; i < N; ++i) {
            for (int64_t a = parent[i]; a >= 0; a = parent[a]) P.anc[static_cast<size_t>(i)].push_back(static_cast<int>(a));
            P.leaf[static_cast<size_t>(i)] = P.children[static_cast<size_t>(i)].empty();
        }
        // permuted blocks (permuteSymmetric, solver.cpp:48-69)
        std::vector<int64_t> inv(static_cast<size_t>(n));
        for (int64_t j = 0; j < n; ++j) inv[static_cast<size_t>(perm[static_cast<size_t>(j)])] = j;
        std::vector<int> owner(static_cast<size_t>(n));
        for (int i = 0; i < N; ++i)
            for (int r = P.off[static_cast<size_t>(i)]; r < P.off[static_cast<size_t>(i)] + P.size[static_cast<size_t>(i)]; ++r)
                owner[static_cast<size_t>(r)] = i;
        P.origK.assign(static_cast<size_t>(N), Mat());
        P.origM.assign(static_cast<size_t>(N), Mat());
        for (int i = 0; i < N; ++i) {
            P.origK[static_cast<size_t>(i)] = Mat(P.size[static_cast<size_t>(i)], P.size[static_cast<size_t>(i)]);
            P.origM[static_cast<size_t>(i)] = Mat(P.size[static_cast<size_t>(i)], P.size[static_cast<size_t>(i)]);
            for (int a : P.anc[static_cast<size_t>(i)]) {
                for (int pass = 0; pass < 2; ++pass) {
                    Csc& c = (pass ? P.origMc : P.origKc)[{a, i}];
                    c.rows = P.size[static_cast<size_t>(a)];
                    c.cols = P.size[static_cast<size_t>(i)];
                    c.cp.assign(static_cast<size_t>(c.cols) + 1, 0);
                }
            }
        }
        // coupling entries by column (node column j, ancestor row r)
        for (int pass = 0; pass < 2; ++pass) {
            const int64_t* rp = pass ? mp : kp;
            const int32_t* ci = pass ? mc : kc;
            const double* vv = pass ? mv : kv;
            auto& diag = pass ? P.origM : P.origK;
            auto& cp = pass ? P.origMc : P.origKc;
            // count, then fill (CSC over the node's local columns)
            std::map<std::pair<int, int>, std::vector<std::pair<int, std::pair<int, double>>>> ent;
            for (int64_t o = 0; o < n; ++o) {
                const int64_t r = inv[static_cast<size_t>(o)];
                const int ri = owner[static_cast<size_t>(r)];
                for (int64_t e = rp[o]; e < rp[o + 1]; ++e) {
                    const int64_t c = inv[static_cast<size_t>(ci[e])];
                    const int cn = owner[static_cast<size_t>(c)];
                    if (ri == cn) {
                        diag[static_cast<size_t>(ri)](static_cast<int>(r - P.off[static_cast<size_t>(ri)]),
                                                      static_cast<int>(c - P.off[static_cast<size_t>(ri)])) += vv[e];
                    } else if (cp.count({ri, cn})) {   // row in an ancestor of the column's node
                        ent[{ri, cn}].push_back({static_cast<int>(c - P.off[static_cast<size_t>(cn)]),
                                                 {static_cast<int>(r - P.off[static_cast<size_t>(ri)]), vv[e]}});
                    }
                }
            }
            for (auto& kvp : ent) {
                auto& v = kvp.second;
                std::stable_sort(v.begin(), v.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
                Csc& c = cp[kvp.first];
                for (const auto& t : v) ++c.cp[static_cast<size_t>(t.first) + 1];
                for (int j = 0; j < c.cols; ++j) c.cp[static_cast<size_t>(j) + 1] += c.cp[static_cast<size_t>(j)];
                c.ri.resize(v.size());
                c.v.resize(v.size());
                for (size_t t = 0; t < v.size(); ++t) {
                    c.ri[t] = v[t].second.first;
                    c.v[t] = v[t].second.second;
                }
            }
        }
        const auto t1 = Clock::now();
        Elim E;
        E.P = &P;
        nev = static_cast<int>(std::min<int64_t>(nev, n));
        double tElim = 0, tCond = 0;
        Cond res;
        int64_t pA = 0;
        auto elim = [&]() {
            const auto a = Clock::now();
            E.run(threads);
            tElim += secs(a, Clock::now());
        };
        elim();
        if (fixedKeep > 0) {
            const auto a = Clock::now();
            res = condense(P, E, 0, fixedKeep, 0.0, threads);
            tCond += secs(a, Clock::now());
        } else {
            const int k0 = std::max(4, (3 * nev + N - 1) / N);
            auto a = Clock::now();
            Cond ra = condense(P, E, 0, k0, 0.0, threads);
            tCond += secs(a, Clock::now());
            pA = ra.p;
            std::vector<double> wA;
            Mat qa;
            solveProjected(ra, std::min(nev, ra.p), wA, qa);
            if (static_cast<int>(wA.size()) < nev) throw std::runtime_error("pass A reduced problem too small");
            const double cut = eta * wA[static_cast<size_t>(nev - 1)];
            if (rerunElimination) elim();     // runFused re-runs the elimination per pass
            a = Clock::now();
            res = condense(P, E, 1, 0, cut, threads);
            tCond += secs(a, Clock::now());
        }
        const auto t3 = Clock::now();
        std::vector<double> w;
        Mat Q;
        solveProjected(res, std::min(nev, res.p), w, Q);
        const auto t4 = Clock::now();
        const int m = static_cast<int>(w.size());
        for (int j = 0; j < m; ++j) theta[j] = w[static_cast<size_t>(j)];
        if (Z) {
            // back-transform z_i = Z_i q_i - K^_ii^-1 sum_a K_{a,i}^T z_a (:263-319)
            std::vector<Mat> z(static_cast<size_t>(N));
            for (int l = P.maxLevel; l >= 0; --l) {
                const auto& nodes = P.byLevel[static_cast<size_t>(l)];
                parallelFor(static_cast<int>(nodes.size()), threads, [&](int t) {
                    const int i = nodes[static_cast<size_t>(t)];
                    const int ni = P.size[static_cast<size_t>(i)], ki = res.k[static_cast<size_t>(i)];
                    Mat yi(ni, m), rhs(ni, m);
                    if (ki > 0)
                        gemm('N', 'N', ni, m, ki, 1.0, res.Z[static_cast<size_t>(i)].data(), ni,
                             Q.data() + res.projOff[static_cast<size_t>(i)], Q.r, 0.0, yi.data(), ni);
                    for (int a : P.anc[static_cast<size_t>(i)]) {
                        const Mat u = E.kcpl(a, i).mulT(z[static_cast<size_t>(a)]);
                        for (size_t e = 0; e < u.a.size(); ++e) rhs.a[e] += u.a[e];
                    }
                    E.solve(i, rhs);
                    for (size_t e = 0; e < yi.a.size(); ++e) yi.a[e] -= rhs.a[e];
                    z[static_cast<size_t>(i)] = std::move(yi);
                });
            }
            // un-permute and M-normalise (solver.cpp:302-311)
            for (int i = 0; i < N; ++i)
                for (int c = 0; c < m; ++c)
                    for (int r = 0; r < P.size[static_cast<size_t>(i)]; ++r)
                        Z[perm[static_cast<size_t>(P.off[static_cast<size_t>(i)] + r)] + static_cast<int64_t>(c) * n] =
                            z[static_cast<size_t>(i)](r, c);
            parallelFor(m, threads, [&](int c) {
                double* x = Z + static_cast<int64_t>(c) * n;
                double mz = 0.0;
                for (int64_t r = 0; r < n; ++r) {
                    double s = 0.0;
                    for (int64_t e = mp[r]; e < mp[r + 1]; ++e) s += mv[e] * x[mc[e]];
                    mz += x[r] * s;
                }
                const double sc = 1.0 / std::sqrt(std::max(mz, 1e-300));
                for (int64_t r = 0; r < n; ++r) x[r] *= sc;
            });
        }
        const auto t5 = Clock::now();
        if (p_out) *p_out = res.p;
        if (pA_out) *pA_out = pA;
        if (timing) {
            timing[0] = secs(t0, t1);
            timing[1] = tElim;
            timing[2] = tCond;
            timing[3] = secs(t3, t4);
            timing[4] = secs(t4, t5);
            timing[5] = secs(t0, t5);
        }
        return 0;
    } catch (const std::exception& e) {
        if (err && errcap > 0) {
            std::strncpy(err, e.what(), static_cast<size_t>(errcap) - 1);
            err[errcap - 1] = 0;
        }
        return 1;
    }
}

}  // extern "C"
