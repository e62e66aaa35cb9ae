// FP64 refinement of the AMLS eigenpairs and the device-resident dense
// generalized eigensolver it uses.
//
// The elimination leaves the exact block factorisation K = L L^T (diagonal
// blocks L_ii, off-diagonal rows L_Si of every front), so K^-1 can be applied
// to a block of vectors with two tree sweeps: forward (levels bottom-up)
// x_i = L_ii^-1 r_i, r_S -= L_Si x_i, and backward (levels top-down)
// x_i = L_ii^-T (x_i - L_Si^T x_S).  The refinement is the subspace
// iteration of AMLS-SIMb (papers/Improving_eigenpairs...md:288-420) on
// nq = nev + extra vectors with T = K^-1 M (the diagonal blocks applied as
// block-triangular GEMMs with the elimination's L_ii^-1),
// accelerated by a Chebyshev
// filter: each outer iteration forms Y_c = C_c(2 T / a - I) Q, the unwanted
// part of T's spectrum being [0, a] with a = 1 / (largest Ritz value), then
//   X = T Y_c,  Kc = X^T (M Y_c),  Mc = X^T M X,  Kc c = theta Mc c,  Q <- X c
// until the relative error of every wanted Ritz value, estimated from the
// geometric contraction of successive changes, is below refineTol.
// Vectors are kept transposed (nq x n, one contiguous column per DOF, in the
// permuted order), the layout of the back-transform.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "host/engine.hpp"

namespace amls_b200 {

namespace {
constexpr int kT = kGemmTile;
constexpr int kTB = kGemmTile;
int cdiv2(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// Tiles by decreasing work (K extent x rows x columns), ties in table order:
// CTAs start in table order, so the heavy tiles go first and the light ones
// fill the last wave.
void sortByWork(std::vector<TileRef>& t, const std::vector<GemmDesc>& d) {
    auto work = [&](const TileRef& r) {
        const GemmDesc& g = d[static_cast<size_t>(r.desc)];
        int64_t kb = g.kChunk > 0 ? static_cast<int64_t>(r.pad) * g.kChunk : 0;
        int64_t ke = g.kChunk > 0 ? std::min<int64_t>(g.K, kb + g.kChunk) : g.K;
        if (g.flags & kTriKUpTo) ke = std::min<int64_t>(ke, r.n0 + kGemmTile);
        if (g.flags & kTriKFrom) kb = std::max<int64_t>(kb, r.n0);
        const int64_t rows = std::min<int64_t>(kGemmTile, g.M - r.m0);
        const int64_t cols = std::min<int64_t>(kGemmTile, g.N - r.n0);
        return std::max<int64_t>(0, ke - kb) * rows * cols;
    };
    std::stable_sort(t.begin(), t.end(), [&](const TileRef& a, const TileRef& b) { return work(a) > work(b); });
}
}  // namespace

#define LAUNCH(call)                                   \
    do {                                               \
        const int cat_ = profBegin(#call);             \
        cudaCheck((call), #call);                      \
        profEnd(cat_);                                 \
        ++launches_;                                   \
    } while (0)

// smallest `want` eigenpairs of (K, M), n x n column-major on the device;
// K and M are overwritten.  w[want] ascending, V (n x want, ld ldv).
// M = L L^T (blocked Cholesky with L^-1), C = L^-1 K L^-T by two triangular
// GEMMs, the symmetric tridiagonal eigensolver on C, V = L^-T Y.
void Engine::denseGenEigDev(double* K, double* M, int n, int want, double* w, double* V,
                            int64_t ldv, cudaStream_t s) {
    const int64_t nn = n;
    double* E = static_cast<double*>(dgE_.ensure(sizeof(double) * nn * nn));
    double* T = static_cast<double*>(dgT_.ensure(sizeof(double) * nn * nn));
    double* Linv = static_cast<double*>(dgLinv_.ensure(sizeof(double) * nn * nn));
    double* Y = static_cast<double*>(dgY_.ensure(sizeof(double) * nn * want));
    double* d = static_cast<double*>(dgD_.ensure(sizeof(double) * 3 * nn));
    double* work = static_cast<double*>(dgWork_.ensure(sizeof(double) * 6 * nn * want));
    int* kOut = static_cast<int*>(dgK_.ensure(sizeof(int) * 4));
    double* inv = static_cast<double*>(dgInv_.ensure(sizeof(double) * (size_t)((n + 63) / 64) * 4096));
    cudaCheck(cudaMemsetAsync(Linv, 0, sizeof(double) * nn * nn, s), "zero");
    Blob b;
    const CholPlan P = buildCholPlan(b, {CholItem{M, nn, nn, inv, Linv, T, -2}});
    std::vector<GemmDesc> g1(1), g2(1), g3(1);
    std::vector<TileRef> t1, t2, t3;
    auto set = [](GemmDesc& g, int64_t Mr, int64_t N, int64_t Kd, int flags, const double* A, int64_t lda,
                  const double* B, int64_t ldb, double* C, int64_t ldc) {
        g = GemmDesc{};
        g.M = static_cast<int32_t>(Mr);
        g.N = static_cast<int32_t>(N);
        g.K = static_cast<int32_t>(Kd);
        g.flags = flags;
        g.A = A;
        g.lda = lda;
        g.B = B;
        g.ldb = ldb;
        g.C = C;
        g.ldc = ldc;
        g.alpha = 1.0;
    };
    auto tiles = [](std::vector<TileRef>& t, int64_t Mr, int64_t N) {
        for (int j = 0; j < cdiv2(N, kT); ++j)
            for (int i = 0; i < cdiv2(Mr, kT); ++i) t.push_back({0, i * kT, j * kT, 0});
    };
    set(g1[0], n, n, n, kTransB | kTriKUpTo, K, nn, Linv, nn, T, nn);              // T = K L^-T
    tiles(t1, n, n);
    set(g2[0], n, n, n, kTransA | kTransB | kTriKUpTo, T, nn, Linv, nn, E, nn);    // C = T^T L^-T
    for (int j = 0; j < cdiv2(n, kT); ++j)              // C is symmetric: tiles on and below
        for (int i = j; i < cdiv2(n, kT); ++i) t2.push_back({0, i * kT, j * kT, 0});   // the diagonal
    set(g3[0], n, want, n, kTransA, Linv, nn, Y, nn, V, ldv);                       // V = L^-T Y
    tiles(t3, n, want);
    const GemmBatch b1 = addBatch(b, g1, t1), b2 = addBatch(b, g2, t2), b3 = addBatch(b, g3, t3);
    FrontDesc fe{E, nn, n, n, -2, 0};
    std::vector<TileRef> feT;                           // 32 x 32 tile pairs (tile units)
    for (int bj = 0; bj < cdiv2(n, 32); ++bj)
        for (int bi = bj; bi < cdiv2(n, 32); ++bi) feT.push_back({0, bi, bj, 0});
    EigDesc ed{};
    ed.A = E;
    ed.lda = nn;
    ed.d = d;
    ed.e = d + nn;
    ed.tau = d + 2 * nn;
    ed.n = n;
    ed.id = -2;
    ed.w = w;
    ed.Y = Y;
    ed.ldy = nn;
    ed.kcap = want;
    ed.kOut = kOut;
    ed.work = work;
    const size_t oFe = b.add(&fe, 1), oE = b.add(&ed, 1), oFeT = b.add(feT);
    std::vector<int> gOf, gFirst{0}, gSize;
    std::vector<int64_t> pOff{0};
    int nCta = 0;
    if (n > kTridiagSmallMax) {
        nCta = tridiagLargeMaxCtas(n);
        gOf.assign(static_cast<size_t>(nCta), 0);
        gSize.push_back(nCta);
    }
    const size_t oGo = b.add(gOf), oGf = b.add(gFirst), oGs = b.add(gSize), oPo = b.add(pOff);
    b.upload(dgBlob_, s);
    runCholPlan(b, P, s);
    {
        // a breakdown of the Cholesky of M (status kDevNotSpd) ends the call:
        // the caller reads the status word
        int st[2] = {0, 0};
        cudaCheck(cudaMemcpyAsync(st, status_.as<int>(), sizeof(st), cudaMemcpyDeviceToHost, s), "status");
        cudaCheck(cudaStreamSynchronize(s), "dense eigensolve");
        if (st[0] == kDevNotSpd) return;
    }
    LAUNCH(launchGemmBatched(b.dev<GemmDesc>(b1.desc), b.dev<TileRef>(b1.tiles), b1.nTiles, s));
    LAUNCH(launchGemmBatched(b.dev<GemmDesc>(b2.desc), b.dev<TileRef>(b2.tiles), b2.nTiles, s));
    LAUNCH(launchSymmetrizeTiles(b.dev<FrontDesc>(oFe), b.dev<TileRef>(oFeT), static_cast<int>(feT.size()), s,
                                 true));
    const EigDesc* dE = b.dev<EigDesc>(oE);
    if (n <= kTridiagSmallMax) LAUNCH(launchTridiagSmall(dE, 1, s));
    else {
        dgP_.ensure(sizeof(double) * kTridiagPBufs * nn);
        LAUNCH(launchTridiagLargeGroups(dE, b.dev<int>(oGo), b.dev<int>(oGf), b.dev<int>(oGs), nCta,
                                        dgP_.as<double>(), b.dev<int64_t>(oPo), n, s));
    }
    LAUNCH(launchBisectWarp(dE, 1, 2, want, 0.0, want, s));
    LAUNCH(launchInverseIter(dE, 1, want, nullptr, s));
    if (n <= kTridiagSmallMax) LAUNCH(launchBackTransformSmem(dE, 1, want, n, s));
    else backTransformBig({ed}, {want}, s);
    LAUNCH(launchGemmBatched(b.dev<GemmDesc>(b3.desc), b.dev<TileRef>(b3.tiles), b3.nTiles, s));
    // the tables live in dgBlob_ until the stream passes this point
    cudaCheck(cudaStreamSynchronize(s), "dense eigensolve");
    const double nd = n;
    catF_[4] += 4.0 / 3.0 * nd * nd * nd;
    catB_[4] += 8.0 / 3.0 * nd * nd * nd;
    catF_[0] += nd * nd * nd / 3.0;
    catF_[2] += nd * nd * nd / 3.0 + 2.0 * nd * nd * nd + 2.0 * nd * nd * want;
}

// Q (nq x n, transposed, permuted order) holds the AMLS Ritz vectors on entry
// and the refined ones on exit (its first nev rows, when `vectors`); theta
// (host, nq) likewise.  Returns the number of iterations.
int Engine::refine(double* Q, int nq, int nev, std::vector<double>& theta, bool vectors, cudaStream_t s) {
    const int64_t n = n_;
    const int64_t sz = n * nq;
    double* R = static_cast<double*>(refR_.ensure(sizeof(double) * sz));
    double* X = static_cast<double*>(refX_.ensure(sizeof(double) * sz));
    double* MX = static_cast<double*>(refMX_.ensure(sizeof(double) * sz));
    double* Kc = static_cast<double*>(refKc_.ensure(sizeof(double) * nq * nq));
    double* Mc = static_cast<double*>(refMc_.ensure(sizeof(double) * nq * nq));
    double* Vc = static_cast<double*>(refV_.ensure(sizeof(double) * nq * nq));
    double* wd = static_cast<double*>(refW_.ensure(sizeof(double) * nq));
    double* Tm = static_cast<double*>(refT_.ensure(sizeof(double) * sz));
    const double* F = kPool_.as<double>();

    // L_ii^-1 (lower triangular, n_i x n_i at eigOff) of every node comes from
    // the elimination; K^-1 is applied with block-triangular GEMMs on it.
    const double* Linv = linvPool_.as<double>();

    // ---- tables: K^-1 sweeps, Rayleigh-Ritz products, subspace update ----
    Blob b;
    std::vector<int32_t> ident(static_cast<size_t>(nq));
    for (int j = 0; j < nq; ++j) ident[static_cast<size_t>(j)] = j;
    std::vector<int64_t> colOffS;
    std::vector<int64_t> colOffStart(nodes_.size(), 0);
    for (int i : order_) {
        colOffStart[static_cast<size_t>(i)] = static_cast<int64_t>(colOffS.size());
        for (int32_t d : nodes_[static_cast<size_t>(i)].S) colOffS.push_back(static_cast<int64_t>(d) * nq);
    }
    Blob idx;
    const size_t oId = idx.add(ident), oCo = idx.add(colOffS);
    idx.upload(refIdx_, s);
    const int32_t* dId = idx.dev<int32_t>(oId);
    const int64_t* dCo = idx.dev<int64_t>(oCo);
    // All sweep descriptors live in one array (`sweep`, tiles index into it),
    // so locking converged vectors can re-point them at the active rows with
    // one upload: M = nq - L, A += L, C += L (every sweep operand A and
    // output C is a block of the vector rows; B is the factor).
    struct Tabs {
        size_t ftT, fgT, bgT, btT;
        int nft, nfg, nbg, nbt;
        // outputs of the split-K triangular products (cleared before the
        // launch, the chunks accumulate with atomics): first element and
        // columns of each node's block of T (forward) and X (backward)
        std::vector<std::pair<double*, int64_t>> ftZero, btZero;
    };
    std::vector<Tabs> tabs(static_cast<size_t>(maxLevel_) + 1);
    std::vector<GemmDesc> sweep;
    double fsolve = 0;
    for (int l = 0; l <= maxLevel_; ++l) {
        std::vector<GemmDesc> ft, bt;
        std::vector<GemmDesc> fg, bg;
        std::vector<TileRef> ftT, fgT, bgT, btT;
        for (int i : byLevel_[static_cast<size_t>(l)]) {
            const Node& nd = nodes_[static_cast<size_t>(i)];
            const int64_t ni = nd.n, si = static_cast<int64_t>(nd.S.size());
            if (ni == 0) continue;
            double* Xi = X + nd.off * nq;
            double* Ti = Tm + nd.off * nq;
            const double* Li = Linv + nd.eigOff;
            // forward: T_i = X_i L_ii^-T  (= (L_ii^-1 x_i)^T)
            GemmDesc tf{};
            tf.M = nq;
            tf.N = static_cast<int32_t>(ni);
            tf.K = static_cast<int32_t>(ni);
            tf.flags = kTransB | kTriKUpTo;
            tf.A = Xi;
            tf.lda = nq;
            tf.B = Li;
            tf.ldb = ni;
            tf.C = Ti;
            tf.ldc = nq;
            tf.alpha = 1.0;
            for (int jt = 0; jt < cdiv2(ni, kTB); ++jt)
                for (int it = 0; it < cdiv2(nq, kTB); ++it)
                    ftT.push_back({static_cast<int32_t>(ft.size()), it * kTB, jt * kTB, 0});
            ft.push_back(tf);
            // backward: X_i = T_i L_ii^-1  (= (L_ii^-T t_i)^T)
            GemmDesc tb{};
            tb.M = nq;
            tb.N = static_cast<int32_t>(ni);
            tb.K = static_cast<int32_t>(ni);
            tb.flags = kTriKFrom;
            tb.A = Ti;
            tb.lda = nq;
            tb.B = Li;
            tb.ldb = ni;
            tb.C = Xi;
            tb.ldc = nq;
            tb.alpha = 1.0;
            for (int jt = 0; jt < cdiv2(ni, kTB); ++jt)
                for (int it = 0; it < cdiv2(nq, kTB); ++it)
                    btT.push_back({static_cast<int32_t>(bt.size()), it * kTB, jt * kTB, 0});
            bt.push_back(tb);
            fsolve += 2.0 * nq * ni * ni;
            if (si > 0) {
                GemmDesc g{};
                g.M = nq;
                g.N = static_cast<int32_t>(si);
                g.K = static_cast<int32_t>(ni);
                g.flags = kTransB | kScatter | kAtomic;
                g.A = Tm + nd.off * nq;
                g.lda = nq;
                g.B = F + nd.frontOff + ni;
                g.ldb = nd.ld;
                g.C = X;
                g.alpha = -1.0;
                g.rowIdx = dId;
                g.colOff = dCo + colOffStart[static_cast<size_t>(i)];
                for (int jt = 0; jt < cdiv2(si, kTB); ++jt)
                    for (int it = 0; it < cdiv2(nq, kTB); ++it)
                        fgT.push_back({static_cast<int32_t>(fg.size()), it * kTB, jt * kTB, 0});
                fg.push_back(g);
                GemmDesc h{};
                h.M = nq;
                h.N = static_cast<int32_t>(ni);
                h.K = static_cast<int32_t>(si);
                h.flags = kGatherA | kAccumulate;
                h.A = X;
                h.lda = nq;
                h.aMap = sIdxDev_ + nd.mapCol;
                h.B = F + nd.frontOff + ni;
                h.ldb = nd.ld;
                h.C = Tm + nd.off * nq;
                h.ldc = nq;
                h.alpha = -1.0;
                h.beta = 1.0;
                for (int jt = 0; jt < cdiv2(ni, kTB); ++jt)
                    for (int it = 0; it < cdiv2(nq, kTB); ++it)
                        bgT.push_back({static_cast<int32_t>(bg.size()), it * kTB, jt * kTB, 0});
                bg.push_back(h);
                fsolve += 4.0 * nq * ni * si;
            }
        }
        auto append = [&](const std::vector<GemmDesc>& d, std::vector<TileRef>& t) {
            const int base = static_cast<int>(sweep.size());
            sweep.insert(sweep.end(), d.begin(), d.end());
            for (TileRef& r : t) r.desc += base;
        };
        // The backward products T_i -= X_S^T-gathered L_Si of the upper
        // levels have few 64 x 64 tiles (N = n_i is small) and long K = s_i:
        // below four waves of three CTAs per SM, split K into chunks of at
        // least 256 (the kernel accumulates chunks with atomics; beta is 1).
        {
            constexpr int kWaveTiles = 4 * 3 * 148;
            if (!bg.empty() && static_cast<int>(bgT.size()) < kWaveTiles) {
                const int want = cdiv2(kWaveTiles, static_cast<int64_t>(bgT.size()));
                bgT.clear();
                for (size_t q = 0; q < bg.size(); ++q) {
                    GemmDesc& h = bg[q];
                    const int split = std::min(want, h.K / 256);
                    int chunks = 1;
                    if (split >= 2) {
                        h.kChunk = (cdiv2(h.K, split) + 15) / 16 * 16;
                        chunks = cdiv2(h.K, h.kChunk);
                    }
                    for (int kc = 0; kc < chunks; ++kc)
                        for (int jt = 0; jt < cdiv2(h.N, kTB); ++jt)
                            for (int it = 0; it < cdiv2(nq, kTB); ++it)
                                bgT.push_back({static_cast<int32_t>(q), it * kTB, jt * kTB, kc});
                }
            }
        }
        // The triangular products of the upper levels (n_i of hundreds to
        // thousands, few nodes) have few tiles of very unequal K (k up to the
        // tile's column, or from it): below four waves, split K into chunks
        // of at least 256 as well, clearing the outputs first.
        {
            constexpr int kWaveTiles = 4 * 3 * 148;
            auto splitTri = [&](std::vector<GemmDesc>& d, std::vector<TileRef>& t, bool upTo,
                                std::vector<std::pair<double*, int64_t>>& zero) {
                if (d.empty() || static_cast<int>(t.size()) >= kWaveTiles) return;
                const int want = cdiv2(kWaveTiles, static_cast<int64_t>(t.size()));
                bool any = false;
                for (GemmDesc& g : d) {
                    const int split = std::min(want, g.K / 256);
                    if (split >= 2) {
                        g.kChunk = (cdiv2(g.K, split) + 15) / 16 * 16;
                        any = true;
                    }
                }
                if (!any) return;
                t.clear();
                for (size_t q = 0; q < d.size(); ++q) {
                    const GemmDesc& g = d[q];
                    const int chunks = g.kChunk > 0 ? cdiv2(g.K, g.kChunk) : 1;
                    if (g.kChunk > 0) zero.push_back({g.C, g.N});
                    for (int jt = 0; jt < cdiv2(g.N, kTB); ++jt) {
                        // K range of the tile's columns: [0, 64 (jt + 1)) or [64 jt, K)
                        const int kLo = upTo ? 0 : jt * kTB, kHi = upTo ? std::min(g.K, (jt + 1) * kTB) : g.K;
                        for (int kc = 0; kc < chunks; ++kc) {
                            const int c0 = g.kChunk > 0 ? kc * g.kChunk : 0;
                            const int c1 = g.kChunk > 0 ? std::min(g.K, c0 + g.kChunk) : g.K;
                            if (c1 <= kLo || c0 >= kHi) continue;
                            for (int it = 0; it < cdiv2(nq, kTB); ++it)
                                t.push_back({static_cast<int32_t>(q), it * kTB, jt * kTB, kc});
                        }
                    }
                }
            };
            splitTri(ft, ftT, true, tabs[static_cast<size_t>(l)].ftZero);
            splitTri(bt, btT, false, tabs[static_cast<size_t>(l)].btZero);
        }
        sortByWork(ftT, ft);
        sortByWork(fgT, fg);
        sortByWork(bgT, bg);
        sortByWork(btT, bt);
        append(ft, ftT);
        append(fg, fgT);
        append(bg, bgT);
        append(bt, btT);
        Tabs& T = tabs[static_cast<size_t>(l)];
        T.ftT = b.add(ftT); T.nft = static_cast<int>(ftT.size());
        T.fgT = b.add(fgT); T.nfg = static_cast<int>(fgT.size());
        T.bgT = b.add(bgT); T.nbg = static_cast<int>(bgT.size());
        T.btT = b.add(btT); T.nbt = static_cast<int>(btT.size());
        if (opt_.verbosity >= 3) {   // sweep plan: descriptors and 64 x 64 tiles per launch
            double fTri = 0, fOff = 0;
            for (const GemmDesc& g : ft) fTri += 1.0 * g.M * g.N * g.K;
            for (const GemmDesc& g : fg) fOff += 2.0 * g.M * g.N * g.K;
            std::fprintf(stderr,
                         "[amls_b200] sweep level %d: nodes %zu tri tiles %d (%.3g flop) off-diagonal "
                         "descs %zu tiles %d/%d (%.3g flop)\n",
                         l, ft.size(), T.nft, fTri, fg.size(), T.nfg, T.nbg, fOff);
        }
    }
    const size_t oSweep = b.add(sweep);
    // Rayleigh-Ritz products: Kc = X R^T, Mc = X MX^T (split-K over n), Q = Vc^T X
    const int chunk = 4096;
    std::vector<GemmDesc> rr(2), up(1);
    std::vector<TileRef> rrT, upT;
    for (int q = 0; q < 2; ++q) {
        GemmDesc& g = rr[static_cast<size_t>(q)];
        g.M = g.N = nq;
        g.K = static_cast<int32_t>(n);
        g.flags = kTransB;
        g.A = X;
        g.lda = nq;
        g.B = q == 0 ? R : MX;
        g.ldb = nq;
        g.C = q == 0 ? Kc : Mc;
        g.ldc = nq;
        g.alpha = 1.0;
        g.kChunk = chunk;
        // Kc and Mc are symmetric: the tiles on and below the diagonal, the
        // upper triangle mirrored afterwards
        for (int kc = 0; kc < cdiv2(n, chunk); ++kc)
            for (int jt = 0; jt < cdiv2(nq, kTB); ++jt)
                for (int it = jt; it < cdiv2(nq, kTB); ++it) rrT.push_back({q, it * kTB, jt * kTB, kc});
    }
    // subspace update Q = Vc^T X and, for the next iteration, M Q = Vc^T (M X)
    // (the first K^-1 M application's right-hand side, a GEMM instead of a
    // sparse product) and K Q = Vc^T R on the rows that will be locked (R =
    // K X holds for every row: X = K^-1 R on the active rows, and the locked
    // rows carry K Q)
    double* MQ = static_cast<double*>(refMQ_.ensure(sizeof(double) * sz));
    double* KQ = static_cast<double*>(refKQ_.ensure(sizeof(double) * sz));
    up.resize(3);
    for (int q = 0; q < 3; ++q) {
        GemmDesc& g = up[static_cast<size_t>(q)];
        g.M = q == 2 ? 0 : nq;                           // KQ rows: set when locking
        g.N = static_cast<int32_t>(n);
        g.K = nq;
        g.flags = kTransA;
        g.A = Vc;
        g.lda = nq;
        g.B = q == 0 ? X : q == 1 ? MX : R;
        g.ldb = nq;
        g.C = q == 0 ? Q : q == 1 ? MQ : KQ;
        g.ldc = nq;
        g.alpha = 1.0;
    }
    for (int q = 0; q < 3; ++q)
        for (int jt = 0; jt < cdiv2(n, kTB); ++jt)
            for (int it = 0; it < cdiv2(q == 2 ? nev : nq, kTB); ++it)
                upT.push_back({q, it * kTB, jt * kTB, 0});
    const int nUp1 = cdiv2(n, kTB) * cdiv2(nq, kTB);     // the Q = Vc^T X tiles come first
    FrontDesc sym[2] = {{Kc, nq, nq, nq, -3, 0}, {Mc, nq, nq, nq, -3, 0}};
    std::vector<TileRef> symT;                          // 32 x 32 tile pairs (tile units)
    for (int q = 0; q < 2; ++q)
        for (int bj = 0; bj < cdiv2(nq, 32); ++bj)
            for (int bi = bj; bi < cdiv2(nq, 32); ++bi) symT.push_back({q, bi, bj, 0});
    const size_t oRR = b.add(rr), oRRT = b.add(rrT), oUP = b.add(up), oUPT = b.add(upT),
                 oSym = b.add(sym, 2), oSymT = b.add(symT);
    b.upload(refBlob_, s);

    const double dn = static_cast<double>(n), dq = nq;
    // Soft locking: the leading `lock` Ritz vectors (a multiple of the tile
    // height, all with converged values) stay in the Rayleigh-Ritz basis as
    // they are (X = Q, R = K Q, M X = M Q on those rows) and get no K^-1 M
    // applications; the sweeps and sparse products run on rows [lock, nq).
    int lock = 0;
    auto setLock = [&](int L) {
        lock = L;
        std::vector<GemmDesc> act(sweep);
        for (GemmDesc& g : act) {
            g.M = nq - L;
            g.A += L;
            g.C += L;
        }
        cudaCheck(cudaMemcpyAsync(b.dev<GemmDesc>(oSweep), act.data(), sizeof(GemmDesc) * act.size(),
                                  cudaMemcpyHostToDevice, s), "lock");
    };
    auto spmmLaunch = [&](const double* Y, double* out, double* out2) {
        LAUNCH(launchSpmmSuperT(supDesc_.as<SpmmSuper>(), nSup_, supCols_.as<int32_t>(), supVal_.as<double>(),
                                invDev_.as<int64_t>(), Y + lock, nq - lock, nq, out + lock, s,
                                out2 ? out2 + lock : nullptr));
    };
    auto spmmWork = [&]() {
        const int m = nq - lock;
        catF_[8] += 2.0 * nnzM_ * m;
        catB_[8] += 12.0 * nnzM_ + 16.0 * dn * m;
    };
    auto spmm = [&](const double* Y, double* out, double* out2) {
        spmmLaunch(Y, out, out2);
        spmmWork();
    };
    // the K^-1 M application on Y (nq x n): X = K^-1 (M Y), with M Y given or
    // formed; keepR keeps R = M Y (= K X, for the Rayleigh-Ritz step), the
    // filter's inner applications form M Y in X directly
    auto applyLaunches = [&](const double* Y, const double* MY, bool keepR) {
        if (MY) {
            cudaCheck(cudaMemcpyAsync(X, MY, sizeof(double) * sz, cudaMemcpyDeviceToDevice, s), "copy");
            if (keepR) cudaCheck(cudaMemcpyAsync(R, MY, sizeof(double) * sz, cudaMemcpyDeviceToDevice, s), "copy");
        } else {
            spmmLaunch(Y, X, keepR ? R : nullptr);
        }
        const GemmDesc* sw = b.dev<GemmDesc>(oSweep);
        // clears the active rows [lock, nq) of split-K outputs (nq x cols blocks)
        auto clearRows = [&](const std::vector<std::pair<double*, int64_t>>& z) {
            for (const auto& [p0, cols] : z)
                cudaCheck(cudaMemset2DAsync(p0 + lock, sizeof(double) * static_cast<size_t>(nq), 0,
                                            sizeof(double) * static_cast<size_t>(nq - lock),
                                            static_cast<size_t>(cols), s), "clear");
        };
        for (int l = 0; l <= maxLevel_; ++l) {          // forward sweep
            const Tabs& T = tabs[static_cast<size_t>(l)];
            clearRows(T.ftZero);
            LAUNCH(launchGemmBatched(sw, b.dev<TileRef>(T.ftT), T.nft, s));
            LAUNCH(launchGemmBatched(sw, b.dev<TileRef>(T.fgT), T.nfg, s));
        }
        for (int l = maxLevel_; l >= 0; --l) {          // backward sweep
            const Tabs& T = tabs[static_cast<size_t>(l)];
            LAUNCH(launchGemmBatched(sw, b.dev<TileRef>(T.bgT), T.nbg, s));
            clearRows(T.btZero);
            LAUNCH(launchGemmBatched(sw, b.dev<TileRef>(T.btT), T.nbt, s));
        }
    };
    // The first refinement of an analysis launches eagerly (a one-shot solve
    // gains nothing from capturing); later ones capture each application the
    // first time its locked rows and buffers occur and replay the graph after
    // (the sweep descriptors it reads are re-uploaded in place, so a replay
    // sees the current ones).
    const bool useGraphs = !profiling_ && refineEagerRuns_ > 0;
    auto applyT = [&](const double* Y, const double* MY, bool keepR) {
        if (!useGraphs) {
            applyLaunches(Y, MY, keepR);
        } else {
            // everything the captured launches hold by value: the locked
            // rows, the operand and output buffers (the split-K clears write
            // into X and Tm), the launch tables and the sizes
            const std::array<uintptr_t, 10> key{static_cast<uintptr_t>(lock), reinterpret_cast<uintptr_t>(Y),
                                                reinterpret_cast<uintptr_t>(MY), keepR ? 1u : 0u,
                                                reinterpret_cast<uintptr_t>(X), reinterpret_cast<uintptr_t>(R),
                                                reinterpret_cast<uintptr_t>(Tm),
                                                reinterpret_cast<uintptr_t>(b.dev<char>(0)),
                                                static_cast<uintptr_t>(nq), static_cast<uintptr_t>(n)};
            auto it = applyGraphs_.find(key);
            if (it == applyGraphs_.end()) {
                cudaGraph_t g = nullptr;
                cudaCheck(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "capture refinement");
                const int64_t l0 = launches_;
                try {
                    applyLaunches(Y, MY, keepR);
                } catch (...) {
                    cudaStreamEndCapture(s, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                cudaCheck(cudaStreamEndCapture(s, &g), "capture refinement");
                const int64_t cnt = launches_ - l0;
                launches_ = l0;
                cudaGraphExec_t ex = nullptr;
                const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
                cudaGraphDestroy(g);
                cudaCheck(e, "instantiate refinement graph");
                it = applyGraphs_.emplace(key, std::make_pair(ex, cnt)).first;
            }
            cudaCheck(cudaGraphLaunch(it->second.first, s), "launch refinement graph");
            launches_ += it->second.second;
        }
        if (!MY) spmmWork();
        catF_[2] += fsolve * (nq - lock) / dq;
    };
    // Chebyshev recurrence buffers (degree = refine - 1)
    int cheb = std::max(0, opt_.refine - 1);
    double* Y1 = cheb >= 1 ? static_cast<double*>(refY1_.ensure(sizeof(double) * sz)) : nullptr;
    double* Y2 = cheb >= 2 ? static_cast<double*>(refY2_.ensure(sizeof(double) * sz)) : nullptr;
    std::vector<double> prev(theta.begin(), theta.end());
    std::vector<double> prevChange(static_cast<size_t>(nev), -1.0);
    bool haveMQ = false;                                 // MQ = M Q is current
    int it = 0;
    for (; it < std::max(1, opt_.refineMaxIter); ++it) {
        // filter: Y_c = C_c(2 T / a - I) Q on the damped interval [0, a] of
        // T = K^-1 M, a = 1 / (largest Ritz value), then X = T Y_c
        const double a = 1.0 / prev.back();
        const double sc = 2.0 / a;
        const double* Yc = Q;
        const double* MYc = haveMQ ? MQ : nullptr;
        if (cheb >= 1) {
            double* Ym1 = Q;
            double* Yk = Y1;
            applyT(Q, MYc, false);
            LAUNCH(launchAxpby3(sz, sc, X, -1.0, Q, 0.0, nullptr, Y1, s));     // Y1 = s T Q - Q
            for (int k = 1; k < cheb; ++k) {
                double* Yn = (k == 1) ? Y2 : (Ym1 == Q ? Y2 : Ym1);
                applyT(Yk, nullptr, false);
                // Y_{k+1} = 2 (s T Y_k - Y_k) - Y_{k-1}
                LAUNCH(launchAxpby3(sz, 2.0 * sc, X, -2.0, Yk, -1.0, Ym1, Yn, s));
                Ym1 = Yk;
                Yk = Yn;
            }
            Yc = Yk;
            MYc = nullptr;
        }
        applyT(Yc, MYc, true);                           // X = T Y_c, R = M Y_c = K X
        spmm(X, MX, nullptr);
        if (lock > 0) {
            const size_t pitch = sizeof(double) * static_cast<size_t>(nq), w = sizeof(double) * lock;
            cudaCheck(cudaMemcpy2DAsync(X, pitch, Q, pitch, w, n, cudaMemcpyDeviceToDevice, s), "lock");
            cudaCheck(cudaMemcpy2DAsync(R, pitch, KQ, pitch, w, n, cudaMemcpyDeviceToDevice, s), "lock");
            cudaCheck(cudaMemcpy2DAsync(MX, pitch, MQ, pitch, w, n, cudaMemcpyDeviceToDevice, s), "lock");
        }
        cudaCheck(cudaMemsetAsync(Kc, 0, sizeof(double) * nq * nq, s), "zero");
        cudaCheck(cudaMemsetAsync(Mc, 0, sizeof(double) * nq * nq, s), "zero");
        LAUNCH(launchGemmBatched(b.dev<GemmDesc>(oRR), b.dev<TileRef>(oRRT), static_cast<int>(rrT.size()), s));
        LAUNCH(launchSymmetrizeTiles(b.dev<FrontDesc>(oSym), b.dev<TileRef>(oSymT), static_cast<int>(symT.size()),
                                     s, true));
        denseGenEigDev(Kc, Mc, nq, nq, wd, Vc, nq, s);
        std::vector<double> th(static_cast<size_t>(nq));
        int st[2] = {0, 0};
        cudaCheck(cudaMemcpyAsync(th.data(), wd, sizeof(double) * nq, cudaMemcpyDeviceToHost, s), "theta");
        cudaCheck(cudaMemcpyAsync(st, status_.as<int>(), sizeof(st), cudaMemcpyDeviceToHost, s), "status");
        cudaCheck(cudaStreamSynchronize(s), "refine");
        if (st[0] == kDevNotSpd && cheb > 0) {
            // The filter amplifies low modes by up to C_c(2 theta_max / theta_1 - 1):
            // a trace of them in a high column can take the column over, and
            // the filtered block loses rank (Cholesky of Mc breaks down).  Q
            // is unchanged until the update below, so redo the iteration
            // with a lower degree, and keep that degree from now on.
            --cheb;
            cudaCheck(cudaMemsetAsync(status_.as<int>(), 0, 2 * sizeof(int), s), "status");
            if (opt_.verbosity > 1)
                std::fprintf(stderr, "[amls_b200] refine: filtered block lost rank, degree now %d\n", cheb);
            --it;
            continue;
        }
        catF_[2] += 2.0 * dn * dq * dq;                 // lower triangles of Kc and Mc
        catB_[2] += 8.0 * (3.0 * dn * dq);
        // error estimate per wanted value: change * r / (1 - r), r the observed
        // contraction of the change (geometric convergence)
        double est = 0.0;
        int prefix = 0;                                 // leading wanted values already below tol
        bool inPrefix = true;
        for (int j = 0; j < nev; ++j) {
            const double ch = std::fabs(th[static_cast<size_t>(j)] - prev[static_cast<size_t>(j)]) /
                              std::fabs(th[static_cast<size_t>(j)]);
            const double pc = prevChange[static_cast<size_t>(j)];
            double e;
            if (pc <= 0.0) e = (it == 0) ? 1.0 : ch;    // no ratio yet
            else {
                const double rr = std::min(0.95, ch / pc);
                e = ch * std::max(rr, 0.05) / (1.0 - rr);
            }
            est = std::max(est, std::max(e, ch * 1e-3));
            if (inPrefix && std::max(e, ch * 1e-3) <= opt_.refineTol) ++prefix;
            else inPrefix = false;
            prevChange[static_cast<size_t>(j)] = ch;
        }
        prev = th;
        if (opt_.verbosity > 1)
            std::fprintf(stderr, "[amls_b200] refine it %d: estimated max rel error %.3e, converged prefix %d\n",
                         it + 1, est, prefix);
        const bool last = est <= opt_.refineTol || it + 1 >= std::max(1, opt_.refineMaxIter);
        // rows to lock next: the converged prefix rounded down to whole tiles
        const int nextLock = last ? lock : std::max(lock, std::min(prefix, nq - 1) / kTB * kTB);
        if (!last && nextLock > 0) {
            GemmDesc kq = up[2];
            kq.M = nextLock;
            cudaCheck(cudaMemcpyAsync(b.dev<GemmDesc>(oUP) + 2, &kq, sizeof(kq), cudaMemcpyHostToDevice, s),
                      "lock");
        }
        // Q = Vc^T X, and M Q (and K Q on the rows to lock) for the next
        // iteration unless this is the last; the last needs only the nev
        // wanted rows of Q, and none when no vectors are recovered
        if (last) {
            GemmDesc q0 = up[0];
            q0.M = nev;
            cudaCheck(cudaMemcpyAsync(b.dev<GemmDesc>(oUP), &q0, sizeof(q0), cudaMemcpyHostToDevice, s), "update");
        }
        if (!last || vectors) {
            LAUNCH(launchGemmBatched(b.dev<GemmDesc>(oUP), b.dev<TileRef>(oUPT),
                                    last ? nUp1 : static_cast<int>(upT.size()), s));
            catF_[2] += (last ? static_cast<double>(nev) / dq : 2.0 + static_cast<double>(nextLock) / dq) *
                        2.0 * dn * dq * dq;
            catB_[2] += 8.0 * (last ? 2.0 : 4.0) * dn * dq;
        }
        haveMQ = !last;
        if (nextLock != lock) {
            if (opt_.verbosity > 1)
                std::fprintf(stderr, "[amls_b200] refine: %d vectors locked\n", nextLock);
            setLock(nextLock);
        }
        if (est <= opt_.refineTol) {
            ++it;
            break;
        }
    }
    theta = prev;
    if (!useGraphs) ++refineEagerRuns_;
    checkStatus("refinement");
    return it;
}

}  // namespace amls_b200
