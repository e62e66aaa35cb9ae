// Batched right-looking partial Cholesky with L^-1, shared by the
// elimination (the fronts of one tree level) and the dense generalized
// eigensolver of the Rayleigh-Ritz step.
//
// For each item F ((n + s) x n, ld): the top n x n lower triangle becomes
// L = chol(F_nn), the bottom s x n block L_S = F_S L^-T (the reference's
// factorNode_ + X = K^-1 K_{i,a} solves, gaussian_elimination.cpp:458-598,
// in multifrontal form), `inv` receives the 64 x 64 diagonal-block inverses
// and `linv` (n x n, ld n, zero above the diagonal on entry) L^-1.
//   per 64-wide column block J:  diagonal block factored and inverted
//     (launchCholDiag64), panel F[j1:, J] <- F[j1:, J] inv(L_JJ)^T (a GEMM in
//     place: one column tile per CTA reads its rows before writing), trailing
//     update F[j1:, j1:n] -= F[j1:, J] F[j1:n, J]^T (lower-triangle tiles);
//   L^-1 by doubling: with the diagonal blocks of size b complete, each pair
//     of neighbouring blocks A = [a0, a1), B = [a1, b1) gets
//     L^-1[B, A] = -L^-1[B, B] (L[B, A] L^-1[A, A])   (two GEMMs per step).
// Every step is one launch over all items.
#include <algorithm>

#include "host/engine.hpp"

namespace amls_b200 {

namespace {
constexpr int kT = kGemmTile;
int cdivC(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

GemmDesc gemmC(int64_t M, int64_t N, int64_t K, int flags, const double* A, int64_t lda,
               const double* B, int64_t ldb, double* C, int64_t ldc, double alpha, double beta) {
    GemmDesc d{};
    d.M = static_cast<int32_t>(M);
    d.N = static_cast<int32_t>(N);
    d.K = static_cast<int32_t>(K);
    d.flags = flags;
    d.A = A;
    d.lda = lda;
    d.B = B;
    d.ldb = ldb;
    d.C = C;
    d.ldc = ldc;
    d.alpha = alpha;
    d.beta = beta;
    return d;
}

void tilesOf(std::vector<TileRef>& t, int desc, int64_t M, int64_t N) {
    for (int j = 0; j < cdivC(N, kT); ++j)
        for (int i = 0; i < cdivC(M, kT); ++i) t.push_back({desc, i * kT, j * kT, 0});
}
}  // namespace

#define LAUNCH(call)                                   \
    do {                                               \
        const int cat_ = profBegin(#call);             \
        cudaCheck((call), #call);                      \
        profEnd(cat_);                                 \
        ++launches_;                                   \
    } while (0)

Engine::GemmBatch Engine::addBatch(Blob& b, const std::vector<GemmDesc>& d, const std::vector<TileRef>& t) {
    GemmBatch g;
    g.desc = b.add(d);
    g.tiles = b.add(t);
    g.nTiles = static_cast<int>(t.size());
    return g;
}

Engine::CholPlan Engine::buildCholPlan(Blob& b, const std::vector<CholItem>& items) {
    CholPlan P;
    std::vector<FrontDesc> fr;
    std::vector<TrsmDesc> iv;
    std::vector<TileRef> it;
    int64_t maxN = 0;
    for (const CholItem& c : items) {
        FrontDesc f{};
        f.F = c.F;
        f.ld = c.ld;
        f.n = static_cast<int32_t>(c.n);
        f.rows = static_cast<int32_t>(c.ld);
        f.node = c.node;
        fr.push_back(f);
        TrsmDesc t{};
        t.L = c.F;
        t.ldl = c.ld;
        t.X = c.linv;
        t.ldx = c.n;
        t.n = static_cast<int32_t>(c.n);
        t.inv = c.inv;
        for (int J = 0; J < cdivC(c.n, 64); ++J) it.push_back({static_cast<int32_t>(iv.size()), J, 0, 0});
        iv.push_back(t);
        maxN = std::max(maxN, c.n);
    }
    P.fronts = b.add(fr);
    P.invd = b.add(iv);
    P.invTiles = b.add(it);
    P.nFront = static_cast<int>(fr.size());
    P.nInvTiles = static_cast<int>(it.size());
    P.nChol = cdivC(maxN, 64);
    for (int J = 0; J < P.nChol; ++J) {
        std::vector<GemmDesc> dp, dt;
        std::vector<TileRef> tp, tt;
        for (const CholItem& c : items) {
            const int64_t n = c.n, ld = c.ld, j0 = static_cast<int64_t>(J) * 64;
            if (j0 >= n) continue;
            const int64_t nb = std::min<int64_t>(64, n - j0), j1 = j0 + nb;
            double* Fp = c.F + j1 + j0 * ld;
            if (ld > j1) {
                dp.push_back(gemmC(ld - j1, nb, nb, kTransB | kTriKUpTo, Fp, ld, c.inv + static_cast<int64_t>(J) * 4096,
                                   64, Fp, ld, 1.0, 0.0));
                tilesOf(tp, static_cast<int>(dp.size()) - 1, ld - j1, nb);
            }
            if (n > j1) {
                const int d = static_cast<int>(dt.size());
                dt.push_back(gemmC(ld - j1, n - j1, nb, kTransB | kAccumulate, Fp, ld, Fp, ld, c.F + j1 + j1 * ld, ld,
                                   -1.0, 1.0));
                for (int jt = 0; jt < cdivC(n - j1, kT); ++jt)
                    for (int i = 0; i < cdivC(ld - j1, kT); ++i)
                        if ((i + 1) * kT > jt * kT) tt.push_back({d, i * kT, jt * kT, 0});
            }
        }
        P.panel.push_back(addBatch(b, dp, tp));
        P.trail.push_back(addBatch(b, dt, tt));
    }
    for (int64_t blk = 64; blk < maxN; blk *= 2) {
        std::vector<GemmDesc> d1, d2;
        std::vector<TileRef> t1, t2;
        for (const CholItem& c : items) {
            const int64_t n = c.n, ld = c.ld;
            for (int64_t a0 = 0; a0 + blk < n; a0 += 2 * blk) {
                const int64_t a1 = a0 + blk, b1 = std::min(n, a0 + 2 * blk);
                d1.push_back(gemmC(b1 - a1, a1 - a0, a1 - a0, kTriKFrom, c.F + a1 + a0 * ld, ld,
                                   c.linv + a0 + a0 * n, n, c.scratch + a1 + a0 * n, n, 1.0, 0.0));
                tilesOf(t1, static_cast<int>(d1.size()) - 1, b1 - a1, a1 - a0);
                d2.push_back(gemmC(b1 - a1, a1 - a0, b1 - a1, kTriAUpTo, c.linv + a1 + a1 * n, n,
                                   c.scratch + a1 + a0 * n, n, c.linv + a1 + a0 * n, n, -1.0, 0.0));
                tilesOf(t2, static_cast<int>(d2.size()) - 1, b1 - a1, a1 - a0);
            }
        }
        P.dbl.push_back(addBatch(b, d1, t1));
        P.dbl.push_back(addBatch(b, d2, t2));
    }
    return P;
}

void Engine::runCholPlan(const Blob& b, const CholPlan& P, cudaStream_t s) {
    const FrontDesc* fr = b.dev<FrontDesc>(P.fronts);
    const TrsmDesc* iv = b.dev<TrsmDesc>(P.invd);
    for (int J = 0; J < P.nChol; ++J) {
        LAUNCH(launchCholDiag64(fr, iv, P.nFront, J, status_.as<int>(), s));
        const GemmBatch& p = P.panel[static_cast<size_t>(J)];
        const GemmBatch& t = P.trail[static_cast<size_t>(J)];
        LAUNCH(launchGemmBatched(b.dev<GemmDesc>(p.desc), b.dev<TileRef>(p.tiles), p.nTiles, s));
        LAUNCH(launchGemmBatched(b.dev<GemmDesc>(t.desc), b.dev<TileRef>(t.tiles), t.nTiles, s));
    }
    LAUNCH(launchPlaceDiagInv(iv, b.dev<TileRef>(P.invTiles), P.nInvTiles, s));
    for (const GemmBatch& g : P.dbl)
        LAUNCH(launchGemmBatched(b.dev<GemmDesc>(g.desc), b.dev<TileRef>(g.tiles), g.nTiles, s));
}

}  // namespace amls_b200
