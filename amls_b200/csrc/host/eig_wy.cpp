// Blocked back-transform of tridiagonal eigenvectors for the matrices above
// the one-CTA size (n > kTridiagSmallMax).
//
// After the Householder tridiagonalisation A holds v_k (v_k[0] = 1 at row
// k + 1) below the subdiagonal of column k, and the eigenvectors of A are
// Q y with Q = H_0 H_1 ... H_{n-3}.  Grouping 64 reflectors,
// H_{k0} ... H_{k0+nb-1} = I - V T V^T (compact WY, LAPACK dlarft forward
// columnwise), so, from the last block to the first,
//   W = V^T Y[k0+1:, :]   (split-K GEMM)
//   W <- T W              (GEMM)
//   Y[k0+1:, :] -= V W    (GEMM)
// with every matrix of the call batched into the same launches.  The upper
// triangle of A is zeroed first, so V is read straight from A; the T factors
// come from S = V^T V (one batched split-K GEMM) and a small kernel.  The
// per-reflector shared-memory kernel, with its n sequential steps per CTA,
// remains for the smaller matrices.
#include <algorithm>

#include "host/engine.hpp"

namespace amls_b200 {

namespace {
constexpr int kT = kGemmTile;
constexpr int kWyBlock = 64;
constexpr int kSplitK = 128;
int cdivW(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

GemmDesc gemmW(int64_t M, int64_t N, int64_t K, int flags, const double* A, int64_t lda,
               const double* B, int64_t ldb, double* C, int64_t ldc, double alpha, double beta,
               int kChunk = 0) {
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
    d.kChunk = kChunk;
    return d;
}

void tilesW(std::vector<TileRef>& t, int desc, int64_t M, int64_t N, int64_t K, int kChunk) {
    const int nk = kChunk > 0 ? cdivW(K, kChunk) : 1;
    for (int kc = 0; kc < nk; ++kc)
        for (int j = 0; j < cdivW(N, kT); ++j)
            for (int i = 0; i < cdivW(M, kT); ++i) t.push_back({desc, i * kT, j * kT, kc});
}
}  // namespace

#define LAUNCH(call)                                   \
    do {                                               \
        const int cat_ = profBegin(#call);             \
        cudaCheck((call), #call);                      \
        profEnd(cat_);                                 \
        ++launches_;                                   \
    } while (0)

void Engine::backTransformBig(const std::vector<EigDesc>& descs, const std::vector<int>& kv,
                              cudaStream_t s) {
    std::vector<EigDesc> big;
    std::vector<int> kb;
    for (size_t i = 0; i < descs.size(); ++i)
        if (descs[i].n > kTridiagSmallMax && kv[i] > 0) {
            big.push_back(descs[i]);
            kb.push_back(std::min(kv[i], static_cast<int>(descs[i].kcap)));
        }
    if (big.empty()) return;
    const int G = static_cast<int>(big.size());
    std::vector<int> nblk(static_cast<size_t>(G));
    std::vector<int64_t> blkBase(static_cast<size_t>(G)), wOff(static_cast<size_t>(G));
    int64_t nBlk = 0, wTot = 0;
    int maxBlk = 0;
    for (int g = 0; g < G; ++g) {
        const int64_t nr = big[static_cast<size_t>(g)].n - 2;
        nblk[static_cast<size_t>(g)] = cdivW(nr, kWyBlock);
        blkBase[static_cast<size_t>(g)] = nBlk;
        nBlk += nblk[static_cast<size_t>(g)];
        wOff[static_cast<size_t>(g)] = wTot;
        wTot += static_cast<int64_t>(kWyBlock) * kb[static_cast<size_t>(g)];
        maxBlk = std::max(maxBlk, nblk[static_cast<size_t>(g)]);
    }
    double* S = static_cast<double*>(wyS_.ensure(sizeof(double) * 2 * 4096 * nBlk));
    double* T = S + 4096 * nBlk;
    double* W = static_cast<double*>(wyW_.ensure(sizeof(double) * 2 * wTot));
    double* W2 = W + wTot;

    Blob b;
    // S = V^T V and the T factors of every block
    std::vector<GemmDesc> sd;
    std::vector<TileRef> st;
    std::vector<WyBlock> wb;
    auto blockGeom = [&](int g, int j, int64_t& k0, int& nb, int64_t& m, const double*& V) {
        const EigDesc& D = big[static_cast<size_t>(g)];
        k0 = static_cast<int64_t>(j) * kWyBlock;
        nb = static_cast<int>(std::min<int64_t>(kWyBlock, D.n - 2 - k0));
        m = D.n - k0 - 1;
        V = D.A + (k0 + 1) + k0 * D.lda;
    };
    for (int g = 0; g < G; ++g) {
        const EigDesc& D = big[static_cast<size_t>(g)];
        for (int j = 0; j < nblk[static_cast<size_t>(g)]; ++j) {
            int64_t k0, m;
            int nb;
            const double* V;
            blockGeom(g, j, k0, nb, m, V);
            double* Sg = S + 4096 * (blkBase[static_cast<size_t>(g)] + j);
            double* Tg = T + 4096 * (blkBase[static_cast<size_t>(g)] + j);
            sd.push_back(gemmW(nb, nb, m, kTransA, V, D.lda, V, D.lda, Sg, 64, 1.0, 0.0, kSplitK));
            tilesW(st, static_cast<int>(sd.size()) - 1, nb, nb, m, kSplitK);
            wb.push_back(WyBlock{D.tau + k0, Sg, Tg, nb, 0});
        }
    }
    struct Step {
        size_t aD, aT, bD, bT, cD, cT;
        int na, nbT, nc;
    };
    std::vector<Step> steps(static_cast<size_t>(maxBlk));
    double flops = 0;
    for (int t = 0; t < maxBlk; ++t) {
        std::vector<GemmDesc> ad, bd, cd;
        std::vector<TileRef> at, bt, ct;
        for (int g = 0; g < G; ++g) {
            if (nblk[static_cast<size_t>(g)] <= t) continue;
            const int j = nblk[static_cast<size_t>(g)] - 1 - t;
            const EigDesc& D = big[static_cast<size_t>(g)];
            int64_t k0, m;
            int nb;
            const double* V;
            blockGeom(g, j, k0, nb, m, V);
            const int k = kb[static_cast<size_t>(g)];
            double* Ysub = D.Y + (k0 + 1);
            double* Wg = W + wOff[static_cast<size_t>(g)];
            double* W2g = W2 + wOff[static_cast<size_t>(g)];
            const double* Tg = T + 4096 * (blkBase[static_cast<size_t>(g)] + j);
            ad.push_back(gemmW(nb, k, m, kTransA, V, D.lda, Ysub, D.ldy, Wg, 64, 1.0, 0.0, kSplitK));
            tilesW(at, static_cast<int>(ad.size()) - 1, nb, k, m, kSplitK);
            bd.push_back(gemmW(nb, k, nb, 0, Tg, 64, Wg, 64, W2g, 64, 1.0, 0.0));
            tilesW(bt, static_cast<int>(bd.size()) - 1, nb, k, nb, 0);
            cd.push_back(gemmW(m, k, nb, kAccumulate, V, D.lda, W2g, 64, Ysub, D.ldy, -1.0, 1.0));
            tilesW(ct, static_cast<int>(cd.size()) - 1, m, k, nb, 0);
            flops += 4.0 * m * nb * k + 2.0 * nb * nb * k;
        }
        Step& S_ = steps[static_cast<size_t>(t)];
        S_.aD = b.add(ad); S_.aT = b.add(at); S_.na = static_cast<int>(at.size());
        S_.bD = b.add(bd); S_.bT = b.add(bt); S_.nbT = static_cast<int>(bt.size());
        S_.cD = b.add(cd); S_.cT = b.add(ct); S_.nc = static_cast<int>(ct.size());
    }
    const size_t oBig = b.add(big), oSD = b.add(sd), oST = b.add(st), oWB = b.add(wb);
    b.upload(wyBlob_, s);
    LAUNCH(launchZeroUpper(b.dev<EigDesc>(oBig), G, s));
    cudaCheck(cudaMemsetAsync(S, 0, sizeof(double) * 4096 * nBlk, s), "zero");
    LAUNCH(launchGemmBatched(b.dev<GemmDesc>(oSD), b.dev<TileRef>(oST), static_cast<int>(st.size()), s));
    LAUNCH(launchWyT(b.dev<WyBlock>(oWB), static_cast<int>(wb.size()), s));
    for (const Step& S_ : steps) {
        cudaCheck(cudaMemsetAsync(W, 0, sizeof(double) * wTot, s), "zero");
        LAUNCH(launchGemmBatched(b.dev<GemmDesc>(S_.aD), b.dev<TileRef>(S_.aT), S_.na, s));
        LAUNCH(launchGemmBatched(b.dev<GemmDesc>(S_.bD), b.dev<TileRef>(S_.bT), S_.nbT, s));
        LAUNCH(launchGemmBatched(b.dev<GemmDesc>(S_.cD), b.dev<TileRef>(S_.cT), S_.nc, s));
    }
    // the tables live in wyBlob_ until the stream passes this point
    cudaCheck(cudaStreamSynchronize(s), "back-transform");
    catF_[7] += flops;
}

}  // namespace amls_b200
