// Shift-invert Lanczos (SIL) nodes, host side: which nodes take the
// reference's SIL branch, their device state, the per-solve factorisation of
// K^_ii - sigma M^_ii and the per-pass Lanczos runs with the reference's
// ncv schedule and selection (src/amls/shift_invert_lanczos.hpp:126-203,
// src/amls/eigenpair_solver.hpp:38-82).  Kernels: kernels/sil.cu.
//
// The selected Ritz pairs (lambda_t, x_t), x_t M^-orthonormal, enter the
// engine's local form like dense eigenpairs: Y = L_ii^T X diag(lambda)^-1/2
// (so that L_ii^-T Y = Z_i diag(mu)^-1/2, the scaled local modes), the mode's
// nu = 1/lambda, and, because Ritz vectors are not exact eigenvectors of
// C_i = L_ii^-1 M^_ii L_ii^-T, the product C_i Y = L_ii^-1 (M^ X)
// diag(lambda)^-1/2 for the right projection M-bar_{S,i} Z_i - K_{S,i}
// K^_ii^-1 M^_ii Z_i (subspace_condensation.cpp:204-232), which for dense
// nodes uses C_i Y = Y diag(nu).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "host/engine.hpp"

namespace amls_b200 {

namespace {
int cdivS(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

GemmDesc gemmS(int64_t M, int64_t N, int64_t K, int flags, const double* A, int64_t lda, const double* B,
               int64_t ldb, double* C, int64_t ldc) {
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
    d.alpha = 1.0;
    d.beta = 0.0;
    return d;
}

void tiles64(std::vector<TileRef>& t, int desc, int64_t M, int64_t N) {
    for (int j = 0; j < cdivS(N, kGemmTile); ++j)
        for (int i = 0; i < cdivS(M, kGemmTile); ++i) t.push_back({desc, i * kGemmTile, j * kGemmTile, 0});
}

void tiles32(std::vector<TileRef>& t, int desc, int64_t r, int64_t c) {
    for (int j = 0; j < cdivS(c, 32); ++j)
        for (int i = 0; i < cdivS(r, 32); ++i) t.push_back({desc, i * 32, j * 32, 0});
}
}  // namespace

#define LAUNCH(call)                                   \
    do {                                               \
        const int cat_ = profBegin(#call);             \
        cudaCheck((call), #call);                      \
        profEnd(cat_);                                 \
        ++launches_;                                   \
    } while (0)

void Engine::silAnalyze(const int64_t* kp, const int32_t* kc, const int64_t* mp, const int32_t* mc) {
    const int N = static_cast<int>(nodes_.size());
    silSep_.clear();
    silLeafCand_.clear();
    silMPat_.assign(static_cast<size_t>(N), {});
    sil_.clear();
    silOf_.assign(static_cast<size_t>(N), -1);
    silPlanSet_.clear();
    silPlanned_ = false;
    silSepTotal_ = 0;
    if (opt_.silMode < 0) return;
    std::vector<char> mark;
    for (int i : order_) {
        const Node& nd = nodes_[static_cast<size_t>(i)];
        const int64_t n = nd.n;
        if (n == 0) continue;
        if (nd.level == 0) {
            // leaves: decided per solve from the nonzero values of K_ii (the
            // reference counts the nonzero entries of the dense block,
            // eigenpair_solver.hpp:73-81); the pattern of M_ii for the products
            if (opt_.silMode == 0 && n < 200) continue;
            auto& pat = silMPat_[static_cast<size_t>(i)];
            for (int64_t lr = 0; lr < n; ++lr) {
                const int64_t old = perm_[static_cast<size_t>(nd.off + lr)];
                for (int64_t e = mp[old]; e < mp[old + 1]; ++e) {
                    const int64_t c = inv_[static_cast<size_t>(mc[e])];
                    if (owner_[static_cast<size_t>(c)] == i)
                        pat.push_back(static_cast<int32_t>(lr * n + (c - nd.off)));   // row-major key
                }
            }
            silLeafCand_.push_back(i);
            continue;
        }
        bool use = opt_.silMode > 0;
        if (!use && n >= 200) {
            // separators: K^_ii carries the updates of its descendants, dense
            // over each descendant's coupling rows inside the node; counted
            // from that structure (exact cancellation to zero is not modelled)
            const double lim = 0.15 * static_cast<double>(n) * static_cast<double>(n);
            mark.assign(static_cast<size_t>(n * n), 0);
            int64_t cnt = 0;
            auto put = [&](int64_t r, int64_t c) {
                char& m = mark[static_cast<size_t>(r + c * n)];
                if (!m) {
                    m = 1;
                    ++cnt;
                }
            };
            for (int64_t r = nd.off; r < nd.off + n; ++r) {
                const int64_t old = perm_[static_cast<size_t>(r)];
                for (int64_t e = kp[old]; e < kp[old + 1]; ++e) {
                    const int64_t c = inv_[static_cast<size_t>(kc[e])];
                    if (owner_[static_cast<size_t>(c)] == i) put(r - nd.off, c - nd.off);
                }
            }
            for (int kk = 0; kk < N && static_cast<double>(cnt) < lim; ++kk) {
                const Node& D = nodes_[static_cast<size_t>(kk)];
                if (std::find(D.anc.begin(), D.anc.end(), i) == D.anc.end()) continue;
                auto lo = std::lower_bound(D.S.begin(), D.S.end(), static_cast<int32_t>(nd.off));
                auto hi = std::lower_bound(D.S.begin(), D.S.end(), static_cast<int32_t>(nd.off + n));
                for (auto x = lo; x != hi; ++x)
                    for (auto y = lo; y != hi; ++y) put(*x - nd.off, *y - nd.off);
            }
            use = static_cast<double>(cnt) < lim;
        }
        if (!use) continue;
        silSep_.push_back(i);
        silSepOff_[i] = silSepTotal_;
        silSepTotal_ += n * n;
    }
    if (!silSep_.empty()) silSepK_.ensure(sizeof(double) * static_cast<size_t>(silSepTotal_));
    if (!silLeafCand_.empty()) {
        // count descriptors over the candidate leaves' K front diagonal blocks
        std::vector<SilCountDesc> cd;
        for (size_t q = 0; q < silLeafCand_.size(); ++q) {
            const Node& nd = nodes_[static_cast<size_t>(silLeafCand_[q])];
            cd.push_back(SilCountDesc{nullptr, nd.ld, static_cast<int32_t>(nd.n), 0});
        }
        silCountDescH_ = cd;
        silCount_.ensure(sizeof(unsigned long long) * silLeafCand_.size());
    }
}

void Engine::silBuildStatic() {
    silCopy_.assign(static_cast<size_t>(maxLevel_) + 1, SilLevelCopy());
    // separators: K^_ii copied before the level's in-place Cholesky (inside
    // the elimination graph)
    std::vector<std::vector<SilCopyDesc>> cd(static_cast<size_t>(maxLevel_) + 1);
    std::vector<std::vector<TileRef>> ct(static_cast<size_t>(maxLevel_) + 1);
    for (int i : silSep_) {
        const Node& nd = nodes_[static_cast<size_t>(i)];
        auto& d = cd[static_cast<size_t>(nd.level)];
        tiles32(ct[static_cast<size_t>(nd.level)], static_cast<int>(d.size()), nd.n, nd.n);
        d.push_back(SilCopyDesc{kPool_.as<double>() + nd.frontOff, nd.ld, silSepK_.as<double>() + silSepOff_.at(i),
                                static_cast<int32_t>(nd.n), 0});
    }
    for (int l = 0; l <= maxLevel_; ++l) {
        SilLevelCopy& c = silCopy_[static_cast<size_t>(l)];
        c.desc = sblob_.add(cd[static_cast<size_t>(l)]);
        c.tiles = sblob_.add(ct[static_cast<size_t>(l)]);
        c.nTiles = static_cast<int>(ct[static_cast<size_t>(l)].size());
    }
    for (SilCountDesc& d : silCountDescH_) d.F = nullptr;
    for (size_t q = 0; q < silLeafCand_.size(); ++q)
        silCountDescH_[q].F = kPool_.as<double>() + nodes_[static_cast<size_t>(silLeafCand_[q])].frontOff;
    silCountDesc_ = sblob_.add(silCountDescH_);
}

// the SIL nodes of this solve: the separators picked at analysis and the
// leaves whose K_ii has fewer than 0.15 n^2 nonzero values (silMode 0) or
// every leaf (silMode 1); a new set rebuilds the node plan
void Engine::silChoose(cudaStream_t s) {
    if (opt_.silMode < 0) return;
    std::vector<int> set(silSep_.begin(), silSep_.end());
    if (!silLeafCand_.empty()) {
        const int nc = static_cast<int>(silLeafCand_.size());
        if (opt_.silMode > 0) {
            set.insert(set.end(), silLeafCand_.begin(), silLeafCand_.end());
        } else {
            LAUNCH(launchSilCountNonzero(sblob_.dev<SilCountDesc>(silCountDesc_), nc,
                                         silCount_.as<unsigned long long>(), s));
            std::vector<unsigned long long> cnt(static_cast<size_t>(nc));
            cudaCheck(cudaMemcpyAsync(cnt.data(), silCount_.as<unsigned long long>(), sizeof(unsigned long long) * nc,
                                      cudaMemcpyDeviceToHost, s), "SIL counts");
            cudaCheck(cudaStreamSynchronize(s), "SIL counts");
            for (int q = 0; q < nc; ++q) {
                const double nn = static_cast<double>(nodes_[static_cast<size_t>(silLeafCand_[static_cast<size_t>(q)])].n);
                if (static_cast<double>(cnt[static_cast<size_t>(q)]) < 0.15 * nn * nn)
                    set.push_back(silLeafCand_[static_cast<size_t>(q)]);
            }
        }
    }
    std::sort(set.begin(), set.end(), [&](int x, int y) {
        return nodes_[static_cast<size_t>(x)].off < nodes_[static_cast<size_t>(y)].off;
    });
    if (!silPlanned_ || set != silPlanSet_) silPlan(set);
    // leaves: K_ii = K^_ii straight from the assembled front (before the
    // elimination factors it in place)
    if (silLeafCopyNTiles_ > 0)
        LAUNCH(launchSilSymCopy(silBlob_.dev<SilCopyDesc>(silLeafCopyDesc_), silBlob_.dev<TileRef>(silLeafCopyTiles_),
                                silLeafCopyNTiles_, s));
}

void Engine::silPlan(const std::vector<int>& set) {
    const int N = static_cast<int>(nodes_.size());
    sil_.clear();
    silOf_.assign(static_cast<size_t>(N), -1);
    silMRowH_.clear();
    silMColH_.clear();
    silMOffH_.clear();
    silMatTotal_ = silVecTotal_ = silInvTotal_ = 0;
    silPlanSet_ = set;
    silPlanned_ = true;
    silLeafCopyNTiles_ = silSepCopyNTiles_ = 0;
    silBlob_.clear();
    if (set.empty()) return;
    for (int i : set) {
        const Node& nd = nodes_[static_cast<size_t>(i)];
        const int64_t n = nd.n;
        SilNode sn;
        sn.node = i;
        sn.mat = silMatTotal_;
        sn.vec = silVecTotal_;
        sn.inv = silInvTotal_;
        sn.csr = static_cast<int64_t>(silMRowH_.size());
        sn.ent = static_cast<int64_t>(silMColH_.size());
        silMatTotal_ += n * n;
        silVecTotal_ += 5 * n;
        silInvTotal_ += static_cast<int64_t>(cdivS(n, 64)) * 4096;
        // local CSR of M^_ii, values read from the M front's lower triangle:
        // a leaf's block is the original M_ii (its pattern), a separator's is
        // dense after the updates of its descendants
        const int64_t e0 = static_cast<int64_t>(silMColH_.size());
        auto lowerOff = [&](int64_t r, int64_t c) {
            return r >= c ? nd.frontOff + r + c * nd.ld : nd.frontOff + c + r * nd.ld;
        };
        const auto& pat = silMPat_[static_cast<size_t>(i)];
        size_t q = 0;
        for (int64_t lr = 0; lr < n; ++lr) {
            silMRowH_.push_back(static_cast<int32_t>(static_cast<int64_t>(silMColH_.size()) - e0));
            if (nd.level == 0) {
                for (; q < pat.size() && pat[q] / n == lr; ++q) {
                    const int64_t lc = pat[q] % n;
                    silMColH_.push_back(static_cast<int32_t>(lc));
                    silMOffH_.push_back(lowerOff(lr, lc));
                }
            } else {
                for (int64_t lc = 0; lc < n; ++lc) {
                    silMColH_.push_back(static_cast<int32_t>(lc));
                    silMOffH_.push_back(lowerOff(lr, lc));
                }
            }
        }
        silMRowH_.push_back(static_cast<int32_t>(static_cast<int64_t>(silMColH_.size()) - e0));
        silOf_[static_cast<size_t>(i)] = static_cast<int>(sil_.size());
        sil_.push_back(sn);
    }
    const size_t nS = sil_.size();
    const size_t mat = static_cast<size_t>(std::max<int64_t>(silMatTotal_, 1));
    silA_.ensure(sizeof(double) * mat);
    silL_.ensure(sizeof(double) * mat);
    silLinv_.ensure(sizeof(double) * mat);
    silScratch_.ensure(sizeof(double) * mat);
    silB_.ensure(sizeof(double) * mat);
    silQ_.ensure(sizeof(double) * mat);
    silMQ_.ensure(sizeof(double) * mat);
    silQT_.ensure(sizeof(double) * mat);
    silVec_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(silVecTotal_, 1)));
    silInv_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(silInvTotal_, 1)));
    silState_.ensure(sizeof(int32_t) * 2 * nS);
    silSigma_.ensure(sizeof(double) * nS);
    silThr_.ensure(sizeof(double) * nS);
    silKOut_.ensure(sizeof(int32_t) * nS);
    silMRow_.ensure(sizeof(int32_t) * silMRowH_.size());
    silMCol_.ensure(sizeof(int32_t) * std::max<size_t>(silMColH_.size(), 1));
    silMOff_.ensure(sizeof(int64_t) * std::max<size_t>(silMOffH_.size(), 1));
    cudaCheck(cudaMemcpyAsync(silMRow_.as<int32_t>(), silMRowH_.data(), sizeof(int32_t) * silMRowH_.size(),
                              cudaMemcpyHostToDevice, stream_), "upload");
    cudaCheck(cudaMemcpyAsync(silMCol_.as<int32_t>(), silMColH_.data(), sizeof(int32_t) * silMColH_.size(),
                              cudaMemcpyHostToDevice, stream_), "upload");
    cudaCheck(cudaMemcpyAsync(silMOff_.as<int64_t>(), silMOffH_.data(), sizeof(int64_t) * silMOffH_.size(),
                              cudaMemcpyHostToDevice, stream_), "upload");
    // L^-1 of A is written below the diagonal only
    cudaCheck(cudaMemsetAsync(silLinv_.as<double>(), 0, sizeof(double) * mat, stream_), "zero");

    // node tables
    double* A = silA_.as<double>();
    std::vector<SilCopyDesc> leafCp, sepCp, low;
    std::vector<TileRef> leafT, sepT, lowT;
    std::vector<SilShiftDesc> sh;
    std::vector<CholItem> items;
    std::vector<GemmDesc> bd;
    std::vector<TileRef> bt;
    for (size_t b = 0; b < nS; ++b) {
        const SilNode& sn = sil_[b];
        const Node& nd = nodes_[static_cast<size_t>(sn.node)];
        const int64_t n = nd.n;
        if (nd.level == 0) {
            tiles32(leafT, static_cast<int>(leafCp.size()), n, n);
            leafCp.push_back(SilCopyDesc{kPool_.as<double>() + nd.frontOff, nd.ld, A + sn.mat, static_cast<int32_t>(n), 0});
        } else {
            tiles32(sepT, static_cast<int>(sepCp.size()), n, n);
            sepCp.push_back(SilCopyDesc{silSepK_.as<double>() + silSepOff_.at(sn.node), n, A + sn.mat,
                                        static_cast<int32_t>(n), 0});
        }
        tiles32(lowT, static_cast<int>(low.size()), n, n);
        low.push_back(SilCopyDesc{kPool_.as<double>() + nd.frontOff, nd.ld, silL_.as<double>() + sn.mat,
                                  static_cast<int32_t>(n), 1});
        sh.push_back(SilShiftDesc{A + sn.mat, mPool_.as<double>() + nd.frontOff, nd.ld,
                                  silSigma_.as<double>() + b, static_cast<int32_t>(n), 0});
        items.push_back(CholItem{A + sn.mat, n, n, silInv_.as<double>() + sn.inv, silLinv_.as<double>() + sn.mat,
                                 silScratch_.as<double>() + sn.mat, sn.node});
        // B = L^-T L^-1 (L^-1 zero above its diagonal)
        tiles64(bt, static_cast<int>(bd.size()), n, n);
        bd.push_back(gemmS(n, n, n, kTransA | kTriKFrom, silLinv_.as<double>() + sn.mat, n,
                           silLinv_.as<double>() + sn.mat, n, silB_.as<double>() + sn.mat, n));
    }
    silLeafCopyDesc_ = silBlob_.add(leafCp);
    silLeafCopyTiles_ = silBlob_.add(leafT);
    silLeafCopyNTiles_ = static_cast<int>(leafT.size());
    silSepCopyDesc_ = silBlob_.add(sepCp);
    silSepCopyTiles_ = silBlob_.add(sepT);
    silSepCopyNTiles_ = static_cast<int>(sepT.size());
    silLowerDesc_ = silBlob_.add(low);
    silLowerTiles_ = silBlob_.add(lowT);
    silLowerNTiles_ = static_cast<int>(lowT.size());
    silShiftDesc_ = silBlob_.add(sh);
    silChol_ = buildCholPlan(silBlob_, items);
    silBGemm_ = addBatch(silBlob_, bd, bt);
    silBlob_.upload(silBlobBuf_, stream_);
    cudaCheck(cudaStreamSynchronize(stream_), "SIL plan");
}

void Engine::silPrepare(cudaStream_t s) {
    if (sil_.empty()) return;
    const int nS = static_cast<int>(sil_.size());
    if (silSepCopyNTiles_ > 0)
        LAUNCH(launchSilSymCopy(silBlob_.dev<SilCopyDesc>(silSepCopyDesc_), silBlob_.dev<TileRef>(silSepCopyTiles_),
                                silSepCopyNTiles_, s));
    LAUNCH(launchSilShift(silBlob_.dev<SilShiftDesc>(silShiftDesc_), nS, s));
    LAUNCH(launchSilSymCopy(silBlob_.dev<SilCopyDesc>(silLowerDesc_), silBlob_.dev<TileRef>(silLowerTiles_),
                            silLowerNTiles_, s));
    runCholPlan(silBlob_, silChol_, s);
    LAUNCH(launchGemmBatched(silBlob_.dev<GemmDesc>(silBGemm_.desc), silBlob_.dev<TileRef>(silBGemm_.tiles),
                             silBGemm_.nTiles, s));
    cudaCheck(cudaMemsetAsync(silState_.as<int32_t>(), 0, sizeof(int32_t) * 2 * nS, s), "SIL state");
    checkStatus("shift-invert factorisation");
}

void Engine::silSelect(int mode, const std::vector<int>& wantP, const std::vector<double>& hiP,
                       std::vector<int>& kSel, cudaStream_t s) {
    const int N = static_cast<int>(nodes_.size());
    kSel.assign(static_cast<size_t>(N), -1);
    const int nS = static_cast<int>(sil_.size());
    if (nS == 0) return;
    std::vector<int> target(static_cast<size_t>(nS), 0), ncv(static_cast<size_t>(nS), 0),
        cap(static_cast<size_t>(nS), 0), cnt(static_cast<size_t>(nS), 0);
    std::vector<char> att(static_cast<size_t>(nS), 0), done(static_cast<size_t>(nS), 1);
    std::vector<int> want(static_cast<size_t>(nS));
    std::vector<double> hi(static_cast<size_t>(nS));
    for (int b = 0; b < nS; ++b) {
        const int pc = pencilOf_[static_cast<size_t>(sil_[static_cast<size_t>(b)].node)];
        want[static_cast<size_t>(b)] = wantP[static_cast<size_t>(pc)];
        hi[static_cast<size_t>(b)] = hiP[static_cast<size_t>(pc)];
    }
    for (int b = 0; b < nS; ++b) {
        const int n = static_cast<int>(nodes_[static_cast<size_t>(sil_[static_cast<size_t>(b)].node)].n);
        const int want_ = want[static_cast<size_t>(b)];
        if (mode == 0) {
            // index mode only for k < 4n/5 (eigenpair_solver.hpp:54-57)
            if (want_ < (n * 4) / 5) {
                att[b] = 1;
                done[b] = 0;
                target[b] = std::min(n, std::max(4 * want_ + 16, 48));   // shift_invert_lanczos.hpp:181
            }
        } else {
            att[b] = 1;
            done[b] = 0;
            ncv[b] = std::min(n, 96);                                   // :137-138
            cap[b] = std::min(n, 1536);
            target[b] = ncv[b];
        }
    }
    std::vector<int32_t> st(static_cast<size_t>(2 * nS));
    auto readStates = [&]() {
        cudaCheck(cudaMemcpyAsync(st.data(), silState_.as<int32_t>(), sizeof(int32_t) * 2 * nS,
                                  cudaMemcpyDeviceToHost, s), "SIL state");
        cudaCheck(cudaStreamSynchronize(s), "SIL state");
    };
    auto eigDesc = [&](int b, int m) {
        const SilNode& sn = sil_[static_cast<size_t>(b)];
        double* v = silVec_.as<double>() + sn.vec;
        const int64_t n = nodes_[static_cast<size_t>(sn.node)].n;
        EigDesc e{};
        e.d = v + 3 * n;       // alpha
        e.e = v + 4 * n;       // beta
        e.n = m;
        e.lda = std::max(m, 1);
        e.id = sn.node;
        e.kcap = m;
        e.kOut = silKOut_.as<int32_t>() + b;
        return e;
    };
    readStates();
    for (;;) {
        std::vector<SilDesc> d(static_cast<size_t>(nS));
        int maxSteps = 0;
        for (int b = 0; b < nS; ++b) {
            const SilNode& sn = sil_[static_cast<size_t>(b)];
            const Node& nd = nodes_[static_cast<size_t>(sn.node)];
            const int64_t n = nd.n;
            double* v = silVec_.as<double>() + sn.vec;
            SilDesc& x = d[static_cast<size_t>(b)];
            x.n = static_cast<int32_t>(n);
            x.target = target[static_cast<size_t>(b)];
            x.active = (att[b] && !done[b]) ? 1 : 0;
            x.state = silState_.as<int32_t>() + 2 * b;
            x.B = silB_.as<double>() + sn.mat;
            x.Q = silQ_.as<double>() + sn.mat;
            x.MQ = silMQ_.as<double>() + sn.mat;
            x.QT = silQT_.as<double>() + sn.mat;
            x.w = v;
            x.mw = v + n;
            x.coef = v + 2 * n;
            x.alpha = v + 3 * n;
            x.beta = v + 4 * n;
            x.mRow = silMRow_.as<int32_t>() + sn.csr;
            x.mCol = silMCol_.as<int32_t>() + sn.ent;
            x.mOff = silMOff_.as<int64_t>() + sn.ent;
            x.mBase = mPool_.as<double>();
            if (x.active && st[static_cast<size_t>(2 * b + 1)] == 0 && st[static_cast<size_t>(2 * b)] < x.target)
                maxSteps = std::max(maxSteps, x.target - st[static_cast<size_t>(2 * b)]);
        }
        if (maxSteps > 0) {
            Blob bl;
            const size_t o = bl.add(d);
            bl.upload(silRunBlob_, s);
            LAUNCH(launchSilLanczos(bl.dev<SilDesc>(o), nS, maxSteps, s));
            readStates();
        }
        if (mode == 0) break;
        // Ritz values <= hi per node: nu >= 1 / (hi - sigma)
        std::vector<EigDesc> ed(static_cast<size_t>(nS));
        for (int b = 0; b < nS; ++b) ed[static_cast<size_t>(b)] = eigDesc(b, st[static_cast<size_t>(2 * b)]);
        Blob be;
        const size_t oe = be.add(ed);
        const size_t oh = be.add(hi);
        be.upload(silEigBlob_, s);
        LAUNCH(launchSilThreshold(silSigma_.as<double>(), nS, be.dev<double>(oh), silThr_.as<double>(), s));
        LAUNCH(launchCountAbove(be.dev<EigDesc>(oe), nS, silThr_.as<double>(), s));
        std::vector<int32_t> kc(static_cast<size_t>(nS));
        cudaCheck(cudaMemcpyAsync(kc.data(), silKOut_.as<int32_t>(), sizeof(int32_t) * nS, cudaMemcpyDeviceToHost, s),
                  "SIL counts");
        cudaCheck(cudaStreamSynchronize(s), "SIL counts");
        bool pending = false;
        for (int b = 0; b < nS; ++b) {
            cnt[static_cast<size_t>(b)] = kc[static_cast<size_t>(b)];
            if (!att[b] || done[b]) continue;
            const int m = st[static_cast<size_t>(2 * b)];
            const int c = kc[static_cast<size_t>(b)];
            // :145-150 (the residual test there always passes: the reference's
            // beta[m-1] is never set, so its residual estimate is 0)
            if (c < m && c > 0) done[b] = 1;
            else if (ncv[b] >= cap[b] || m < ncv[b]) done[b] = 1;
            else {
                ncv[b] = std::min(cap[b], ncv[b] * 2);
                target[b] = ncv[b];
                pending = true;
            }
        }
        if (!pending) break;
    }
    // selection: index mode keeps min(k, m) pairs, used when that is k
    // (eigenpair_solver.hpp:58-59); interval mode keeps every Ritz value in
    // (-inf, hi], used when there is one (:42-43)
    silM_.assign(static_cast<size_t>(nS), 0);
    silSOff_.assign(static_cast<size_t>(nS), 0);
    silNuOff_.assign(static_cast<size_t>(nS), 0);
    std::vector<EigDesc> sel;
    int64_t sTot = 0, nuTot = 0, wTot = 0;
    int maxK = 0;
    for (int b = 0; b < nS; ++b) {
        if (!att[b]) continue;
        const int m = st[static_cast<size_t>(2 * b)];
        silM_[static_cast<size_t>(b)] = m;
        int k = 0;
        if (mode == 0) {
            const int w = want[static_cast<size_t>(b)];
            k = (std::min(w, m) == w) ? w : 0;
        }
        else k = cnt[static_cast<size_t>(b)];
        if (k <= 0) continue;
        kSel[static_cast<size_t>(sil_[static_cast<size_t>(b)].node)] = k;
        silSOff_[static_cast<size_t>(b)] = sTot;
        silNuOff_[static_cast<size_t>(b)] = nuTot;
        sTot += static_cast<int64_t>(m) * k;
        nuTot += k;
        wTot += 8 * static_cast<int64_t>(m) * k + 8 * m;
        maxK = std::max(maxK, k);
    }
    if (maxK == 0) return;
    silS_.ensure(sizeof(double) * static_cast<size_t>(sTot));
    silNu_.ensure(sizeof(double) * static_cast<size_t>(nuTot));
    silWork_.ensure(sizeof(double) * static_cast<size_t>(wTot));
    int64_t wo = 0;
    for (int b = 0; b < nS; ++b) {
        const int k = kSel[static_cast<size_t>(sil_[static_cast<size_t>(b)].node)];
        if (!att[b] || k <= 0) continue;
        const int m = silM_[static_cast<size_t>(b)];
        EigDesc e = eigDesc(b, m);
        e.kcap = k;
        e.w = silNu_.as<double>() + silNuOff_[static_cast<size_t>(b)];
        e.Y = silS_.as<double>() + silSOff_[static_cast<size_t>(b)];
        e.ldy = m;
        e.work = silWork_.as<double>() + wo;
        wo += 8 * static_cast<int64_t>(m) * k + 8 * m;
        sel.push_back(e);
    }
    // eigenpairs of T_m: the k largest nu (bisection, inverse iteration)
    Blob bs;
    const size_t os = bs.add(sel);
    bs.upload(silEigBlob_, s);
    LAUNCH(launchBisectWarp(bs.dev<EigDesc>(os), static_cast<int>(sel.size()), 0, maxK, 0.0, maxK, s));
    LAUNCH(launchInverseIter(bs.dev<EigDesc>(os), static_cast<int>(sel.size()), maxK, nullptr, s));
    cudaCheck(cudaStreamSynchronize(s), "SIL Ritz pairs");
}

void Engine::silVectors(const std::vector<int>& kSel, const std::vector<int64_t>& projOff, cudaStream_t s) {
    const int N = static_cast<int>(nodes_.size());
    silCYPtr_.assign(static_cast<size_t>(N), nullptr);
    const int nS = static_cast<int>(sil_.size());
    int64_t tot = 0, kTot = 0;
    for (int b = 0; b < nS; ++b) {
        const int k = kSel[static_cast<size_t>(sil_[static_cast<size_t>(b)].node)];
        if (k <= 0) continue;
        tot += nodes_[static_cast<size_t>(sil_[static_cast<size_t>(b)].node)].n * k;
        kTot += k;
    }
    if (tot == 0) return;
    silX_.ensure(sizeof(double) * static_cast<size_t>(tot));
    silP_.ensure(sizeof(double) * static_cast<size_t>(tot));
    silYt_.ensure(sizeof(double) * static_cast<size_t>(tot));
    silCY_.ensure(sizeof(double) * static_cast<size_t>(tot));
    silRs_.ensure(sizeof(double) * static_cast<size_t>(kTot));
    std::vector<SilRitzDesc> rd;
    std::vector<GemmDesc> g1, g2;
    std::vector<TileRef> t1, t2, tc;
    std::vector<CopyDesc> cp;
    int64_t off = 0, ko = 0;
    for (int b = 0; b < nS; ++b) {
        const SilNode& sn = sil_[static_cast<size_t>(b)];
        const int i = sn.node;
        const int k = kSel[static_cast<size_t>(i)];
        if (k <= 0) continue;
        const Node& nd = nodes_[static_cast<size_t>(i)];
        const int64_t n = nd.n, m = silM_[static_cast<size_t>(b)];
        double* X = silX_.as<double>() + off;
        double* P = silP_.as<double>() + off;
        double* Yt = silYt_.as<double>() + off;
        double* CY = silCY_.as<double>() + off;
        double* rs = silRs_.as<double>() + ko;
        const double* S = silS_.as<double>() + silSOff_[static_cast<size_t>(b)];
        rd.push_back(SilRitzDesc{silKOut_.as<int32_t>() + b, silNu_.as<double>() + silNuOff_[static_cast<size_t>(b)],
                                 silSigma_.as<double>() + b, rs, wPool_.as<double>() + projOff[static_cast<size_t>(i)]});
        // X = Q S, P = (M^ Q) S = M^ X
        tiles64(t1, static_cast<int>(g1.size()), n, k);
        g1.push_back(gemmS(n, k, m, 0, silQ_.as<double>() + sn.mat, n, S, m, X, n));
        tiles64(t1, static_cast<int>(g1.size()), n, k);
        g1.push_back(gemmS(n, k, m, 0, silMQ_.as<double>() + sn.mat, n, S, m, P, n));
        // Y^T = D^-1/2 X^T L_ii,  C Y = L_ii^-1 P D^-1/2
        GemmDesc y = gemmS(k, n, n, kTransA | kTriKFrom | kRowScale, X, n, silL_.as<double>() + sn.mat, n, Yt, k);
        y.rowScale = rs;
        tiles64(t2, static_cast<int>(g2.size()), k, n);
        g2.push_back(y);
        GemmDesc c = gemmS(n, k, n, kTriAUpTo | kColScale, linvPool_.as<double>() + nd.eigOff, n, P, n, CY, n);
        c.colScale = rs;
        tiles64(t2, static_cast<int>(g2.size()), n, k);
        g2.push_back(c);
        tiles32(tc, static_cast<int>(cp.size()), k, n);
        cp.push_back(CopyDesc{Yt, k, yPool_.as<double>() + yOff_[static_cast<size_t>(i)], n,
                              static_cast<int32_t>(k), static_cast<int32_t>(n)});
        silCYPtr_[static_cast<size_t>(i)] = CY;
        off += n * k;
        ko += k;
    }
    Blob bl;
    const size_t oR = bl.add(rd), oG1 = bl.add(g1), oT1 = bl.add(t1), oG2 = bl.add(g2), oT2 = bl.add(t2),
                 oC = bl.add(cp), oTc = bl.add(tc);
    bl.upload(silEigBlob_, s);
    LAUNCH(launchSilRitzScale(bl.dev<SilRitzDesc>(oR), static_cast<int>(rd.size()), s));
    LAUNCH(launchGemmBatched(bl.dev<GemmDesc>(oG1), bl.dev<TileRef>(oT1), static_cast<int>(t1.size()), s));
    LAUNCH(launchGemmBatched(bl.dev<GemmDesc>(oG2), bl.dev<TileRef>(oT2), static_cast<int>(t2.size()), s));
    LAUNCH(launchTransposeBatched(bl.dev<CopyDesc>(oC), bl.dev<TileRef>(oTc), static_cast<int>(tc.size()), s));
    cudaCheck(cudaStreamSynchronize(s), "SIL vectors");
}

}  // namespace amls_b200
