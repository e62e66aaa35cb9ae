// AMLS engine implementation (see engine.hpp for the algorithm map).
#include "host/engine.hpp"

#include <chrono>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <functional>
#include <future>
#include <iterator>
#include <mutex>
#include <thread>
#include <cstdio>
#include <numeric>
#include <stdexcept>

namespace amls_b200 {

namespace {

constexpr int kSmallEig = kTridiagSmallMax;   // tridiagonalise n <= this with one CTA per matrix
constexpr int kT = kGemmTile;      // 64

int cdiv(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// tiles of a GEMM descriptor (M x N)
void gemmTiles(std::vector<TileRef>& t, int desc, int64_t M, int64_t N, int tile = kT) {
    for (int j = 0; j < cdiv(N, tile); ++j)
        for (int i = 0; i < cdiv(M, tile); ++i) t.push_back({desc, i * tile, j * tile, 0});
}

void trsmTiles(std::vector<TileRef>& t, int desc, int64_t rows) {
    for (int i = 0; i < cdiv(rows, kTrsmRows); ++i) t.push_back({desc, i * kTrsmRows, 0, 0});
}

void copyTiles(std::vector<TileRef>& t, int desc, int64_t r, int64_t c) {
    for (int j = 0; j < cdiv(c, 32); ++j)
        for (int i = 0; i < cdiv(r, 32); ++i) t.push_back({desc, i * 32, j * 32, 0});
}

GemmDesc gemm(int64_t M, int64_t N, int64_t K, int flags, const double* A, int64_t lda,
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

using Clock = std::chrono::steady_clock;
double secs(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

}  // namespace

// kernels launched only from here
cudaError_t launchGemmBatched(const GemmDesc*, const TileRef*, int, cudaStream_t);

// Every kernel launch goes through LAUNCH: it counts launches and, when
// kernel profiling is on, brackets the launch with CUDA events on the
// engine stream (category from the launcher's name).
#define LAUNCH(call)                                   \
    do {                                               \
        const int cat_ = profBegin(#call);             \
        cudaCheck((call), #call);                      \
        profEnd(cat_);                                 \
        ++launches_;                                   \
    } while (0)

Engine::Engine(int device) : device_(device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        throw AmlsError(AMLS_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "bad device index");
    cudaCheck(cudaSetDevice(device), "cudaSetDevice");
    cudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device);
    status_.ensure(4 * sizeof(int));
    // the result copy's pinned double buffer; without it copies go direct
    void* pin = nullptr;
    if (cudaHostAlloc(&pin, 2 * kPinChunk, cudaHostAllocDefault) == cudaSuccess &&
        cudaEventCreateWithFlags(&pinEv_[0], cudaEventDisableTiming) == cudaSuccess &&
        cudaEventCreateWithFlags(&pinEv_[1], cudaEventDisableTiming) == cudaSuccess) {
        pinRing_ = static_cast<char*>(pin);
    } else {
        cudaGetLastError();
        if (pin) cudaFreeHost(pin);
    }
}

Engine::~Engine() {
    cudaSetDevice(device_);
    dropGraphs();
    for (cudaEvent_t e : evPool_) cudaEventDestroy(e);
    if (evSolve0_) cudaEventDestroy(evSolve0_);
    if (evSolve1_) cudaEventDestroy(evSolve1_);
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
    for (cudaEvent_t e : pinEv_)
        if (e) cudaEventDestroy(e);
    if (pinRing_) cudaFreeHost(pinRing_);
}

// Device -> pageable host copy of a large result through the pinned double
// buffer: chunk c + 1 is copied by the DMA engine while host threads move
// chunk c into the destination (whose first touch also costs page faults,
// spread over the threads).  Returns when dst holds the data.
void Engine::copyToHost(double* dst, const double* src, size_t count, cudaStream_t s) {
    const size_t bytes = count * sizeof(double);
    if (!pinRing_ || bytes < 2 * kPinChunk) {
        cudaCheck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "copy out");
        cudaCheck(cudaStreamSynchronize(s), "copy out");
        return;
    }
    const size_t nChunks = (bytes + kPinChunk - 1) / kPinChunk;
    char* ring[2] = {pinRing_, pinRing_ + kPinChunk};
    auto issue = [&](size_t c) {
        const size_t off = c * kPinChunk, len = std::min(kPinChunk, bytes - off);
        cudaCheck(cudaMemcpyAsync(ring[c & 1], reinterpret_cast<const char*>(src) + off, len,
                                  cudaMemcpyDeviceToHost, s), "copy out");
        cudaCheck(cudaEventRecord(pinEv_[c & 1], s), "copy out");
    };
    unsigned nt = std::thread::hardware_concurrency();
    nt = std::max(1u, std::min(nt, 4u));
    issue(0);
    for (size_t c = 0; c < nChunks; ++c) {
        // the other buffer held chunk c - 1, already moved out below
        if (c + 1 < nChunks) issue(c + 1);
        cudaCheck(cudaEventSynchronize(pinEv_[c & 1]), "copy out");
        const size_t off = c * kPinChunk, len = std::min(kPinChunk, bytes - off);
        char* d = reinterpret_cast<char*>(dst) + off;
        const char* from = ring[c & 1];
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t)
            th.emplace_back([=] {
                const size_t b = len * t / nt, e = len * (t + 1) / nt;
                std::memcpy(d + b, from + b, e - b);
            });
        std::memcpy(d, from, len / nt);
        for (auto& x : th) x.join();
    }
}

int Engine::profBegin(const char* text) {
    if (!profiling_) return -1;
    static const char* keys[kProfCats] = {"launchChol",   "launchTrsm",        "launchGemm",
                                          "launchFrontUp", "launchTridiag",     "launchBisect",
                                          "launchInverse", "launchBackTransform", ""};
    int cat = kProfCats - 1;
    for (int c = 0; c < kProfCats - 1; ++c)
        if (std::strstr(text, keys[c])) {
            cat = c;
            break;
        }
    if (evUsed_ + 2 > evPool_.size()) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            cudaCheck(cudaEventCreate(&e), "cudaEventCreate");
            evPool_.push_back(e);
        }
    }
    cudaCheck(cudaEventRecord(evPool_[evUsed_], stream_), "cudaEventRecord");
    evCat_.push_back(cat);
    evText_.push_back(text);
    return cat;
}

void Engine::profEnd(int cat) {
    if (cat < 0) return;
    cudaCheck(cudaEventRecord(evPool_[evUsed_ + 1], stream_), "cudaEventRecord");
    evUsed_ += 2;
}

void Engine::profCollect() {
    if (!profiling_ || evUsed_ == 0) return;
    cudaCheck(cudaStreamSynchronize(stream_), "profile");
    for (size_t k = 0; k + 1 < evUsed_; k += 2) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, evPool_[k], evPool_[k + 1]);
        const int c = evCat_[k / 2];
        profMs_[c] += ms;
        profCount_[c] += 1;
        if (opt_.verbosity >= 3)   // per-launch log: launcher name and device time
            std::fprintf(stderr, "[amls_b200] launch %.48s %.4f ms\n", evText_[k / 2], ms);
    }
    evUsed_ = 0;
    evCat_.clear();
    evText_.clear();
}

void Engine::setProfiling(bool on) {
    profiling_ = on;
    for (int c = 0; c < kProfCats; ++c) {
        profMs_[c] = 0;
        profCount_[c] = 0;
    }
    evUsed_ = 0;
    evCat_.clear();
}

void Engine::kernelTimes(double* ms, int64_t* counts) const {
    for (int c = 0; c < kProfCats; ++c) {
        if (ms) ms[c] = profMs_[c];
        if (counts) counts[c] = profCount_[c];
    }
}

double Engine::elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3;
}

// ---------------------------------------------------------------------------
// analysis
// ---------------------------------------------------------------------------
void Engine::analyze(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp,
                     const int32_t* mc, const amls_options& opt) {
    const int64_t off[2] = {0, n};
    analyzeBatch(1, off, kp, kc, mp, mc, opt);
}

// A batch of independent pencils is one block-diagonal pencil whose diagonal
// blocks (pencil b: rows and columns pOff[b] .. pOff[b+1]) are partitioned
// separately, as the reference solves each pencil on its own; the trees form
// a forest, and every level-batched launch below covers the same tree level
// of all pencils at once.
void Engine::analyzeBatch(int P, const int64_t* pOff, const int64_t* kp, const int32_t* kc,
                          const int64_t* mp, const int32_t* mc, const amls_options& opt) {
    const int64_t n = pOff[P];
    cudaCheck(cudaSetDevice(device_), "cudaSetDevice");
    analyzed_ = false;
    tridiagDone_ = false;
    stageLevel_ = 0;
    dropGraphs();              // the tables (and buffers) they replay are rebuilt
    if (n <= 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "empty matrix");
    for (int64_t r = 0; r < n; ++r) {
        if (kp[r + 1] < kp[r] || mp[r + 1] < mp[r])
            throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "CSR row pointers not monotone");
    }
    if (opt.precision != AMLS_PRECISION_FP64 && opt.precision != AMLS_PRECISION_MIXED)
        throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "precision must be AMLS_PRECISION_FP64 or AMLS_PRECISION_MIXED");
    opt_ = opt;
    n_ = n;
    nnzK_ = kp[n];
    nnzM_ = mp[n];

    const Clock::time_point ta0 = Clock::now();
    // forest: the trees of the pencils with global node ids and DOF indices
    struct FNode {
        std::vector<int64_t> idx;
        int64_t parent = -1;
        std::vector<int64_t> children;
    };
    std::vector<FNode> forest;
    std::vector<int64_t> post;
    nPencils_ = P;
    pOff_.assign(pOff, pOff + P + 1);
    // super-rows for the products with M (they depend on M's pattern only):
    // built on a host thread while the partition runs, uploaded below
    struct SuperRows {
        std::vector<SpmmSuper> sup;
        std::vector<int32_t> ucols;
        std::vector<int64_t> dst;
        int64_t valOff = 0;
    };
    std::future<SuperRows> superRows = std::async(std::launch::async, [this, n, mp, mc]() {
        std::vector<SpmmSuper> sup;
        std::vector<int32_t> ucols;
        std::vector<int64_t> dst(static_cast<size_t>(std::max<int64_t>(nnzM_, 1)));
        std::vector<int32_t> uni, tmp, pat;
        std::vector<int32_t> posOf(static_cast<size_t>(n), -1);   // column -> position in the current union
        int64_t valOff = 0;
        auto groupEnd = [&](int64_t r) {
            const int64_t len = mp[r + 1] - mp[r];
            int64_t e = r + 1;
            while (e < n && e - r < kSpmmSuperRows && mp[e + 1] - mp[e] == len && std::equal(mc + mp[r], mc + mp[r + 1], mc + mp[e]))
                ++e;
            return e;
        };
        auto sortedPattern = [&](int64_t r, std::vector<int32_t>& out) {
            out.assign(mc + mp[r], mc + mp[r + 1]);
            if (!std::is_sorted(out.begin(), out.end())) std::sort(out.begin(), out.end());
            out.erase(std::unique(out.begin(), out.end()), out.end());
        };
        int64_t r = 0;
        while (r < n) {
            int64_t e = groupEnd(r);
            sortedPattern(r, uni);
            while (e < n) {
                const int64_t e2 = groupEnd(e);
                if (e2 - r > kSpmmSuperRows) break;
                sortedPattern(e, pat);
                tmp.clear();
                std::set_union(uni.begin(), uni.end(), pat.begin(), pat.end(), std::back_inserter(tmp));
                if (static_cast<double>(tmp.size() - uni.size()) > 0.8 * static_cast<double>(pat.size())) break;
                uni.swap(tmp);
                e = e2;
            }
            SpmmSuper S{};
            S.row0 = r;
            S.pencil = static_cast<int32_t>(std::upper_bound(pOff_.begin(), pOff_.end(), r) - pOff_.begin() - 1);
            S.rows = static_cast<int32_t>(e - r);
            S.colOff = static_cast<int64_t>(ucols.size());
            S.len = static_cast<int32_t>(uni.size());
            S.valOff = valOff;
            // every column of rows r..e is in the union, so posOf is fresh for them
            for (size_t t = 0; t < uni.size(); ++t) posOf[static_cast<size_t>(uni[t])] = static_cast<int32_t>(t);
            for (int64_t d = r; d < e; ++d)
                for (int64_t q = mp[d]; q < mp[d + 1]; ++q) {
                    const int64_t t = posOf[static_cast<size_t>(mc[q])];
                    dst[static_cast<size_t>(q)] = valOff + t * kSpmmSuperRows + (d - r);
                }
            ucols.insert(ucols.end(), uni.begin(), uni.end());
            valOff += static_cast<int64_t>(uni.size()) * kSpmmSuperRows;
            sup.push_back(S);
            r = e;
        }
        SuperRows out;
        out.sup = std::move(sup);
        out.ucols = std::move(ucols);
        out.dst = std::move(dst);
        out.valOff = valOff;
        return out;
    });
    pencilOf_.clear();
    pNodes_.assign(static_cast<size_t>(P), 0);
    perm_.clear();
    for (int b = 0; b < P; ++b) {
        const int64_t o = pOff[b], nb = pOff[b + 1] - pOff[b];
        if (nb <= 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "empty pencil in the batch");
        PartitionResult pr;
        if (P == 1) {
            // the graph of |K| + |M| extracted on the GPU, METIS on the host
            std::vector<int64_t> xadj, adj;
            extractGraphDevice(n, kp, kc, mp, mc, xadj, adj);
            pr = recursiveBisectionGraph(n, std::move(xadj), std::move(adj), opt.nLevels, opt.leafSize, opt.numThreads);
        } else {
            // the pencil's diagonal block with local indices
            std::vector<int64_t> bkp(static_cast<size_t>(nb + 1)), bmp(static_cast<size_t>(nb + 1));
            std::vector<int32_t> bkc(static_cast<size_t>(kp[o + nb] - kp[o])), bmc(static_cast<size_t>(mp[o + nb] - mp[o]));
            for (int pass = 0; pass < 2; ++pass) {
                const int64_t* rp = pass ? mp : kp;
                const int32_t* ci = pass ? mc : kc;
                std::vector<int64_t>& orp = pass ? bmp : bkp;
                std::vector<int32_t>& oci = pass ? bmc : bkc;
                for (int64_t r = 0; r <= nb; ++r) orp[static_cast<size_t>(r)] = rp[o + r] - rp[o];
                for (int64_t e = rp[o]; e < rp[o + nb]; ++e) {
                    const int64_t c = ci[e] - o;
                    if (c < 0 || c >= nb) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "batch pencils are coupled");
                    oci[static_cast<size_t>(e - rp[o])] = static_cast<int32_t>(c);
                }
            }
            // one in-process METIS call at a time (it re-seeds at every call)
            pr = recursiveBisection(nb, bkp.data(), bkc.data(), bmp.data(), bmc.data(), opt.nLevels,
                                    opt.leafSize, 1);
        }
        const int64_t base = static_cast<int64_t>(forest.size());
        for (int64_t id = 0; id < pr.tree.nNodes(); ++id) {
            const TreeNode& t = pr.tree.node(id);
            FNode f;
            f.idx.reserve(t.indices.size());
            for (int64_t v : t.indices) f.idx.push_back(v + (P == 1 ? 0 : o));
            f.parent = t.parent < 0 ? -1 : t.parent + base;
            for (int64_t c : t.children) f.children.push_back(c + base);
            forest.push_back(std::move(f));
            pencilOf_.push_back(b);
        }
        for (int64_t id : pr.tree.postOrder()) {
            post.push_back(id + base);
            for (int64_t v : pr.tree.node(id).indices) perm_.push_back(v + (P == 1 ? 0 : o));
        }
        pNodes_[static_cast<size_t>(b)] = static_cast<int>(pr.tree.nNodes());
    }
    const Clock::time_point ta1 = Clock::now();
    inv_.assign(static_cast<size_t>(n), 0);
    for (int64_t j = 0; j < n; ++j) inv_[static_cast<size_t>(perm_[static_cast<size_t>(j)])] = j;
    const int N = static_cast<int>(forest.size());
    nodes_.assign(static_cast<size_t>(N), Node());
    order_.clear();
    for (int64_t id : post) order_.push_back(static_cast<int>(id));
    int64_t acc = 0;
    for (int i : order_) {
        Node& nd = nodes_[static_cast<size_t>(i)];
        nd.off = acc;
        nd.n = static_cast<int64_t>(forest[static_cast<size_t>(i)].idx.size());
        nd.parent = static_cast<int>(forest[static_cast<size_t>(i)].parent);
        for (int64_t a = nd.parent; a >= 0; a = forest[static_cast<size_t>(a)].parent) nd.anc.push_back(static_cast<int>(a));
        acc += nd.n;
    }
    maxLevel_ = 0;
    for (int i : order_) {
        int l = 0;
        for (int64_t c : forest[static_cast<size_t>(i)].children) l = std::max(l, nodes_[static_cast<size_t>(c)].level + 1);
        nodes_[static_cast<size_t>(i)].level = l;
        maxLevel_ = std::max(maxLevel_, l);
    }
    byLevel_.assign(static_cast<size_t>(maxLevel_) + 1, {});
    for (int i : order_) byLevel_[static_cast<size_t>(nodes_[static_cast<size_t>(i)].level)].push_back(i);
    owner_.assign(static_cast<size_t>(n), -1);
    for (int i = 0; i < N; ++i) {
        Node& nd = nodes_[static_cast<size_t>(i)];
        for (int64_t r = nd.off; r < nd.off + nd.n; ++r) owner_[static_cast<size_t>(r)] = i;
        nd.pathPrefix = 0;
        for (int a : nd.anc) nd.pathPrefix += nodes_[static_cast<size_t>(a)].n;
    }
    // subtree start offsets (post-order: a subtree is contiguous, ending at the node)
    std::vector<int64_t> subStart(static_cast<size_t>(N));
    for (int i : order_) {
        int64_t s = nodes_[static_cast<size_t>(i)].off;
        for (int64_t c : forest[static_cast<size_t>(i)].children) s = std::min(s, subStart[static_cast<size_t>(c)]);
        subStart[static_cast<size_t>(i)] = s;
    }

    // symbolic fill: S_i = ancestor DOFs coupled to node i after elimination.
    // A node's set needs the sets its descendants push up, so the nodes go
    // level by level, those of one level in parallel over host threads; the
    // pushes of a level are appended after it (S is sorted and deduplicated,
    // so the order of the pushed entries does not matter).
    std::vector<std::vector<int32_t>> push(static_cast<size_t>(N));
    std::vector<std::vector<int32_t>> up(static_cast<size_t>(N));     // node i's push to its first ancestor owner
    std::vector<int> upTo(static_cast<size_t>(N), -1);
    auto symbolic = [&](int i, std::vector<char>& isAnc) {
        Node& nd = nodes_[static_cast<size_t>(i)];
        for (int a : nd.anc) isAnc[static_cast<size_t>(a)] = 1;
        std::vector<int32_t> S = std::move(push[static_cast<size_t>(i)]);
        for (int64_t r = nd.off; r < nd.off + nd.n; ++r) {
            const int64_t old = perm_[static_cast<size_t>(r)];
            for (int pass = 0; pass < 2; ++pass) {
                const int64_t* rp = pass ? mp : kp;
                const int32_t* ci = pass ? mc : kc;
                for (int64_t e = rp[old]; e < rp[old + 1]; ++e) {
                    const int64_t c = inv_[static_cast<size_t>(ci[e])];
                    const int o = owner_[static_cast<size_t>(c)];
                    if (o == i) continue;
                    if (c < nd.off) {
                        if (c < subStart[static_cast<size_t>(i)])
                            throw AmlsError(AMLS_ERR_PARTITION, "partition couples disjoint subtrees");
                        continue;  // descendant: held in the descendant's front
                    }
                    if (!isAnc[static_cast<size_t>(o)])
                        throw AmlsError(AMLS_ERR_PARTITION, "partition couples disjoint subtrees");
                    S.push_back(static_cast<int32_t>(c));
                }
            }
        }
        std::sort(S.begin(), S.end());
        S.erase(std::unique(S.begin(), S.end()), S.end());
        if (!S.empty()) {
            const int a0 = owner_[static_cast<size_t>(S[0])];
            const Node& A0 = nodes_[static_cast<size_t>(a0)];
            auto& dst = up[static_cast<size_t>(i)];
            for (int32_t c : S)
                if (c >= A0.off + A0.n) dst.push_back(c);
            upTo[static_cast<size_t>(i)] = a0;
        }
        nd.S = std::move(S);
        for (int a : nd.anc) isAnc[static_cast<size_t>(a)] = 0;
    };
    {
        unsigned nt = std::thread::hardware_concurrency();
        nt = std::max(1u, std::min(nt, 32u));
        for (int l = 0; l <= maxLevel_; ++l) {
            const std::vector<int>& lv = byLevel_[static_cast<size_t>(l)];
            const unsigned tn = std::min<unsigned>(nt, static_cast<unsigned>(lv.size()));
            std::exception_ptr err;
            std::mutex errMu;
            std::atomic<size_t> next{0};
            auto work = [&] {
                std::vector<char> isAnc(static_cast<size_t>(N), 0);
                try {
                    for (size_t q = next++; q < lv.size(); q = next++) symbolic(lv[q], isAnc);
                } catch (...) {
                    std::lock_guard<std::mutex> lk(errMu);
                    if (!err) err = std::current_exception();
                }
            };
            if (tn <= 1) {
                work();
            } else {
                std::vector<std::thread> th;
                for (unsigned t = 0; t < tn; ++t) th.emplace_back(work);
                for (auto& x : th) x.join();
            }
            if (err) std::rethrow_exception(err);
            for (int i : lv)
                if (upTo[static_cast<size_t>(i)] >= 0) {
                    auto& dst = push[static_cast<size_t>(upTo[static_cast<size_t>(i)])];
                    const auto& src = up[static_cast<size_t>(i)];
                    dst.insert(dst.end(), src.begin(), src.end());
                    std::vector<int32_t>().swap(up[static_cast<size_t>(i)]);
                }
        }
    }
    // layout
    frontTotal_ = eigTotal_ = vecTotal_ = invTotal_ = 0;
    for (int i : order_) {
        Node& nd = nodes_[static_cast<size_t>(i)];
        nd.ld = nd.n + static_cast<int64_t>(nd.S.size());
        nd.frontOff = frontTotal_;
        frontTotal_ += nd.ld * nd.n;
        nd.eigOff = eigTotal_;
        eigTotal_ += nd.n * nd.n;
        nd.vecOff = vecTotal_;
        vecTotal_ += nd.n;
        nd.invOff = invTotal_;
        invTotal_ += static_cast<int64_t>(cdiv(nd.n, 64)) * 4096;
    }
    // CSR destinations in the fronts (rows split over host threads)
    std::function<void(const int64_t*, const int32_t*, std::vector<int64_t>&, int64_t, int64_t)> rowsDst;
    auto dstMap = [&](const int64_t* rp, const int32_t* ci, std::vector<int64_t>& out) {
        out.assign(static_cast<size_t>(rp[n]), -1);
        unsigned nt = std::thread::hardware_concurrency();
        nt = std::max(1u, std::min(nt, 64u));
        std::vector<std::thread> th;
        std::exception_ptr err;
        std::mutex errMu;
        for (unsigned t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                try {
                    rowsDst(rp, ci, out, n * t / nt, n * (t + 1) / nt);
                } catch (...) {
                    std::lock_guard<std::mutex> lk(errMu);
                    err = std::current_exception();
                }
            });
        for (auto& x : th) x.join();
        if (err) std::rethrow_exception(err);
    };
    auto rowsDstBody = [&](const int64_t* rp, const int32_t* ci, std::vector<int64_t>& out,
                           int64_t rowBeg, int64_t rowEnd) {
        for (int64_t old = rowBeg; old < rowEnd; ++old) {
            const int64_t r = inv_[static_cast<size_t>(old)];
            for (int64_t e = rp[old]; e < rp[old + 1]; ++e) {
                const int64_t c = inv_[static_cast<size_t>(ci[e])];
                const int a = owner_[static_cast<size_t>(c)];
                const Node& A = nodes_[static_cast<size_t>(a)];
                if (owner_[static_cast<size_t>(r)] == a) {
                    out[static_cast<size_t>(e)] = A.frontOff + (r - A.off) + (c - A.off) * A.ld;
                } else if (r > c) {
                    auto it = std::lower_bound(A.S.begin(), A.S.end(), static_cast<int32_t>(r));
                    if (it == A.S.end() || *it != r)
                        throw AmlsError(AMLS_ERR_NUMERIC, "symbolic fill missed an entry");
                    out[static_cast<size_t>(e)] =
                        A.frontOff + A.n + (it - A.S.begin()) + (c - A.off) * A.ld;
                }
            }
        }
    };
    rowsDst = rowsDstBody;
    const Clock::time_point ta2 = Clock::now();
    dstMap(kp, kc, hostKDst_);
    dstMap(mp, mc, hostMDst_);
    const Clock::time_point ta3 = Clock::now();

    // device: original M pattern (for the M-norms), maps
    mRp_.ensure(sizeof(int64_t) * static_cast<size_t>(n + 1));
    mCi_.ensure(sizeof(int32_t) * static_cast<size_t>(std::max<int64_t>(nnzM_, 1)));
    invDev_.ensure(sizeof(int64_t) * static_cast<size_t>(n));
    permDev_.ensure(sizeof(int64_t) * static_cast<size_t>(n));
    kDst_.ensure(sizeof(int64_t) * static_cast<size_t>(std::max<int64_t>(nnzK_, 1)));
    mDst_.ensure(sizeof(int64_t) * static_cast<size_t>(std::max<int64_t>(nnzM_, 1)));
    // super-rows for the products with M: node groups (consecutive rows with
    // identical column patterns, the DOFs of one mesh node) merged greedily
    // with their successors while the rows fit kSpmmSuperRows and each added
    // group brings at most 80 % new columns; a dense block per super-row over
    // the union pattern, filled from the CSR values at each numeric solve
    // through supDst (CSR entry -> block position)
    {
        SuperRows sr = superRows.get();
        std::vector<SpmmSuper>& sup = sr.sup;
        std::vector<int32_t>& ucols = sr.ucols;
        std::vector<int64_t>& dst = sr.dst;
        const int64_t valOff = sr.valOff;
        nSup_ = static_cast<int64_t>(sup.size());
        supValTotal_ = valOff;
        supDesc_.ensure(sizeof(SpmmSuper) * std::max<size_t>(sup.size(), 1));
        supCols_.ensure(sizeof(int32_t) * std::max<size_t>(ucols.size(), 1));
        supDst_.ensure(sizeof(int64_t) * dst.size());
        supVal_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(valOff, 1)));
        cudaCheck(cudaMemcpyAsync(supDesc_.as<SpmmSuper>(), sup.data(), sizeof(SpmmSuper) * sup.size(),
                                  cudaMemcpyHostToDevice, stream_), "upload");
        cudaCheck(cudaMemcpyAsync(supCols_.as<int32_t>(), ucols.data(), sizeof(int32_t) * ucols.size(),
                                  cudaMemcpyHostToDevice, stream_), "upload");
        cudaCheck(cudaMemcpyAsync(supDst_.as<int64_t>(), dst.data(), sizeof(int64_t) * nnzM_,
                                  cudaMemcpyHostToDevice, stream_), "upload");
        cudaCheck(cudaStreamSynchronize(stream_), "upload");
    }
    cudaCheck(cudaMemcpyAsync(mRp_.as<int64_t>(), mp, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, stream_), "upload");
    cudaCheck(cudaMemcpyAsync(mCi_.as<int32_t>(), mc, sizeof(int32_t) * nnzM_, cudaMemcpyHostToDevice, stream_), "upload");
    cudaCheck(cudaMemcpyAsync(invDev_.as<int64_t>(), inv_.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, stream_), "upload");
    cudaCheck(cudaMemcpyAsync(permDev_.as<int64_t>(), perm_.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, stream_), "upload");
    if (P > 1) {
        // pencil of every permuted DOF (the M-norms of a batch are per pencil)
        std::vector<int32_t> pd(static_cast<size_t>(n));
        for (int i = 0; i < N; ++i)
            for (int64_t r = nodes_[static_cast<size_t>(i)].off; r < nodes_[static_cast<size_t>(i)].off + nodes_[static_cast<size_t>(i)].n; ++r)
                pd[static_cast<size_t>(r)] = pencilOf_[static_cast<size_t>(i)];
        pencilDev_.ensure(sizeof(int32_t) * static_cast<size_t>(n));
        cudaCheck(cudaMemcpyAsync(pencilDev_.as<int32_t>(), pd.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream_),
                  "upload");
        cudaCheck(cudaStreamSynchronize(stream_), "upload");
    }
    cudaCheck(cudaMemcpyAsync(kDst_.as<int64_t>(), hostKDst_.data(), sizeof(int64_t) * nnzK_, cudaMemcpyHostToDevice, stream_), "upload");
    cudaCheck(cudaMemcpyAsync(mDst_.as<int64_t>(), hostMDst_.data(), sizeof(int64_t) * nnzM_, cudaMemcpyHostToDevice, stream_), "upload");
    kVal_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(nnzK_, 1)));
    mVal_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(nnzM_, 1)));
    kPool_.ensure(sizeof(double) * static_cast<size_t>(frontTotal_));
    mPool_.ensure(sizeof(double) * static_cast<size_t>(frontTotal_));
    gPool_.ensure(sizeof(double) * static_cast<size_t>(frontTotal_));
    // L_ii^-1 blocks are written below the diagonal only: the rest stays zero
    linvPool_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(eigTotal_, 1)));
    linvScratch_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(eigTotal_, 1)));
    cudaCheck(cudaMemsetAsync(linvPool_.as<double>(), 0, sizeof(double) * static_cast<size_t>(std::max<int64_t>(eigTotal_, 1)),
                              stream_), "zero");
    eigPool_.ensure(sizeof(double) * static_cast<size_t>(eigTotal_));
    dPool_.ensure(sizeof(double) * static_cast<size_t>(vecTotal_));
    ePool_.ensure(sizeof(double) * static_cast<size_t>(vecTotal_));
    tauPool_.ensure(sizeof(double) * static_cast<size_t>(vecTotal_));
    invPool_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(invTotal_, 1)));
    silAnalyze(kp, kc, mp, mc);
    const Clock::time_point ta4 = Clock::now();
    buildStatic();
    cudaCheck(cudaStreamSynchronize(stream_), "analyze");
    analyzed_ = true;
    if (opt_.verbosity >= 2)
        std::fprintf(stderr,
                     "[amls_b200] analyze: partition %.3f s, symbolic + layout %.3f s, CSR maps %.3f s, "
                     "uploads %.3f s, launch tables %.3f s\n",
                     secs(ta0, ta1), secs(ta1, ta2), secs(ta2, ta3), secs(ta3, ta4), secs(ta4, Clock::now()));
}

// adjacency of |K| + |M| without self loops, neighbour lists sorted (the
// partition's input graph), built on the GPU from the CSR patterns
void Engine::extractGraphDevice(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp,
                                const int32_t* mc, std::vector<int64_t>& xadj, std::vector<int64_t>& adj) {
    cudaStream_t s = stream_;
    DevBuf &dkp = grKp_, &dkc = grKc_, &dmp = grMp_, &dmc = grMc_, &dcnt = grCnt_, &dadj = grAdj_;
    const int64_t nk = kp[n], nm = mp[n];
    dkp.ensure(sizeof(int64_t) * (n + 1));
    dmp.ensure(sizeof(int64_t) * (n + 1));
    dkc.ensure(sizeof(int32_t) * std::max<int64_t>(nk, 1));
    dmc.ensure(sizeof(int32_t) * std::max<int64_t>(nm, 1));
    dcnt.ensure(sizeof(int64_t) * (n + 1));
    cudaCheck(cudaMemcpyAsync(dkp.as<int64_t>(), kp, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s), "graph");
    cudaCheck(cudaMemcpyAsync(dmp.as<int64_t>(), mp, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s), "graph");
    cudaCheck(cudaMemcpyAsync(dkc.as<int32_t>(), kc, sizeof(int32_t) * nk, cudaMemcpyHostToDevice, s), "graph");
    cudaCheck(cudaMemcpyAsync(dmc.as<int32_t>(), mc, sizeof(int32_t) * nm, cudaMemcpyHostToDevice, s), "graph");
    LAUNCH(launchGraphCount(n, dkp.as<int64_t>(), dkc.as<int32_t>(), dmp.as<int64_t>(), dmc.as<int32_t>(),
                            dcnt.as<int64_t>(), s));
    std::vector<int64_t> cnt(static_cast<size_t>(n));
    cudaCheck(cudaMemcpyAsync(cnt.data(), dcnt.as<int64_t>(), sizeof(int64_t) * n, cudaMemcpyDeviceToHost, s), "graph");
    cudaCheck(cudaStreamSynchronize(s), "graph");
    xadj.assign(static_cast<size_t>(n) + 1, 0);
    for (int64_t v = 0; v < n; ++v) xadj[static_cast<size_t>(v) + 1] = xadj[static_cast<size_t>(v)] + cnt[static_cast<size_t>(v)];
    cudaCheck(cudaMemcpyAsync(dcnt.as<int64_t>(), xadj.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s),
              "graph");
    dadj.ensure(sizeof(int64_t) * std::max<int64_t>(xadj.back(), 1));
    LAUNCH(launchGraphFill(n, dkp.as<int64_t>(), dkc.as<int32_t>(), dmp.as<int64_t>(), dmc.as<int32_t>(),
                           dcnt.as<int64_t>(), dadj.as<int64_t>(), s));
    adj.resize(static_cast<size_t>(xadj.back()));
    static_assert(sizeof(int64_t) == sizeof(double), "the copy moves 8-byte words");
    copyToHost(reinterpret_cast<double*>(adj.data()), dadj.as<double>(), adj.size(), s);
}

void Engine::buildStatic() {
    // ---- static int maps: extend-add (pmin, rowBase, rowIdx, colOff), panel rows, S ----
    Blob ints;
    std::vector<int32_t> pmin, rowBase, rowIdxAll, rowS, Sall;
    std::vector<int64_t> colOff;
    std::vector<int64_t> rowIdxStart(nodes_.size(), 0);
    for (int i : order_) {
        Node& nd = nodes_[static_cast<size_t>(i)];
        const int64_t s = static_cast<int64_t>(nd.S.size());
        nd.mapCol = static_cast<int64_t>(pmin.size());
        nd.rowS = static_cast<int64_t>(rowS.size());
        rowIdxStart[static_cast<size_t>(i)] = static_cast<int64_t>(rowIdxAll.size());
        int64_t p = 0;
        while (p < s) {
            const int a = owner_[static_cast<size_t>(nd.S[static_cast<size_t>(p)])];
            const Node& A = nodes_[static_cast<size_t>(a)];
            int64_t p1 = p;
            while (p1 < s && owner_[static_cast<size_t>(nd.S[static_cast<size_t>(p1)])] == a) ++p1;
            const int64_t segOff = static_cast<int64_t>(rowIdxAll.size()) - rowIdxStart[static_cast<size_t>(i)];
            for (int64_t pp = p; pp < s; ++pp) {
                const int32_t d = nd.S[static_cast<size_t>(pp)];
                if (pp < p1) {
                    rowIdxAll.push_back(static_cast<int32_t>(d - A.off));
                } else {
                    auto it = std::lower_bound(A.S.begin(), A.S.end(), d);
                    if (it == A.S.end() || *it != d)
                        throw AmlsError(AMLS_ERR_NUMERIC, "symbolic fill is not closed");
                    rowIdxAll.push_back(static_cast<int32_t>(A.n + (it - A.S.begin())));
                }
            }
            for (int64_t q = p; q < p1; ++q) {
                pmin.push_back(static_cast<int32_t>(p));
                colOff.push_back(A.frontOff + (nd.S[static_cast<size_t>(q)] - A.off) * A.ld);
                rowBase.push_back(static_cast<int32_t>(segOff - p));
            }
            p = p1;
        }
        for (int64_t q = 0; q < s; ++q) {
            const int32_t d = nd.S[static_cast<size_t>(q)];
            const Node& A = nodes_[static_cast<size_t>(owner_[static_cast<size_t>(d)])];
            rowS.push_back(static_cast<int32_t>(A.pathPrefix + (d - A.off)));
            Sall.push_back(d);
        }
    }
    const size_t oPmin = ints.add(pmin), oRowBase = ints.add(rowBase), oRowIdx = ints.add(rowIdxAll),
                 oRowS = ints.add(rowS), oS = ints.add(Sall), oColOff = ints.add(colOff);
    ints.upload(staticInts_, stream_);
    const int32_t* dPmin = ints.dev<int32_t>(oPmin);
    const int32_t* dRowBase = ints.dev<int32_t>(oRowBase);
    const int32_t* dRowIdx = ints.dev<int32_t>(oRowIdx);
    const int64_t* dColOff = ints.dev<int64_t>(oColOff);
    sIdxDev_ = ints.dev<int32_t>(oS);
    rowSDev_ = ints.dev<int32_t>(oRowS);

    // ---- level tables ----
    sblob_.clear();
    levelPlans_.assign(static_cast<size_t>(maxLevel_) + 1, LevelPlan());
    double* kP = kPool_.as<double>();
    double* mP = mPool_.as<double>();
    double* gP = gPool_.as<double>();
    double* eP = eigPool_.as<double>();
    double* liP = linvPool_.as<double>();
    double* lsP = linvScratch_.as<double>();
    for (int l = 0; l <= maxLevel_; ++l) {
        LevelPlan& L = levelPlans_[static_cast<size_t>(l)];
        std::vector<FrontDesc> fsym;
        std::vector<CholItem> ci;
        std::vector<TileRef> rt, ut, symT, wT, cT;
        std::vector<GemmDesc> rg, wg, cg;
        std::vector<FrontUpdDesc> ud;
        int64_t maxN = 0, maxRows = 0;
        for (int i : byLevel_[static_cast<size_t>(l)]) {
            const Node& nd = nodes_[static_cast<size_t>(i)];
            const int64_t s = static_cast<int64_t>(nd.S.size());
            FrontDesc fe{};
            fe.F = eP + nd.eigOff;
            fe.ld = nd.n;
            fe.n = fe.rows = static_cast<int32_t>(nd.n);
            fe.node = i;
            for (int bj = 0; bj < cdiv(nd.n, 32); ++bj)
                for (int bi = bj; bi < cdiv(nd.n, 32); ++bi)
                    symT.push_back({static_cast<int32_t>(fsym.size()), bi, bj, 0});
            fsym.push_back(fe);
            maxN = std::max(maxN, nd.n);
            maxRows = std::max(maxRows, nd.ld);
            double* linvP = liP + nd.eigOff;
            ci.push_back(CholItem{kP + nd.frontOff, nd.ld, nd.n, invPool_.as<double>() + nd.invOff, linvP,
                                  lsP + nd.eigOff, i});
            // W = G L^-T over all n + s rows of the M front (G L_ii^-T: the
            // reference's Y solves, K^-1 M columns, in transposed form)
            GemmDesc w = gemm(nd.ld, nd.n, nd.n, kTransB | kTriKUpTo, mP + nd.frontOff, nd.ld, linvP, nd.n,
                              gP + nd.frontOff, nd.ld, 1.0, 0.0);
            gemmTiles(wT, static_cast<int>(wg.size()), nd.ld, nd.n, mTile());
            wg.push_back(w);
            // C = L^-1 G_ii^T L^-T = W_ii^T L^-T
            GemmDesc c = gemm(nd.n, nd.n, nd.n, kTransA | kTransB | kTriKUpTo, gP + nd.frontOff, nd.ld, linvP,
                              nd.n, eP + nd.eigOff, nd.n, 1.0, 0.0);
            gemmTiles(cT, static_cast<int>(cg.size()), nd.n, nd.n, mTile());
            cg.push_back(c);
            if (s > 0) {
                // R = Q - L_Si C / 2  (in place in W's lower block)
                GemmDesc g = gemm(s, nd.n, nd.n, kAccumulate, kP + nd.frontOff + nd.n, nd.ld,
                                  eP + nd.eigOff, nd.n, gP + nd.frontOff + nd.n, nd.ld, -0.5, 1.0);
                gemmTiles(rt, static_cast<int>(rg.size()), s, nd.n, mTile());
                rg.push_back(g);
                FrontUpdDesc u{};
                u.s = static_cast<int32_t>(s);
                u.n = static_cast<int32_t>(nd.n);
                u.A = kP + nd.frontOff + nd.n;
                u.B = gP + nd.frontOff + nd.n;
                u.ld = nd.ld;
                u.pmin = dPmin + nd.mapCol;
                u.colOff = dColOff + nd.mapCol;
                u.rowIdx = dRowIdx + rowIdxStart[static_cast<size_t>(i)];
                u.rowBase = dRowBase + nd.mapCol;
                const int ud_i = static_cast<int>(ud.size());
                for (int qt = 0; qt < cdiv(s, kT); ++qt) {
                    int pm = static_cast<int>(s);
                    for (int64_t q = qt * kT; q < std::min<int64_t>(s, (qt + 1) * kT); ++q)
                        pm = std::min(pm, pmin[static_cast<size_t>(nd.mapCol + q)]);
                    for (int pt = pm / kT; pt < cdiv(s, kT); ++pt) ut.push_back({ud_i, pt * kT, qt * kT, 0});
                }
                ud.push_back(u);
            }
        }
        L.chol = buildCholPlan(sblob_, ci);
        L.symDesc = sblob_.add(fsym);
        L.symTiles = sblob_.add(symT);
        L.nSymTiles = static_cast<int>(symT.size());
        L.w = addBatch(sblob_, wg, wT);
        L.c = addBatch(sblob_, cg, cT);
        L.rDesc = sblob_.add(rg);
        L.rTiles = sblob_.add(rt);
        L.nRTiles = static_cast<int>(rt.size());
        L.uDesc = sblob_.add(ud);
        L.uTiles = sblob_.add(ut);
        L.nUTiles = static_cast<int>(ut.size());
    }
    silBuildStatic();
    sblob_.upload(staticBlob_, stream_);

    // ---- ledger: elimination flops/bytes (total and per kernel category) ----
    for (int c = 0; c < kProfCats; ++c) elimCatF_[c] = elimCatB_[c] = 0;
    for (const Node& nd : nodes_) {
        const double nn = static_cast<double>(nd.n), s = static_cast<double>(nd.S.size());
        elimCatF_[0] += nn * nn * nn / 3.0 + s * nn * nn;               // Cholesky
        elimCatB_[0] += 8.0 * 2.0 * (nn + s) * nn;
        elimCatF_[1] += nn * 64.0 * 64.0 / 3.0;                          // 64 x 64 diagonal inverses
        elimCatB_[1] += 8.0 * 2.0 * nn * 64.0;
        // L^-1 (n^3 / 3), W = G L^-T ((n + s) n^2), C = W_ii^T L^-T (n^3), R (2 s n^2)
        elimCatF_[2] += nn * nn * nn / 3.0 + (nn + s) * nn * nn + nn * nn * nn + 2.0 * s * nn * nn;
        elimCatB_[2] += 8.0 * (2.0 * nn * nn + 2.0 * (nn + s) * nn + 3.0 * nn * nn + 2.0 * s * nn + nn * nn + s * nn);
        elimCatF_[3] += 3.0 * s * s * nn;                                // extend-add
        elimCatB_[3] += 8.0 * (2.0 * s * nn + 2.0 * s * s);
        elimCatB_[8] += 8.0 * (2.0 * (nn + s) * nn + 2.0 * nn * nn);     // assembly, transposes
    }
    double fe = 0, be = 0;
    for (const Node& nd : nodes_) {
        const double nn = static_cast<double>(nd.n), s = static_cast<double>(nd.S.size());
        fe += nn * nn * nn / 3.0 + s * nn * nn;          // partial Cholesky
        fe += nn * nn * nn / 3.0;                        // L_ii^-1
        fe += (nn + s) * nn * nn;                        // W = G L^-T
        fe += nn * nn * nn;                              // C = W_ii^T L^-T
        fe += 2.0 * s * nn * nn;                         // R
        fe += 3.0 * s * s * nn;                          // UK (s^2 n) + UM (2 s^2 n), lower half x2
        be += 8.0 * (2.0 * (nn + s) * nn + nn * nn) * 2.0 + 8.0 * s * s;   // fronts r/w + updates
    }
    work_[0] = fe;
    work_[1] = be;
}

// ---------------------------------------------------------------------------
// elimination
// ---------------------------------------------------------------------------
// The elimination is a fixed launch schedule over tables built by analyze:
// captured once into a CUDA graph and replayed by every later numeric solve
// (the per-launch event instrumentation, when on, runs it eagerly).
void Engine::eliminate(cudaStream_t s) {
    // The first numeric solve of an analysis launches eagerly (a one-shot
    // solve, such as amls_solve, gains nothing from capturing); the second
    // captures the fixed schedule into a graph that later solves replay.
    if (profiling_ || (!elimExec_ && elimEagerRuns_ == 0)) {
        eliminateLaunches(s);
        ++elimEagerRuns_;
        return;
    }
    if (!elimExec_) {
        cudaGraph_t g = nullptr;
        cudaCheck(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "capture elimination");
        const int64_t l0 = launches_;
        try {
            eliminateLaunches(s);
        } catch (...) {
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        cudaCheck(cudaStreamEndCapture(s, &g), "capture elimination");
        elimLaunches_ = launches_ - l0;
        launches_ = l0;
        const cudaError_t e = cudaGraphInstantiate(&elimExec_, g, 0);
        cudaGraphDestroy(g);
        cudaCheck(e, "instantiate elimination graph");
    }
    cudaCheck(cudaGraphLaunch(elimExec_, s), "launch elimination graph");
    launches_ += elimLaunches_;
}

void Engine::dropGraphs() {
    if (elimExec_) cudaGraphExecDestroy(elimExec_);
    elimExec_ = nullptr;
    elimLaunches_ = 0;
    elimEagerRuns_ = 0;
    for (auto& kv : applyGraphs_) cudaGraphExecDestroy(kv.second.first);
    applyGraphs_.clear();
    refineEagerRuns_ = 0;
}

void Engine::eliminateLaunches(cudaStream_t s) {
    for (int l = 0; l <= maxLevel_; ++l) {
        const LevelPlan& L = levelPlans_[static_cast<size_t>(l)];
        const SilLevelCopy& sc = silCopy_[static_cast<size_t>(l)];
        if (sc.nTiles > 0)       // K^_ii of the level's shift-invert nodes, before it is factored in place
            LAUNCH(launchSilSymCopy(sblob_.dev<SilCopyDesc>(sc.desc), sblob_.dev<TileRef>(sc.tiles), sc.nTiles, s));
        runCholPlan(sblob_, L.chol, s);
        LAUNCH(launchGemmM(sblob_.dev<GemmDesc>(L.w.desc), sblob_.dev<TileRef>(L.w.tiles), L.w.nTiles, s));
        LAUNCH(launchGemmM(sblob_.dev<GemmDesc>(L.c.desc), sblob_.dev<TileRef>(L.c.tiles), L.c.nTiles, s));
        LAUNCH(launchSymmetrizeTiles(sblob_.dev<FrontDesc>(L.symDesc), sblob_.dev<TileRef>(L.symTiles),
                                     L.nSymTiles, s));
        LAUNCH(launchGemmM(sblob_.dev<GemmDesc>(L.rDesc), sblob_.dev<TileRef>(L.rTiles),
                                 L.nRTiles, s));
        LAUNCH(launchFrontUpdate(sblob_.dev<FrontUpdDesc>(L.uDesc), sblob_.dev<TileRef>(L.uTiles),
                                 L.nUTiles, kPool_.as<double>(), mPool_.as<double>(), s));
    }
}

// the M-side products of the AMLS approximation: FP64 DMMA or, with
// AMLS_PRECISION_MIXED, the split-BF16 tcgen05 kernel (tables built with
// mTile()-sized tiles)
cudaError_t Engine::launchGemmM(const GemmDesc* d, const TileRef* t, int n, cudaStream_t s) {
    return mixed() ? launchGemmBatchedMixed(d, t, n, status_.as<int>(), s) : launchGemmBatched(d, t, n, s);
}

void Engine::checkStatus(const char* phase) {
    int h[2] = {0, 0};
    cudaCheck(cudaMemcpyAsync(h, status_.as<int>(), sizeof(h), cudaMemcpyDeviceToHost, stream_), "status");
    cudaCheck(cudaStreamSynchronize(stream_), phase);
    if (h[0] == kDevNotSpd)
        throw AmlsError(AMLS_ERR_NOT_SPD, std::string(phase) + ": non-positive pivot at tree node " +
                                              std::to_string(h[1]) +
                                              " (input outside the SPD range; shift K)");
    if (h[0] == kDevIterCap)
        throw AmlsError(AMLS_ERR_ITERATION, std::string(phase) + ": iteration cap at " + std::to_string(h[1]));
    if (h[0] == kDevTimeout)
        throw AmlsError(AMLS_ERR_TIMEOUT, std::string(phase) + ": tensor-core wait timed out in tile " +
                                              std::to_string(h[1]));
}

// ---------------------------------------------------------------------------
// eigen driver
// ---------------------------------------------------------------------------
// Cooperative tridiagonalisation of the matrices in `large`.  A launch runs
// as many column steps as its largest matrix has, each ending in a grid
// barrier, so the matrices go largest first into launches of similar
// orders: a launch takes the next matrices down to 0.4 x its largest order
// (at most tridiagLargeMaxCtas(maxN), one CTA per SM), each matrix given CTAs
// in proportion to n^2 (measured faster than n^3 on the benchmark tree).  The
// stream is synchronised before returning (the launch tables live in `blob`).
void Engine::tridiagLargeAll(const std::vector<EigDesc>& largeIn, DevBuf& pbuf, DevBuf& blob,
                             cudaStream_t s) {
    std::vector<EigDesc> large(largeIn);
    std::stable_sort(large.begin(), large.end(), [](const EigDesc& a, const EigDesc& b) { return a.n > b.n; });
    size_t g0 = 0;
    while (g0 < large.size()) {
        const int maxN = large[g0].n;
        const int maxCta = tridiagLargeMaxCtas(maxN);
        if (maxCta < 1) throw AmlsError(AMLS_ERR_CUDA, "cooperative tridiagonalisation does not fit");
        size_t g1 = g0 + 1;
        while (g1 < large.size() && g1 - g0 < static_cast<size_t>(maxCta) &&
               10 * static_cast<int64_t>(large[g1].n) >= 4 * static_cast<int64_t>(maxN))
            ++g1;
        const int cnt = static_cast<int>(g1 - g0);
        std::vector<EigDesc> part(large.begin() + static_cast<std::ptrdiff_t>(g0),
                                  large.begin() + static_cast<std::ptrdiff_t>(g1));
        std::vector<int> groupOf, groupFirst, groupSize;
        std::vector<int64_t> pOff;
        int64_t pTot = 0;
        double wsum = 0;
        for (auto& e : part) wsum += static_cast<double>(e.n) * e.n;
        std::vector<int> cta(static_cast<size_t>(cnt));
        int used = 0, big = 0;
        for (int g = 0; g < cnt; ++g) {
            const double share = static_cast<double>(part[static_cast<size_t>(g)].n) * part[static_cast<size_t>(g)].n / wsum;
            int c = std::max(1, static_cast<int>(std::floor(maxCta * share)));
            c = std::max(1, std::min(c, maxCta - used - (cnt - g - 1)));
            cta[static_cast<size_t>(g)] = c;
            used += c;
            if (part[static_cast<size_t>(g)].n > part[static_cast<size_t>(big)].n) big = g;
        }
        // the CTAs the rounding leaves over go to the largest matrix, whose
        // column steps set the length of the launch
        cta[static_cast<size_t>(big)] += maxCta - used;
        used = 0;
        for (int g = 0; g < cnt; ++g) {
            const int c = cta[static_cast<size_t>(g)];
            groupFirst.push_back(used);
            groupSize.push_back(c);
            for (int q = 0; q < c; ++q) groupOf.push_back(g);
            used += c;
            pOff.push_back(pTot);
            pTot += part[static_cast<size_t>(g)].n;
        }
        Blob b;
        const size_t oL = b.add(part), oGo = b.add(groupOf), oGf = b.add(groupFirst),
                     oGs = b.add(groupSize), oPo = b.add(pOff);
        b.upload(blob, s);
        pbuf.ensure(sizeof(double) * static_cast<size_t>(kTridiagPBufs * pTot + 1));
        LAUNCH(launchTridiagLargeGroups(b.dev<EigDesc>(oL), b.dev<int>(oGo), b.dev<int>(oGf),
                                        b.dev<int>(oGs), used, pbuf.as<double>(), b.dev<int64_t>(oPo),
                                        maxN, s));
        cudaCheck(cudaStreamSynchronize(s), "tridiagonalise");
        g0 = g1;
    }
}

void Engine::tridiagonalizeAll(cudaStream_t s) {
    std::vector<EigDesc> small, large;
    int maxLargeN = 0;
    for (int i : order_) {
        const Node& nd = nodes_[static_cast<size_t>(i)];
        if (nd.n == 0) continue;
        EigDesc e{};
        e.A = eigPool_.as<double>() + nd.eigOff;
        e.lda = nd.n;
        e.d = dPool_.as<double>() + nd.vecOff;
        e.e = ePool_.as<double>() + nd.vecOff;
        e.tau = tauPool_.as<double>() + nd.vecOff;
        e.n = static_cast<int32_t>(nd.n);
        e.id = i;
        if (nd.n <= kSmallEig) small.push_back(e);
        else {
            large.push_back(e);
            maxLargeN = std::max<int>(maxLargeN, static_cast<int>(nd.n));
        }
    }
    // one CTA per matrix, more matrices than CTA slots: the largest first, so
    // the last wave holds the short ones
    std::stable_sort(small.begin(), small.end(), [](const EigDesc& x, const EigDesc& y) { return x.n > y.n; });
    Blob b;
    const size_t oS = b.add(small);
    b.upload(tlBlob_, s);
    for (const auto& e : small) {
        catF_[4] += 4.0 / 3.0 * e.n * static_cast<double>(e.n) * e.n;
        catB_[4] += 8.0 / 3.0 * e.n * static_cast<double>(e.n) * e.n;
    }
    for (const auto& e : large) {
        catF_[4] += 4.0 / 3.0 * e.n * static_cast<double>(e.n) * e.n;
        catB_[4] += 8.0 / 3.0 * e.n * static_cast<double>(e.n) * e.n;
    }
    (void)maxLargeN;
    if (!small.empty()) LAUNCH(launchTridiagSmall(b.dev<EigDesc>(oS), static_cast<int>(small.size()), s));
    tridiagLargeAll(large, redP_, tlLargeBlob_, s);
    // keep the blob alive until the work is done
    cudaCheck(cudaStreamSynchronize(s), "tridiagonalise");
    tridiagDone_ = true;
}

// modes: 0 = index (the `want` largest nu), 1 = interval (nu >= thr)
void Engine::condense(int mode, const std::vector<int>& wantP, const std::vector<double>& thrP,
                      const std::vector<double>& hiP, Pass& P, cudaStream_t s) {
    const int N = static_cast<int>(nodes_.size());
    const int Pn = nPencils_;
    int want = 0;
    for (int b = 0; b < Pn; ++b) want = std::max(want, wantP[static_cast<size_t>(b)]);
    if (!tridiagDone_) tridiagonalizeAll(s);
    // ---- counts ----
    P.k.assign(static_cast<size_t>(N), 0);
    kOutDev_.ensure(sizeof(int32_t) * static_cast<size_t>(N));
    std::vector<EigDesc> descs(static_cast<size_t>(N));
    for (int i = 0; i < N; ++i) {
        const Node& nd = nodes_[static_cast<size_t>(i)];
        EigDesc e{};
        e.A = eigPool_.as<double>() + nd.eigOff;
        e.lda = std::max<int64_t>(nd.n, 1);
        e.d = dPool_.as<double>() + nd.vecOff;
        e.e = ePool_.as<double>() + nd.vecOff;
        e.tau = tauPool_.as<double>() + nd.vecOff;
        e.n = static_cast<int32_t>(nd.n);
        e.id = i;
        e.kOut = kOutDev_.as<int32_t>() + i;
        e.kcap = (mode == 0) ? static_cast<int32_t>(std::min<int64_t>(wantP[static_cast<size_t>(pencilOf_[static_cast<size_t>(i)])], nd.n))
                             : static_cast<int32_t>(nd.n);
        descs[static_cast<size_t>(i)] = e;
    }
    // per-node thresholds of the interval mode (the pencil's 1 / lambda_cut)
    std::vector<double> thrNode(static_cast<size_t>(N), 0.0);
    for (int i = 0; i < N; ++i) thrNode[static_cast<size_t>(i)] = thrP[static_cast<size_t>(pencilOf_[static_cast<size_t>(i)])];
    // shift-invert Lanczos nodes first (the reference's SIL branch); a node it
    // serves takes no part in the dense eigensolves below
    std::vector<int> kSil;
    silSelect(mode, wantP, hiP, kSil, s);
    for (int i = 0; i < N; ++i)
        if (kSil[static_cast<size_t>(i)] > 0) descs[static_cast<size_t>(i)].kcap = 0;
    {
        Blob b;
        const size_t o = b.add(descs);
        const size_t oThr = b.add(thrNode);
        b.upload(passBlob_, s);
        LAUNCH(launchBisect(b.dev<EigDesc>(o), N, mode == 0 ? 0 : 1, 1 << 30, 0.0, 0, nullptr, s,
                            b.dev<double>(oThr)));
        std::vector<int32_t> kh(static_cast<size_t>(N));
        cudaCheck(cudaMemcpyAsync(kh.data(), kOutDev_.as<int32_t>(), sizeof(int32_t) * N, cudaMemcpyDeviceToHost, s), "k");
        cudaCheck(cudaStreamSynchronize(s), "counts");
        for (int i = 0; i < N; ++i)
            P.k[static_cast<size_t>(i)] = kSil[static_cast<size_t>(i)] > 0 ? kSil[static_cast<size_t>(i)]
                                                                         : kh[static_cast<size_t>(i)];
    }
    // ---- offsets, buffers ----
    P.projOff.assign(static_cast<size_t>(N), 0);
    P.localOff.assign(static_cast<size_t>(N), 0);
    P.pp.assign(static_cast<size_t>(Pn), 0);
    int64_t p = 0, ysz = 0, wsz = 0;
    yOff_.assign(static_cast<size_t>(N), 0);
    int maxK = 0;
    for (int i = 0; i < N; ++i) {
        P.projOff[static_cast<size_t>(i)] = p;     // by node id, as the reference's finalize
        int64_t& pb = P.pp[static_cast<size_t>(pencilOf_[static_cast<size_t>(i)])];
        P.localOff[static_cast<size_t>(i)] = pb;   // inside the node's own pencil
        pb += P.k[static_cast<size_t>(i)];
        p += P.k[static_cast<size_t>(i)];
        yOff_[static_cast<size_t>(i)] = ysz;
        ysz += nodes_[static_cast<size_t>(i)].n * P.k[static_cast<size_t>(i)];
        wsz += 6 * nodes_[static_cast<size_t>(i)].n * P.k[static_cast<size_t>(i)];
        maxK = std::max(maxK, P.k[static_cast<size_t>(i)]);
    }
    P.p = p;
    P.credOff.assign(static_cast<size_t>(Pn), 0);
    P.credTotal = 0;
    for (int b = 0; b < Pn; ++b) {
        const int64_t pb = P.pp[static_cast<size_t>(b)];
        if (pb <= 0) throw AmlsError(AMLS_ERR_NUMERIC, "reduced problem is empty (all nodes truncated)");
        P.credOff[static_cast<size_t>(b)] = P.credTotal;
        P.credTotal += pb * pb;
    }
    yPool_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(ysz, 1)));
    wPool_.ensure(sizeof(double) * static_cast<size_t>(p));
    iiWork_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(wsz, 1)));
    int64_t workOff = 0;
    for (int i = 0; i < N; ++i) {
        EigDesc& e = descs[static_cast<size_t>(i)];
        e.kcap = kSil[static_cast<size_t>(i)] > 0 ? 0 : P.k[static_cast<size_t>(i)];
        e.w = wPool_.as<double>() + P.projOff[static_cast<size_t>(i)];
        e.Y = yPool_.as<double>() + yOff_[static_cast<size_t>(i)];
        e.ldy = std::max<int64_t>(nodes_[static_cast<size_t>(i)].n, 1);
        e.work = iiWork_.as<double>() + workOff;
        workOff += 6 * nodes_[static_cast<size_t>(i)].n * P.k[static_cast<size_t>(i)];
    }

    // Ritz vectors of the shift-invert nodes in the engine's local form
    silVectors(kSil, P.projOff, s);
    silServed_ = 0;
    for (int i = 0; i < N; ++i) silServed_ += kSil[static_cast<size_t>(i)] > 0 ? 1 : 0;

    // ---- projection tables (all levels) ----
    const double* F = kPool_.as<double>();
    const double* G = gPool_.as<double>();
    // panels
    panelOff_.assign(static_cast<size_t>(N), -1);
    int64_t panelTot = 0;
    for (int i = 0; i < N; ++i) {
        const Node& nd = nodes_[static_cast<size_t>(i)];
        if (!nd.anc.empty() && P.k[static_cast<size_t>(i)] > 0) {
            panelOff_[static_cast<size_t>(i)] = panelTot;
            panelTot += nd.pathPrefix * P.k[static_cast<size_t>(i)];
        }
    }
    panelPool_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(panelTot, 1)));
    credPool_.ensure(sizeof(double) * static_cast<size_t>(P.credTotal));
    double* panel = panelPool_.as<double>();
    double* cred = credPool_.as<double>();
    // descendants with k > 0, in post-order, per node; Wt sizes
    std::vector<int> pos(static_cast<size_t>(N));
    for (size_t t = 0; t < order_.size(); ++t) pos[static_cast<size_t>(order_[t])] = static_cast<int>(t);
    std::vector<std::vector<int>> descK(static_cast<size_t>(N));
    for (int kk = 0; kk < N; ++kk) {
        if (P.k[static_cast<size_t>(kk)] <= 0) continue;
        for (int a : nodes_[static_cast<size_t>(kk)].anc) descK[static_cast<size_t>(a)].push_back(kk);
    }
    std::vector<int64_t> wtOff(static_cast<size_t>(N), 0), Ksum(static_cast<size_t>(N), 0);
    int64_t wtTot = 0;
    for (int i = 0; i < N; ++i) {
        auto& D = descK[static_cast<size_t>(i)];
        std::sort(D.begin(), D.end(), [&](int x, int y) { return pos[static_cast<size_t>(x)] < pos[static_cast<size_t>(y)]; });
        for (int kk : D) Ksum[static_cast<size_t>(i)] += P.k[static_cast<size_t>(kk)];
        wtOff[static_cast<size_t>(i)] = wtTot;
        wtTot += Ksum[static_cast<size_t>(i)] * nodes_[static_cast<size_t>(i)].n;
    }
    wtPool_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(wtTot, 1)));
    double* wt = wtPool_.as<double>();
    const double* Y = yPool_.as<double>();

    Blob b;
    const size_t oDescs = b.add(descs);
    const size_t oThrNode = b.add(thrNode);
    // per-node index arrays for the scatters (own blob, uploaded first so the
    // GEMM descriptors can point into it)
    std::vector<int32_t> descRowIdx, nodeRowIdx;
    std::vector<int64_t> descColOff, nodeColOff, panelColOff, initColOff;
    std::vector<int64_t> oDescRow(static_cast<size_t>(N)), oDescCol(static_cast<size_t>(N)),
        oNodeRow(static_cast<size_t>(N)), oNodeCol(static_cast<size_t>(N)),
        oPanelCol(static_cast<size_t>(N)), oInitCol(static_cast<size_t>(N));
    std::vector<int64_t> diagDst;                  // reduced-matrix diagonal of every mode
    for (int i = 0; i < N; ++i) {
        const int pc = pencilOf_[static_cast<size_t>(i)];
        const int64_t pb = P.pp[static_cast<size_t>(pc)], cb = P.credOff[static_cast<size_t>(pc)];
        for (int a = 0; a < P.k[static_cast<size_t>(i)]; ++a)
            diagDst.push_back(cb + (P.localOff[static_cast<size_t>(i)] + a) * (pb + 1));
        oDescRow[static_cast<size_t>(i)] = static_cast<int64_t>(descRowIdx.size());
        oDescCol[static_cast<size_t>(i)] = static_cast<int64_t>(descColOff.size());
        oPanelCol[static_cast<size_t>(i)] = static_cast<int64_t>(panelColOff.size());
        for (int kk : descK[static_cast<size_t>(i)]) {
            const int64_t pk = P.localOff[static_cast<size_t>(kk)];
            for (int bcol = 0; bcol < P.k[static_cast<size_t>(kk)]; ++bcol) {
                descRowIdx.push_back(static_cast<int32_t>(pk + bcol));
                descColOff.push_back(cb + (pk + bcol) * pb);
                panelColOff.push_back(panelOff_[static_cast<size_t>(kk)] + bcol * nodes_[static_cast<size_t>(kk)].pathPrefix);
            }
        }
        oNodeRow[static_cast<size_t>(i)] = static_cast<int64_t>(nodeRowIdx.size());
        oNodeCol[static_cast<size_t>(i)] = static_cast<int64_t>(nodeColOff.size());
        oInitCol[static_cast<size_t>(i)] = static_cast<int64_t>(initColOff.size());
        const int64_t pi = P.localOff[static_cast<size_t>(i)];
        for (int a = 0; a < P.k[static_cast<size_t>(i)]; ++a) {
            nodeRowIdx.push_back(static_cast<int32_t>(pi + a));
            nodeColOff.push_back(cb + (pi + a) * pb);
            initColOff.push_back(panelOff_[static_cast<size_t>(i)] + a * nodes_[static_cast<size_t>(i)].pathPrefix);
        }
    }
    struct LevelTabs {
        size_t pjD, pjT, g1D, g1T, g2D, g2T, midD, midT, i1D, i1T, i2D, i2T;
        int npjT, ng1T, ng2T, nmidT, ni1T, ni2T;
    };
    std::vector<LevelTabs> tabs(static_cast<size_t>(maxLevel_) + 1);
    Blob idx;
    const size_t xDR = idx.add(descRowIdx), xDC = idx.add(descColOff), xNR = idx.add(nodeRowIdx),
                 xNC = idx.add(nodeColOff), xPC = idx.add(panelColOff), xIC = idx.add(initColOff),
                 xDD = idx.add(diagDst);
    idx.upload(idxBlob_, s);
    const int32_t* dDR = idx.dev<int32_t>(xDR);
    const int64_t* dDC = idx.dev<int64_t>(xDC);
    const int32_t* dNR = idx.dev<int32_t>(xNR);
    const int64_t* dNC = idx.dev<int64_t>(xNC);
    const int64_t* dPC = idx.dev<int64_t>(xPC);
    const int64_t* dIC = idx.dev<int64_t>(xIC);
    const int64_t* dDD = idx.dev<int64_t>(xDD);
    const double* wDev = wPool_.as<double>();

    double fc = 0, bc = 0;
    const double fcEig = 0.0;
    for (int l = 0; l <= maxLevel_; ++l) {
        std::vector<GemmDesc> pj, g1, g2, mid, i1, i2;
        std::vector<TileRef> pjT, g1T, g2T, midT, i1T, i2T;
        for (int i : byLevel_[static_cast<size_t>(l)]) {
            const Node& nd = nodes_[static_cast<size_t>(i)];
            const int64_t ni = nd.n, si = static_cast<int64_t>(nd.S.size());
            const int64_t Ki = Ksum[static_cast<size_t>(i)];
            const int ki = P.k[static_cast<size_t>(i)];
            double* wti = wt + wtOff[static_cast<size_t>(i)];
            const double* Yi = Y + yOff_[static_cast<size_t>(i)];
            if (Ki > 0 && ni > 0) {
                // wt (Ki x ni) = [panel rows of node i, each descendant's
                // columns]^T L_ii^-T: the descendants' M-bar columns solved
                // with K^_ii, in transposed form
                int64_t colPos = 0;
                const double* linvI = linvPool_.as<double>() + nd.eigOff;
                for (int kk : descK[static_cast<size_t>(i)]) {
                    const Node& nk = nodes_[static_cast<size_t>(kk)];
                    const int ck = P.k[static_cast<size_t>(kk)];
                    if (ck > 0) {
                        GemmDesc g = gemm(ck, ni, ni, kTransA | kTransB | kTriKUpTo,
                                          panel + panelOff_[static_cast<size_t>(kk)] + nd.pathPrefix,
                                          nk.pathPrefix, linvI, ni, wti + colPos, Ki, 1.0, 0.0);
                        gemmTiles(pjT, static_cast<int>(pj.size()), ck, ni, mTile());
                        pj.push_back(g);
                    }
                    colPos += ck;
                }
                fc += static_cast<double>(Ki) * ni * ni;
                if (ki > 0) {
                    GemmDesc a = gemm(ki, Ki, ni, kTransA | kTransB | kScatter, Yi, ni, wti, Ki, cred, 0, 1.0, 0.0);
                    a.rowIdx = dNR + oNodeRow[static_cast<size_t>(i)];
                    a.colOff = dDC + oDescCol[static_cast<size_t>(i)];
                    gemmTiles(g1T, static_cast<int>(g1.size()), ki, Ki, mTile());
                    g1.push_back(a);
                    GemmDesc a2 = gemm(Ki, ki, ni, kScatter, wti, Ki, Yi, ni, cred, 0, 1.0, 0.0);
                    a2.rowIdx = dDR + oDescRow[static_cast<size_t>(i)];
                    a2.colOff = dNC + oNodeCol[static_cast<size_t>(i)];
                    gemmTiles(g2T, static_cast<int>(g2.size()), Ki, ki, mTile());
                    g2.push_back(a2);
                    fc += 4.0 * ki * Ki * ni;
                }
                if (si > 0) {
                    GemmDesc m = gemm(si, Ki, ni, kTransB | kScatter | kAccumulate, F + nd.frontOff + ni, nd.ld,
                                      wti, Ki, panel, 0, -1.0, 0.0);
                    m.rowIdx = rowSDev_ + nd.rowS;
                    m.colOff = dPC + oPanelCol[static_cast<size_t>(i)];
                    gemmTiles(midT, static_cast<int>(mid.size()), si, Ki, mTile());
                    mid.push_back(m);
                    fc += 2.0 * si * Ki * ni;
                }
            }
            if (ki > 0 && si > 0 && panelOff_[static_cast<size_t>(i)] >= 0) {
                GemmDesc a = gemm(si, ki, ni, kScatter, G + nd.frontOff + ni, nd.ld, Yi, ni, panel, 0, 1.0, 0.0);
                a.rowIdx = rowSDev_ + nd.rowS;
                a.colOff = dIC + oInitCol[static_cast<size_t>(i)];
                gemmTiles(i1T, static_cast<int>(i1.size()), si, ki, mTile());
                i1.push_back(a);
                // - L_Si C_i Y / 2: C_i Y = Y diag(nu) for exact local
                // eigenvectors; shift-invert Ritz vectors bring C_i Y itself
                const double* cy = silCYPtr_.empty() ? nullptr : silCYPtr_[static_cast<size_t>(i)];
                GemmDesc a2 = cy ? gemm(si, ki, ni, kScatter | kAccumulate, F + nd.frontOff + ni, nd.ld, cy, ni,
                                        panel, 0, -0.5, 0.0)
                                 : gemm(si, ki, ni, kScatter | kAccumulate | kColScale, F + nd.frontOff + ni,
                                        nd.ld, Yi, ni, panel, 0, -0.5, 0.0);
                a2.rowIdx = rowSDev_ + nd.rowS;
                a2.colOff = dIC + oInitCol[static_cast<size_t>(i)];
                if (!cy) a2.colScale = wDev + P.projOff[static_cast<size_t>(i)];
                gemmTiles(i2T, static_cast<int>(i2.size()), si, ki, mTile());
                i2.push_back(a2);
                fc += 4.0 * si * ki * ni;
            }
            bc += 8.0 * (static_cast<double>(Ki) * ni * 3 + si * (Ki + ki) * 2);
        }
        LevelTabs& T = tabs[static_cast<size_t>(l)];
        T.pjD = b.add(pj); T.pjT = b.add(pjT); T.npjT = static_cast<int>(pjT.size());
        T.g1D = b.add(g1); T.g1T = b.add(g1T); T.ng1T = static_cast<int>(g1T.size());
        T.g2D = b.add(g2); T.g2T = b.add(g2T); T.ng2T = static_cast<int>(g2T.size());
        T.midD = b.add(mid); T.midT = b.add(midT); T.nmidT = static_cast<int>(midT.size());
        T.i1D = b.add(i1); T.i1T = b.add(i1T); T.ni1T = static_cast<int>(i1T.size());
        T.i2D = b.add(i2); T.i2T = b.add(i2T); T.ni2T = static_cast<int>(i2T.size());
    }
    b.upload(passBlob_, s);

    // ---- local eigenpairs (largest nu of C_i) ----
    const EigDesc* dd = b.dev<EigDesc>(oDescs);
    int maxNodeN = 1;
    for (const Node& nd : nodes_) maxNodeN = std::max<int>(maxNodeN, static_cast<int>(nd.n));
    LAUNCH(launchBisectWarp(dd, N, mode == 0 ? 0 : 1, 1 << 30, 0.0, maxK, s, b.dev<double>(oThrNode)));
    LAUNCH(launchInverseIter(dd, N, maxK, nullptr, s));
    LAUNCH(launchBackTransformSmem(dd, N, maxK, std::min(maxNodeN, kTridiagSmallMax), s));
    {
        std::vector<int> kv(P.k.begin(), P.k.end());
        for (int i = 0; i < N; ++i)
            if (kSil[static_cast<size_t>(i)] > 0) kv[static_cast<size_t>(i)] = 0;
        backTransformBig(descs, kv, s);
    }

    // ---- projection ----
    LAUNCH(launchZero(panel, panelTot, s));
    LAUNCH(launchZero(cred, P.credTotal, s));
    LAUNCH(launchScatterAdd(wDev, dDD, p, 1.0, cred, s));    // diagonal blocks: diag(nu)
    for (int l = 0; l <= maxLevel_; ++l) {
        const LevelTabs& T = tabs[static_cast<size_t>(l)];
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.pjD), b.dev<TileRef>(T.pjT), T.npjT, s));
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.g1D), b.dev<TileRef>(T.g1T), T.ng1T, s));
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.g2D), b.dev<TileRef>(T.g2T), T.ng2T, s));
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.midD), b.dev<TileRef>(T.midT), T.nmidT, s));
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.i1D), b.dev<TileRef>(T.i1T), T.ni1T, s));
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.i2D), b.dev<TileRef>(T.i2T), T.ni2T, s));
    }
    // ledger (local eig: bisection + inverse iteration + back-transform;
    // tridiagonalisation counted once per solve)
    for (int i = 0; i < N; ++i) {
        const double nn = static_cast<double>(nodes_[static_cast<size_t>(i)].n), kk = P.k[static_cast<size_t>(i)];
        fc += 4.0 * nn * nn * kk;
        catF_[5] += 60.0 * 6.0 * nn * kk;
        catF_[6] += 4.0 * 12.0 * nn * kk;
        catB_[6] += 8.0 * 6.0 * nn * kk;
        catF_[7] += 4.0 * nn * nn * kk;
        catB_[7] += 8.0 * (nn * nn / 2.0 + 2.0 * nn * kk);
    }
    catF_[2] += fc - fcEig;   // projection GEMMs / TRSMs share the GEMM and TRSM pipes
    catB_[2] += bc;
    work_[2] += fc;
    work_[3] += bc;
    cudaCheck(cudaStreamSynchronize(s), "condense");
}

// per pencil the largest wantP[b] eigenvalues nu of its reduced matrix
// Kp^-1/2 Mp Kp^-1/2 (theta = 1/nu ascending) and, with vectors, their
// eigenvectors at redY_ + P.vOff[b] (pp_b x mMax, ld pp_b; columns beyond
// the pencil's count are zero)
void Engine::reducedSolve(Pass& P, const std::vector<int>& wantP, cudaStream_t s, bool vectors) {
    const int Pn = nPencils_;
    std::vector<int> want(static_cast<size_t>(Pn));
    int wMax = 0;
    int64_t pTot = 0, workTot = 0;
    for (int b = 0; b < Pn; ++b) {
        const int64_t pb = P.pp[static_cast<size_t>(b)];
        want[static_cast<size_t>(b)] = static_cast<int>(std::min<int64_t>(wantP[static_cast<size_t>(b)], pb));
        wMax = std::max(wMax, want[static_cast<size_t>(b)]);
        pTot += pb;
        workTot += 6 * pb * want[static_cast<size_t>(b)];
    }
    P.vOff.assign(static_cast<size_t>(Pn), 0);
    int64_t yTot = 0;
    for (int b = 0; b < Pn; ++b) {
        P.vOff[static_cast<size_t>(b)] = yTot;
        yTot += P.pp[static_cast<size_t>(b)] * wMax;
    }
    redD_.ensure(sizeof(double) * static_cast<size_t>(pTot));
    redE_.ensure(sizeof(double) * static_cast<size_t>(pTot));
    redTau_.ensure(sizeof(double) * static_cast<size_t>(pTot));
    redW_.ensure(sizeof(double) * static_cast<size_t>(std::max(1, Pn * wMax)));
    redY_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(yTot, 1)));
    redWork_.ensure(sizeof(double) * static_cast<size_t>(std::max<int64_t>(workTot, 1)));
    redK_.ensure(sizeof(int32_t) * static_cast<size_t>(Pn));
    if (vectors && Pn > 1) LAUNCH(launchZero(redY_.as<double>(), yTot, s));
    std::vector<EigDesc> all, small, large;
    int64_t vo = 0, wo = 0;
    int maxSmallN = 1;
    for (int b = 0; b < Pn; ++b) {
        const int64_t pb = P.pp[static_cast<size_t>(b)];
        EigDesc e{};
        e.A = credPool_.as<double>() + P.credOff[static_cast<size_t>(b)];
        e.lda = pb;
        e.d = redD_.as<double>() + vo;
        e.e = redE_.as<double>() + vo;
        e.tau = redTau_.as<double>() + vo;
        e.n = static_cast<int32_t>(pb);
        e.id = -1 - b;
        e.w = redW_.as<double>() + static_cast<int64_t>(b) * wMax;
        e.Y = redY_.as<double>() + P.vOff[static_cast<size_t>(b)];
        e.ldy = pb;
        e.kcap = want[static_cast<size_t>(b)];
        e.kOut = redK_.as<int32_t>() + b;
        e.work = redWork_.as<double>() + wo;
        vo += pb;
        wo += 6 * pb * want[static_cast<size_t>(b)];
        all.push_back(e);
        if (pb <= kSmallEig) {
            small.push_back(e);
            maxSmallN = std::max<int>(maxSmallN, static_cast<int>(pb));
        } else {
            large.push_back(e);
        }
    }
    Blob b;
    const size_t oA = b.add(all), oS = b.add(small);
    b.upload(redBlob_, s);
    if (!small.empty()) LAUNCH(launchTridiagSmall(b.dev<EigDesc>(oS), static_cast<int>(small.size()), s));
    if (!large.empty()) tridiagLargeAll(large, redP_, tlLargeBlob_, s);
    LAUNCH(launchBisectWarp(b.dev<EigDesc>(oA), Pn, 0, wMax, 0.0, wMax, s));
    if (vectors) {
        LAUNCH(launchInverseIter(b.dev<EigDesc>(oA), Pn, wMax, nullptr, s));
        LAUNCH(launchBackTransformSmem(b.dev<EigDesc>(oA), Pn, wMax, std::min(maxSmallN, kTridiagSmallMax), s));
        if (!large.empty()) {
            std::vector<int> kv;
            for (const EigDesc& e : large) kv.push_back(e.kcap);
            backTransformBig(large, kv, s);
        }
    }
    std::vector<double> nu(static_cast<size_t>(std::max(1, Pn * wMax)));
    std::vector<int32_t> kk(static_cast<size_t>(Pn));
    cudaCheck(cudaMemcpyAsync(nu.data(), redW_.as<double>(), sizeof(double) * Pn * wMax, cudaMemcpyDeviceToHost, s),
              "theta");
    cudaCheck(cudaMemcpyAsync(kk.data(), redK_.as<int32_t>(), sizeof(int32_t) * Pn, cudaMemcpyDeviceToHost, s), "k");
    cudaCheck(cudaStreamSynchronize(s), "reduced");
    P.theta.assign(static_cast<size_t>(Pn), {});
    P.got.assign(static_cast<size_t>(Pn), 0);
    P.mMax = 0;
    for (int q = 0; q < Pn; ++q) {
        const int g = std::min<int>(kk[static_cast<size_t>(q)], want[static_cast<size_t>(q)]);
        P.got[static_cast<size_t>(q)] = g;
        P.mMax = std::max(P.mMax, g);
        auto& th = P.theta[static_cast<size_t>(q)];
        th.resize(static_cast<size_t>(g));
        for (int j = 0; j < g; ++j) th[static_cast<size_t>(j)] = 1.0 / nu[static_cast<size_t>(q * wMax + j)];
        const double pp = static_cast<double>(P.pp[static_cast<size_t>(q)]);
        catF_[4] += 4.0 / 3.0 * pp * pp * pp;
        catB_[4] += 8.0 / 3.0 * pp * pp * pp;
        catF_[5] += 60.0 * 6.0 * pp * g;
        catF_[6] += 4.0 * 12.0 * pp * g;
        catB_[6] += 8.0 * 6.0 * pp * g;
        catF_[7] += 4.0 * pp * pp * g;
        catB_[7] += 8.0 * (pp * pp / 2.0 + 2.0 * pp * g);
        work_[4] += 4.0 / 3.0 * pp * pp * pp + 4.0 * pp * pp * g;
        work_[5] += 8.0 * pp * pp * pp / 3.0;
    }
}

void Engine::backtransform(const Pass& P, int m, cudaStream_t s) {
    const int N = static_cast<int>(nodes_.size());
    const int Pn = nPencils_;
    ztPool_.ensure(sizeof(double) * static_cast<size_t>(m * n_));
    sqrtTheta_.ensure(sizeof(double) * static_cast<size_t>(m * Pn));
    std::vector<double> st(static_cast<size_t>(m * Pn), 0.0);       // per pencil, zero beyond its count
    for (int q = 0; q < Pn; ++q)
        for (int j = 0; j < std::min<int>(m, P.got[static_cast<size_t>(q)]); ++j)
            st[static_cast<size_t>(q * m + j)] = std::sqrt(P.theta[static_cast<size_t>(q)][static_cast<size_t>(j)]);
    cudaCheck(cudaMemcpyAsync(sqrtTheta_.as<double>(), st.data(), sizeof(double) * m * Pn, cudaMemcpyHostToDevice, s),
              "sqrt theta");
    double* zt = ztPool_.as<double>();
    // u_i = (y v_i D_theta)^T - z_S L_Si, then z_i = u_i L_ii^-1 (transposed
    // layout, m x n_i blocks); u lives in a second buffer of the same layout
    double* ut = static_cast<double*>(zTmp_.ensure(sizeof(double) * static_cast<size_t>(m * n_)));
    const double* F = kPool_.as<double>();
    const double* Y = yPool_.as<double>();
    const double* V = redY_.as<double>();
    Blob b;
    struct Tabs { size_t g1D, g1T, g2D, g2T, tD, tT; int n1, n2, nt; };
    std::vector<Tabs> tabs(static_cast<size_t>(maxLevel_) + 1);
    double fb = 0;
    for (int l = maxLevel_; l >= 0; --l) {
        std::vector<GemmDesc> g1, g2, tr;
        std::vector<TileRef> g1T, g2T, tT;
        for (int i : byLevel_[static_cast<size_t>(l)]) {
            const Node& nd = nodes_[static_cast<size_t>(i)];
            const int64_t ni = nd.n, si = static_cast<int64_t>(nd.S.size());
            const int ki = P.k[static_cast<size_t>(i)];
            if (ni == 0) continue;
            double* zi = zt + nd.off * m;
            double* ui = ut + nd.off * m;
            const int pc = pencilOf_[static_cast<size_t>(i)];
            GemmDesc a = gemm(m, ni, ki, kTransA | kTransB | kRowScale,
                              V + P.vOff[static_cast<size_t>(pc)] + P.localOff[static_cast<size_t>(i)],
                              P.pp[static_cast<size_t>(pc)], Y + yOff_[static_cast<size_t>(i)],
                              std::max<int64_t>(ni, 1), ui, m, 1.0, 0.0);
            a.rowScale = sqrtTheta_.as<double>() + static_cast<int64_t>(pc) * m;
            gemmTiles(g1T, static_cast<int>(g1.size()), m, ni, mTile());
            g1.push_back(a);
            if (si > 0) {
                GemmDesc c = gemm(m, ni, si, kGatherA | kAccumulate, zt, m, F + nd.frontOff + ni, nd.ld, ui, m, -1.0, 1.0);
                c.aMap = sIdxDev_ + nd.mapCol;
                gemmTiles(g2T, static_cast<int>(g2.size()), m, ni, mTile());
                g2.push_back(c);
            }
            GemmDesc t = gemm(m, ni, ni, kTriKFrom, ui, m, linvPool_.as<double>() + nd.eigOff, ni, zi, m, 1.0, 0.0);
            gemmTiles(tT, static_cast<int>(tr.size()), m, ni, mTile());
            tr.push_back(t);
            fb += 2.0 * m * ni * (ki + si) + static_cast<double>(m) * ni * ni;
        }
        Tabs& T = tabs[static_cast<size_t>(l)];
        T.g1D = b.add(g1); T.g1T = b.add(g1T); T.n1 = static_cast<int>(g1T.size());
        T.g2D = b.add(g2); T.g2T = b.add(g2T); T.n2 = static_cast<int>(g2T.size());
        T.tD = b.add(tr); T.tT = b.add(tT); T.nt = static_cast<int>(tT.size());
    }
    (void)N;
    b.upload(passBlob_, s);
    for (int l = maxLevel_; l >= 0; --l) {
        const Tabs& T = tabs[static_cast<size_t>(l)];
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.g1D), b.dev<TileRef>(T.g1T), T.n1, s));
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.g2D), b.dev<TileRef>(T.g2T), T.n2, s));
        LAUNCH(launchGemmM(b.dev<GemmDesc>(T.tD), b.dev<TileRef>(T.tT), T.nt, s));
    }
    catF_[2] += fb;
    catB_[2] += 8.0 * 3.0 * m * static_cast<double>(n_);
    catB_[8] += 8.0 * (12.0 * nnzM_ + 3.0 * m * static_cast<double>(n_));
    work_[6] += fb + 4.0 * static_cast<double>(nnzM_) * m;
    work_[7] += 8.0 * (2.0 * m * n_ * 3 + 12.0 * nnzM_);
    cudaCheck(cudaStreamSynchronize(s), "backtransform");
}

// ---------------------------------------------------------------------------
// numeric solve
// ---------------------------------------------------------------------------
// values in, fronts assembled, shift-invert nodes chosen, elimination
// (replayed graph) and the shift-invert factorisations; returns the time
// after the value upload
Engine::Clock::time_point Engine::numericElimination(const double* kv, const double* mv, bool valuesOnDevice,
                                                     cudaStream_t s) {
    cudaCheck(cudaMemsetAsync(status_.as<int>(), 0, 2 * sizeof(int), s), "status");
    if (valuesOnDevice) {
        cudaCheck(cudaMemcpyAsync(kVal_.as<double>(), kv, sizeof(double) * nnzK_, cudaMemcpyDeviceToDevice, s), "values");
        cudaCheck(cudaMemcpyAsync(mVal_.as<double>(), mv, sizeof(double) * nnzM_, cudaMemcpyDeviceToDevice, s), "values");
    } else {
        cudaCheck(cudaMemcpyAsync(kVal_.as<double>(), kv, sizeof(double) * nnzK_, cudaMemcpyHostToDevice, s), "values");
        cudaCheck(cudaMemcpyAsync(mVal_.as<double>(), mv, sizeof(double) * nnzM_, cudaMemcpyHostToDevice, s), "values");
    }
    cudaCheck(cudaStreamSynchronize(s), "upload");
    const auto t1 = Clock::now();
    // assemble fronts
    LAUNCH(launchZero(kPool_.as<double>(), frontTotal_, s));
    LAUNCH(launchZero(mPool_.as<double>(), frontTotal_, s));
    LAUNCH(launchScatterAdd(kVal_.as<double>(), kDst_.as<int64_t>(), nnzK_, 1.0, kPool_.as<double>(), s));
    if (opt_.shift != 0.0)
        LAUNCH(launchScatterAdd(mVal_.as<double>(), mDst_.as<int64_t>(), nnzM_, opt_.shift, kPool_.as<double>(), s));
    LAUNCH(launchScatterAdd(mVal_.as<double>(), mDst_.as<int64_t>(), nnzM_, 1.0, mPool_.as<double>(), s));
    LAUNCH(launchZero(supVal_.as<double>(), supValTotal_, s));
    LAUNCH(launchScatterAdd(mVal_.as<double>(), supDst_.as<int64_t>(), nnzM_, 1.0, supVal_.as<double>(), s));
    silChoose(s);            // shift-invert nodes of this solve (leaves by their nonzero values)
    eliminate(s);
    checkStatus("elimination");
    silPrepare(s);
    return t1;
}

void Engine::solveValues(const double* kv, const double* mv, bool valuesOnDevice, double* theta,
                         double* Z, bool outputsOnDevice, int64_t* pOut, double* timing, int64_t* mOut) {
    if (!analyzed_) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "amls_solve_values before amls_analyze");
    cudaCheck(cudaSetDevice(device_), "cudaSetDevice");
    if (opt_.nev <= 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "nev must be positive");
    const int64_t nev = std::min<int64_t>(opt_.nev, n_);
    cudaStream_t s = stream_;
    stageLevel_ = 0;
    launches_ = 0;
    for (int t = 2; t < AMLS_WORK_SLOTS; ++t) work_[t] = 0;
    for (int c = 0; c < kProfCats; ++c) {
        catF_[c] = elimCatF_[c];
        catB_[c] = elimCatB_[c];
    }
    tridiagDone_ = false;
    const auto t0 = Clock::now();
    if (!evSolve0_) {
        cudaCheck(cudaEventCreate(&evSolve0_), "cudaEventCreate");
        cudaCheck(cudaEventCreate(&evSolve1_), "cudaEventCreate");
    }
    cudaCheck(cudaEventRecord(evSolve0_, s), "cudaEventRecord");
    const auto t1 = numericElimination(kv, mv, valuesOnDevice, s);
    const auto t2 = Clock::now();
    double tRed = 0;
    Pass P;
    const int Pn = nPencils_;
    std::vector<int> nevP(static_cast<size_t>(Pn));
    for (int q = 0; q < Pn; ++q)
        nevP[static_cast<size_t>(q)] = static_cast<int>(std::min<int64_t>(opt_.nev, pOff_[q + 1] - pOff_[q]));
    const std::vector<double> zeroP(static_cast<size_t>(Pn), 0.0);
    if (opt_.fixedKeep > 0) {
        condense(0, std::vector<int>(static_cast<size_t>(Pn), static_cast<int>(opt_.fixedKeep)), zeroP, zeroP, P, s);
        pA_ = P.p;
    } else {
        if (!opt_.twoPass)
            throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "twoPass=false with fixedKeep=0 cannot set the cut");
        // pass A: k0 = max(4, ceil(3 nev / N)) per pencil (solver.cpp:246-248)
        std::vector<int> k0(static_cast<size_t>(Pn));
        for (int q = 0; q < Pn; ++q) {
            const int64_t Nq = pNodes_[static_cast<size_t>(q)];
            k0[static_cast<size_t>(q)] = static_cast<int>(std::max<int64_t>(4, (3 * nevP[static_cast<size_t>(q)] + Nq - 1) / Nq));
        }
        Pass A;
        condense(0, k0, zeroP, zeroP, A, s);
        pA_ = A.p;
        const auto ta = Clock::now();
        std::vector<int> wA(static_cast<size_t>(Pn));
        for (int q = 0; q < Pn; ++q)
            wA[static_cast<size_t>(q)] = static_cast<int>(std::min<int64_t>(nevP[static_cast<size_t>(q)], A.pp[static_cast<size_t>(q)]));
        reducedSolve(A, wA, s, false);
        tRed += secs(ta, Clock::now());
        // lambda_cut = eta * lambda_hat per pencil (:252-258)
        std::vector<double> thr(static_cast<size_t>(Pn)), hi(static_cast<size_t>(Pn));
        for (int q = 0; q < Pn; ++q) {
            const int nq = nevP[static_cast<size_t>(q)];
            if (A.got[static_cast<size_t>(q)] < nq)
                throw AmlsError(AMLS_ERR_NUMERIC, "pass A reduced problem too small (p < nev); reduce nLevels or grow leafSize");
            const double lambdaHat = A.theta[static_cast<size_t>(q)][static_cast<size_t>(nq - 1)];
            const double lambdaCut = opt_.thresholdFactor * lambdaHat;
            if (opt_.verbosity > 0 && Pn == 1)
                std::fprintf(stderr, "[amls_b200] pass A: p0=%lld lambda_hat=%.10g lambda_cut=%.10g\n",
                             static_cast<long long>(A.p), lambdaHat, lambdaCut);
            // keep mu <= lambda_cut  <=>  nu >= 1 / lambda_cut (all local mu > 0)
            thr[static_cast<size_t>(q)] = lambdaCut > 0 ? 1.0 / lambdaCut : 1e300;
            hi[static_cast<size_t>(q)] = lambdaCut;
        }
        condense(1, std::vector<int>(static_cast<size_t>(Pn), 0), thr, hi, P, s);
    }
    const auto t3 = Clock::now();
    pFinal_ = P.p;
    for (int q = 0; q < Pn; ++q)
        if (P.pp[static_cast<size_t>(q)] > opt_.denseProjectedMax && opt_.verbosity > 0)
            std::fprintf(stderr, "[amls_b200] warning: p=%lld exceeds denseProjectedMax=%lld (dense solve used)\n",
                         static_cast<long long>(P.pp[static_cast<size_t>(q)]),
                         static_cast<long long>(opt_.denseProjectedMax));
    std::vector<int> nq(static_cast<size_t>(Pn));
    for (int q = 0; q < Pn; ++q)
        nq[static_cast<size_t>(q)] = static_cast<int>(std::min<int64_t>(nevP[static_cast<size_t>(q)], P.pp[static_cast<size_t>(q)]));
    if (opt_.refine) {
        if (Pn > 1) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "refinement is available for a single pencil only");
        const int64_t extra = opt_.refineExtra >= 0 ? opt_.refineExtra : nev / 2 + 16;
        nq[0] = static_cast<int>(std::min<int64_t>(P.p, std::min<int64_t>(n_, nev + extra)));
    }
    reducedSolve(P, nq, s);
    std::vector<int> want(static_cast<size_t>(Pn));
    for (int q = 0; q < Pn; ++q)
        want[static_cast<size_t>(q)] = std::min(nevP[static_cast<size_t>(q)], P.got[static_cast<size_t>(q)]);
    const auto t4 = Clock::now();
    tRed += secs(t3, t4);
    const bool recover = opt_.recoverVectors && Z != nullptr;
    refineIters_ = 0;
    refineNq_ = 0;
    int mZ = 0;                        // columns of zOut_
    if (opt_.refine) {
        const int got = P.got[0];
        backtransform(P, got, s);
        refineNq_ = got;
        refineIters_ = refine(ztPool_.as<double>(), got, want[0], P.theta[0], recover, s);
        P.theta[0].resize(static_cast<size_t>(want[0]));
        if (recover) finalizeVectors(ztPool_.as<double>(), got, want[0], s);
        mZ = want[0];
    } else if (recover) {
        mZ = P.mMax;
        backtransform(P, mZ, s);
        finalizeVectors(ztPool_.as<double>(), mZ, mZ, s);
    }
    for (int q = 0; q < Pn; ++q) P.theta[static_cast<size_t>(q)].resize(static_cast<size_t>(want[static_cast<size_t>(q)]));
    const auto t5 = Clock::now();
    // outputs: pencil q's values at theta + q * nev (one pencil: theta[0 ..
    // want)); Z is n x nev column-major, pencil q in its own rows, columns
    // beyond its count zero
    const int64_t zCols = nev;   // every column of the caller's n x nev Z is written
    std::vector<double> th(static_cast<size_t>(Pn == 1 ? std::max(want[0], 1) : Pn * nev), 0.0);
    for (int q = 0; q < Pn; ++q)
        std::copy(P.theta[static_cast<size_t>(q)].begin(), P.theta[static_cast<size_t>(q)].end(),
                  th.begin() + static_cast<int64_t>(q) * (Pn == 1 ? 0 : nev));
    const int64_t thN = Pn == 1 ? want[0] : Pn * nev;
    if (mOut)
        for (int q = 0; q < Pn; ++q) mOut[q] = want[static_cast<size_t>(q)];
    const cudaMemcpyKind zk = outputsOnDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (outputsOnDevice)
        cudaCheck(cudaMemcpyAsync(theta, th.data(), sizeof(double) * thN, cudaMemcpyHostToDevice, s), "theta");
    else
        std::copy(th.begin(), th.begin() + thN, theta);
    if (recover) {
        const int64_t mc = std::min<int64_t>(mZ, zCols);
        if (mc > 0) {
            if (outputsOnDevice) cudaCheck(cudaMemcpyAsync(Z, zOut_.as<double>(), sizeof(double) * mc * n_, zk, s), "Z");
            else copyToHost(Z, zOut_.as<double>(), static_cast<size_t>(mc * n_), s);
        }
        if (zCols > mc) {
            if (outputsOnDevice)
                cudaCheck(cudaMemsetAsync(Z + mc * n_, 0, sizeof(double) * (zCols - mc) * n_, s), "Z");
            else
                std::fill(Z + mc * n_, Z + zCols * n_, 0.0);
        }
    }
    cudaCheck(cudaEventRecord(evSolve1_, s), "cudaEventRecord");
    cudaCheck(cudaStreamSynchronize(s), "outputs");
    const auto t6 = Clock::now();
    profCollect();
    lastTheta_ = P.theta[0];
    lastHasVectors_ = recover && Pn == 1;
    if (pOut) *pOut = P.p;
    if (timing) {
        timing[AMLS_T_UPLOAD] = secs(t0, t1);
        timing[AMLS_T_ELIMINATION] = secs(t1, t2);
        timing[AMLS_T_CONDENSE] = secs(t2, t3) - (tRed - secs(t3, t4));
        timing[AMLS_T_REDUCED] = tRed;
        timing[AMLS_T_BACKTRANSFORM] = secs(t4, t5) + secs(t5, t6);
        timing[AMLS_T_TOTAL] = secs(t0, t6);
        timing[AMLS_T_DEVICE] = elapsed(evSolve0_, evSolve1_);
    }
}


// ---------------------------------------------------------------------------
// batched dense generalized eigensolver: M_b = L L^T, C = L^-1 K_b L^-T,
// smallest eigenpairs of C, x = L^-T y (dsygvx itype 1 semantics)
// ---------------------------------------------------------------------------
void Engine::sygvxBatched(int batch, const int64_t* n, const int64_t* matOff, const double* K,
                          const double* M, int mode, int64_t il, int64_t iu, double lo, double hi,
                          const int64_t* cap, const int64_t* wOff, double* w, const int64_t* vOff,
                          double* V, int64_t* m) {
    (void)il;
    (void)lo;
    cudaCheck(cudaSetDevice(device_), "cudaSetDevice");
    if (batch <= 0) return;
    cudaStream_t s = stream_;
    int64_t matTot = 0, vecTot = 0, yTot = 0, wTot = 0, workTot = 0, maxN = 0;
    std::vector<int64_t> mo(static_cast<size_t>(batch)), vo(static_cast<size_t>(batch)),
        yo(static_cast<size_t>(batch)), wo(static_cast<size_t>(batch)), ko(static_cast<size_t>(batch)),
        kc(static_cast<size_t>(batch));
    for (int b = 0; b < batch; ++b) {
        const int64_t nb = n[b];
        if (nb < 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "negative matrix order");
        const int64_t want = mode == 0 ? std::min<int64_t>(iu, nb) : nb;
        kc[static_cast<size_t>(b)] = std::max<int64_t>(0, std::min<int64_t>(want, cap[b]));
        mo[static_cast<size_t>(b)] = matTot;
        matTot += nb * nb;
        vo[static_cast<size_t>(b)] = vecTot;
        vecTot += nb;
        yo[static_cast<size_t>(b)] = yTot;
        yTot += nb * kc[static_cast<size_t>(b)];
        wo[static_cast<size_t>(b)] = wTot;
        wTot += kc[static_cast<size_t>(b)];
        ko[static_cast<size_t>(b)] = workTot;
        workTot += 6 * nb * kc[static_cast<size_t>(b)];
        maxN = std::max(maxN, nb);
    }
    DevBuf dF, dG, dE, dd, de, dtau, dY, dYt, dw, dk, dwork, blob, tl, pbuf;
    double* F = static_cast<double*>(dF.ensure(sizeof(double) * (matTot + 1)));
    double* G = static_cast<double*>(dG.ensure(sizeof(double) * (matTot + 1)));
    double* E = static_cast<double*>(dE.ensure(sizeof(double) * (matTot + 1)));
    double* Yd = static_cast<double*>(dY.ensure(sizeof(double) * (yTot + 1)));
    double* Ytd = static_cast<double*>(dYt.ensure(sizeof(double) * (yTot + 1)));
    for (int b = 0; b < batch; ++b) {
        const size_t bytes = sizeof(double) * static_cast<size_t>(n[b] * n[b]);
        cudaCheck(cudaMemcpyAsync(F + mo[static_cast<size_t>(b)], M + matOff[b], bytes, cudaMemcpyHostToDevice, s), "upload M");
        cudaCheck(cudaMemcpyAsync(G + mo[static_cast<size_t>(b)], K + matOff[b], bytes, cudaMemcpyHostToDevice, s), "upload K");
    }
    dd.ensure(sizeof(double) * (vecTot + 1));
    de.ensure(sizeof(double) * (vecTot + 1));
    dtau.ensure(sizeof(double) * (vecTot + 1));
    dw.ensure(sizeof(double) * (wTot + 1));
    dk.ensure(sizeof(int32_t) * batch);
    dwork.ensure(sizeof(double) * (workTot + 1));
    cudaCheck(cudaMemsetAsync(status_.as<int>(), 0, 2 * sizeof(int), s), "status");
    std::vector<FrontDesc> fF, fE;
    std::vector<TrsmDesc> t1, t2, t3;
    std::vector<TileRef> t1T, t2T, t3T, cpT, cp2T;
    std::vector<CopyDesc> cp, cp2;
    std::vector<EigDesc> small, large, all;
    int maxLargeN = 0;
    for (int b = 0; b < batch; ++b) {
        const int64_t nb = n[b];
        if (nb == 0) continue;
        double* Fb = F + mo[static_cast<size_t>(b)];
        double* Gb = G + mo[static_cast<size_t>(b)];
        double* Eb = E + mo[static_cast<size_t>(b)];
        FrontDesc f{Fb, nb, static_cast<int32_t>(nb), static_cast<int32_t>(nb), b, 0};
        fF.push_back(f);
        fE.push_back(FrontDesc{Eb, nb, static_cast<int32_t>(nb), static_cast<int32_t>(nb), b, 0});
        TrsmDesc a{Fb, nb, Gb, nb, static_cast<int32_t>(nb), static_cast<int32_t>(nb), 0, 0};
        trsmTiles(t1T, static_cast<int>(t1.size()), nb);
        t1.push_back(a);
        CopyDesc c{Gb, nb, Eb, nb, static_cast<int32_t>(nb), static_cast<int32_t>(nb)};
        copyTiles(cpT, static_cast<int>(cp.size()), nb, nb);
        cp.push_back(c);
        TrsmDesc a2{Fb, nb, Eb, nb, static_cast<int32_t>(nb), static_cast<int32_t>(nb), 0, 0};
        trsmTiles(t2T, static_cast<int>(t2.size()), nb);
        t2.push_back(a2);
        const int64_t kb = kc[static_cast<size_t>(b)];
        EigDesc e{};
        e.A = Eb;
        e.lda = nb;
        e.d = dd.as<double>() + vo[static_cast<size_t>(b)];
        e.e = de.as<double>() + vo[static_cast<size_t>(b)];
        e.tau = dtau.as<double>() + vo[static_cast<size_t>(b)];
        e.n = static_cast<int32_t>(nb);
        e.id = b;
        e.w = dw.as<double>() + wo[static_cast<size_t>(b)];
        e.Y = Yd + yo[static_cast<size_t>(b)];
        e.ldy = nb;
        e.kcap = static_cast<int32_t>(kb);
        e.kOut = dk.as<int32_t>() + b;
        e.work = dwork.as<double>() + ko[static_cast<size_t>(b)];
        all.push_back(e);
        if (nb <= kSmallEig) small.push_back(e);
        else {
            large.push_back(e);
            maxLargeN = std::max<int>(maxLargeN, static_cast<int>(nb));
        }
        if (kb > 0) {
            // Y (nb x kb) -> Yt (kb x nb), Yt <- Yt L^-1, Yt -> Y
            CopyDesc y1{Yd + yo[static_cast<size_t>(b)], nb, Ytd + yo[static_cast<size_t>(b)], kb,
                        static_cast<int32_t>(nb), static_cast<int32_t>(kb)};
            copyTiles(cp2T, static_cast<int>(cp2.size()), nb, kb);
            cp2.push_back(y1);
            TrsmDesc a3{Fb, nb, Ytd + yo[static_cast<size_t>(b)], kb, static_cast<int32_t>(nb),
                        static_cast<int32_t>(kb), 0, 1};
            trsmTiles(t3T, static_cast<int>(t3.size()), kb);
            t3.push_back(a3);
        }
    }
    // back-copy descriptors (Yt -> Y)
    std::vector<CopyDesc> cp3;
    std::vector<TileRef> cp3T;
    for (const CopyDesc& c : cp2) {
        CopyDesc r{c.out, c.ldout, const_cast<double*>(c.in), c.ldin, c.c, c.r};
        copyTiles(cp3T, static_cast<int>(cp3.size()), c.c, c.r);
        cp3.push_back(r);
    }
    Blob B;
    std::vector<TileRef> symT;                          // 32 x 32 tile pairs of every C (tile units)
    for (size_t q = 0; q < fE.size(); ++q)
        for (int bj = 0; bj < cdiv(fE[q].n, 32); ++bj)
            for (int bi = bj; bi < cdiv(fE[q].n, 32); ++bi) symT.push_back({static_cast<int32_t>(q), bi, bj, 0});
    const size_t oSymT = B.add(symT);
    const size_t ofF = B.add(fF), ofE = B.add(fE), ot1 = B.add(t1), ot1T = B.add(t1T), ocp = B.add(cp),
                 ocpT = B.add(cpT), ot2 = B.add(t2), ot2T = B.add(t2T), oS = B.add(small), oL = B.add(large),
                 oA = B.add(all), ocp2 = B.add(cp2), ocp2T = B.add(cp2T), ot3 = B.add(t3), ot3T = B.add(t3T),
                 ocp3 = B.add(cp3), ocp3T = B.add(cp3T);
    B.upload(blob, s);
    const int nb = static_cast<int>(fF.size());
    const int maxBlocks = cdiv(maxN, kCholBlock), maxRowTiles = cdiv(maxN, kTrsmRows);
    for (int jb = 0; jb < maxBlocks; ++jb) {
        LAUNCH(launchCholDiag(B.dev<FrontDesc>(ofF), nb, jb, status_.as<int>(), s));
        LAUNCH(launchCholPanel(B.dev<FrontDesc>(ofF), nb, jb, maxRowTiles, s));
    }
    LAUNCH(launchTrsmRows(B.dev<TrsmDesc>(ot1), B.dev<TileRef>(ot1T), static_cast<int>(t1T.size()), s));
    LAUNCH(launchTransposeBatched(B.dev<CopyDesc>(ocp), B.dev<TileRef>(ocpT), static_cast<int>(cpT.size()), s));
    LAUNCH(launchTrsmRows(B.dev<TrsmDesc>(ot2), B.dev<TileRef>(ot2T), static_cast<int>(t2T.size()), s));
    LAUNCH(launchSymmetrizeTiles(B.dev<FrontDesc>(ofE), B.dev<TileRef>(oSymT), static_cast<int>(symT.size()), s));
    if (!small.empty()) LAUNCH(launchTridiagSmall(B.dev<EigDesc>(oS), static_cast<int>(small.size()), s));
    (void)oL;
    (void)maxLargeN;
    tridiagLargeAll(large, pbuf, tlLargeBlob_, s);
    int maxK = 0;
    for (auto x : kc) maxK = std::max<int>(maxK, static_cast<int>(x));
    const int bmode = mode == 0 ? 2 : 3;
    LAUNCH(launchBisect(B.dev<EigDesc>(oA), static_cast<int>(all.size()), bmode, static_cast<int>(iu), hi, maxK,
                        nullptr, s));
    LAUNCH(launchInverseIter(B.dev<EigDesc>(oA), static_cast<int>(all.size()), maxK, nullptr, s));
    LAUNCH(launchBackTransform(B.dev<EigDesc>(oA), static_cast<int>(all.size()), maxK, s));
    LAUNCH(launchTransposeBatched(B.dev<CopyDesc>(ocp2), B.dev<TileRef>(ocp2T), static_cast<int>(cp2T.size()), s));
    LAUNCH(launchTrsmRows(B.dev<TrsmDesc>(ot3), B.dev<TileRef>(ot3T), static_cast<int>(t3T.size()), s));
    LAUNCH(launchTransposeBatched(B.dev<CopyDesc>(ocp3), B.dev<TileRef>(ocp3T), static_cast<int>(cp3T.size()), s));
    checkStatus("sygvx");
    std::vector<int32_t> kh(static_cast<size_t>(batch), 0);
    cudaCheck(cudaMemcpy(kh.data(), dk.as<int32_t>(), sizeof(int32_t) * batch, cudaMemcpyDeviceToHost), "k");
    int idx = 0;
    for (int b = 0; b < batch; ++b) {
        if (n[b] == 0) {
            m[b] = 0;
            continue;
        }
        const int64_t kb = std::min<int64_t>(kh[static_cast<size_t>(idx++)], kc[static_cast<size_t>(b)]);
        m[b] = kb;
        if (kb <= 0) continue;
        cudaCheck(cudaMemcpy(w + wOff[b], dw.as<double>() + wo[static_cast<size_t>(b)], sizeof(double) * kb,
                             cudaMemcpyDeviceToHost), "w");
        cudaCheck(cudaMemcpy(V + vOff[b], Yd + yo[static_cast<size_t>(b)], sizeof(double) * kb * n[b],
                             cudaMemcpyDeviceToHost), "V");
    }
    (void)ko;
}

// ---------------------------------------------------------------------------
// stage-by-stage solve (one pencil)
// ---------------------------------------------------------------------------
void Engine::stageEliminate(const double* kv, const double* mv, bool onDevice) {
    if (!analyzed_) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "amls_eliminate before amls_analyze");
    if (nPencils_ != 1) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "stage calls need a single pencil");
    cudaCheck(cudaSetDevice(device_), "cudaSetDevice");
    launches_ = 0;
    for (int t = 2; t < AMLS_WORK_SLOTS; ++t) work_[t] = 0;
    for (int c = 0; c < kProfCats; ++c) {
        catF_[c] = elimCatF_[c];
        catB_[c] = elimCatB_[c];
    }
    tridiagDone_ = false;
    stageLevel_ = 0;
    numericElimination(kv, mv, onDevice, stream_);
    stageLevel_ = 1;
}

void Engine::stageCondense(int mode, int k, double lambdaCut, int64_t* pOut) {
    if (stageLevel_ < 1) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "amls_condense before amls_eliminate");
    if (mode != 0 && mode != 1) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "mode must be 0 (fixed count) or 1 (threshold)");
    if (mode == 0 && k <= 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "fixed count must be positive");
    stage_ = Pass();
    const double thr = lambdaCut > 0 ? 1.0 / lambdaCut : 1e300;
    condense(mode, {mode == 0 ? k : 0}, {mode == 0 ? 0.0 : thr}, {mode == 0 ? 0.0 : lambdaCut}, stage_, stream_);
    stageLevel_ = 2;
    if (pOut) *pOut = stage_.p;
}

void Engine::stageModes(int32_t* kNode, double* mu) const {
    if (stageLevel_ < 2) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "no condensed pass on the handle");
    if (kNode) std::copy(stage_.k.begin(), stage_.k.end(), kNode);
    if (mu) {
        std::vector<double> nu(static_cast<size_t>(stage_.p));
        cudaCheck(cudaMemcpy(nu.data(), wPool_.as<double>(), sizeof(double) * stage_.p, cudaMemcpyDeviceToHost), "modes");
        for (int64_t j = 0; j < stage_.p; ++j) mu[j] = 1.0 / nu[static_cast<size_t>(j)];
    }
}

void Engine::stageReduced(int want, bool vectors, double* theta, int64_t* mOut) {
    if (stageLevel_ < 2) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "amls_reduced_eig before amls_condense");
    if (want <= 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "want must be positive");
    reducedSolve(stage_, {want}, stream_, vectors);
    const auto& th = stage_.theta[0];
    if (theta) std::copy(th.begin(), th.end(), theta);
    if (mOut) *mOut = static_cast<int64_t>(th.size());
    stageLevel_ = vectors ? 4 : 3;
}

void Engine::stageBacktransform(double* Z, bool onDevice, int64_t* mOut) {
    if (stageLevel_ < 4) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "amls_backtransform needs amls_reduced_eig with vectors");
    const int m = stage_.got[0];
    backtransform(stage_, m, stream_);
    finalizeVectors(ztPool_.as<double>(), m, m, stream_);
    if (Z)
        cudaCheck(cudaMemcpy(Z, zOut_.as<double>(), sizeof(double) * m * n_,
                             onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost), "Z");
    if (mOut) *mOut = m;
    stageLevel_ = 5;
}

void Engine::stageRefine(int nev, double* theta, double* Z, bool onDevice, int64_t* iters) {
    if (stageLevel_ < 5) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "amls_refine needs amls_backtransform first");
    if (opt_.refine < 1)
        throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "amls_refine needs an analysis with refine >= 1 (applications per step)");
    const int m = stage_.got[0];
    if (nev <= 0 || nev > m) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "nev must be 1 .. the back-transformed count");
    std::vector<double> th = stage_.theta[0];
    const int it = refine(ztPool_.as<double>(), m, nev, th, Z != nullptr, stream_);
    th.resize(static_cast<size_t>(nev));
    if (theta) std::copy(th.begin(), th.end(), theta);
    if (Z) {
        finalizeVectors(ztPool_.as<double>(), m, nev, stream_);
        cudaCheck(cudaMemcpy(Z, zOut_.as<double>(), sizeof(double) * nev * n_,
                             onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost), "Z");
    }
    if (iters) *iters = it;
    lastTheta_ = th;
    lastHasVectors_ = Z != nullptr;
    stageLevel_ = 1;          // the basis in ztPool_ is consumed
}

void Engine::tree(int64_t* nNodes, int64_t* parent, int64_t* size, int32_t* level) const {
    const int N = static_cast<int>(nodes_.size());
    if (nNodes) *nNodes = N;
    for (int i = 0; i < N; ++i) {
        const Node& nd = nodes_[static_cast<size_t>(i)];
        if (parent) parent[i] = nd.parent;
        if (size) size[i] = nd.n;
        if (level) level[i] = nd.level;
    }
}

void Engine::sensitivities(int64_t nelem, int nd, const int64_t* dofmap, int32_t ntypes,
                           const int32_t* elemType, const double* Kbar,
                           const double* Mbar, const double* weights, double gapTol, double* gE,
                           double* gRho, double* dE, double* dRho, int32_t* simple) {
    if (!lastHasVectors_ || lastTheta_.empty())
        throw AmlsError(AMLS_ERR_INVALID_ARGUMENT,
                        "sensitivities need a preceding solve with recovered eigenvectors");
    if (nd <= 0 || nd > 96) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "element DOF count must be 1..96");
    if (ntypes < 1) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "element type count must be >= 1");
    if (elemType) {
        for (int64_t e = 0; e < nelem; ++e)
            if (elemType[e] < 0 || elemType[e] >= ntypes)
                throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "element type out of range");
    } else if (ntypes != 1) {
        throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "element types needed when ntypes > 1");
    }
    for (int64_t q = 0; q < nelem * nd; ++q)
        if (dofmap[q] < -1 || dofmap[q] >= n_)
            throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "dofmap entry out of range");
    cudaCheck(cudaSetDevice(device_), "cudaSetDevice");
    cudaStream_t s = stream_;
    const int nm = static_cast<int>(lastTheta_.size());
    // simple-eigenvalue test (relative gap to the neighbours above gapTol)
    std::vector<double> w(static_cast<size_t>(nm));
    for (int k = 0; k < nm; ++k) {
        const double lk = lastTheta_[static_cast<size_t>(k)];
        double gap = 1e300;
        if (k > 0) gap = std::min(gap, std::fabs(lk - lastTheta_[static_cast<size_t>(k - 1)]));
        if (k + 1 < nm) gap = std::min(gap, std::fabs(lastTheta_[static_cast<size_t>(k + 1)] - lk));
        const bool ok = gap > gapTol * std::fabs(lk);
        if (simple) simple[k] = ok ? 1 : 0;
        w[static_cast<size_t>(k)] = ok ? (weights ? weights[k] : 0.0) : std::nan("");
    }
    int64_t* dDof = static_cast<int64_t*>(senDof_.ensure(sizeof(int64_t) * nelem * nd));
    const int64_t nmat = static_cast<int64_t>(ntypes) * nd * nd;
    double* dEl = static_cast<double*>(senEl_.ensure(sizeof(double) * (2 * nmat + 2 * nm)));
    int32_t* dType = nullptr;
    if (elemType) {
        dType = static_cast<int32_t*>(senType_.ensure(sizeof(int32_t) * nelem));
        cudaCheck(cudaMemcpyAsync(dType, elemType, sizeof(int32_t) * nelem, cudaMemcpyHostToDevice, s), "types");
    }
    const size_t outN = static_cast<size_t>(nelem) * (2 + (dE ? nm : 0) + (dRho ? nm : 0));
    double* dOut = static_cast<double*>(senOut_.ensure(sizeof(double) * outN));
    cudaCheck(cudaMemcpyAsync(dDof, dofmap, sizeof(int64_t) * nelem * nd, cudaMemcpyHostToDevice, s), "dofmap");
    cudaCheck(cudaMemcpyAsync(dEl, Kbar, sizeof(double) * nmat, cudaMemcpyHostToDevice, s), "Kbar");
    cudaCheck(cudaMemcpyAsync(dEl + nmat, Mbar, sizeof(double) * nmat, cudaMemcpyHostToDevice, s), "Mbar");
    cudaCheck(cudaMemcpyAsync(dEl + 2 * nmat, lastTheta_.data(), sizeof(double) * nm, cudaMemcpyHostToDevice, s), "theta");
    cudaCheck(cudaMemcpyAsync(dEl + 2 * nmat + nm, w.data(), sizeof(double) * nm, cudaMemcpyHostToDevice, s), "weights");
    double* oE = dOut;
    double* oR = dOut + nelem;
    double* odE = dE ? dOut + 2 * nelem : nullptr;
    double* odR = dRho ? dOut + 2 * nelem + (dE ? nelem * nm : 0) : nullptr;
    LAUNCH(launchSensitivity(nelem, nd, dDof, dType, dEl, dEl + nmat, zOut_.as<double>(), n_, nm,
                             dEl + 2 * nmat, dEl + 2 * nmat + nm, oE, oR, odE, odR, s));
    if (gE) cudaCheck(cudaMemcpyAsync(gE, oE, sizeof(double) * nelem, cudaMemcpyDeviceToHost, s), "gE");
    if (gRho) cudaCheck(cudaMemcpyAsync(gRho, oR, sizeof(double) * nelem, cudaMemcpyDeviceToHost, s), "gRho");
    if (dE) cudaCheck(cudaMemcpyAsync(dE, odE, sizeof(double) * nelem * nm, cudaMemcpyDeviceToHost, s), "dE");
    if (dRho) cudaCheck(cudaMemcpyAsync(dRho, odR, sizeof(double) * nelem * nm, cudaMemcpyDeviceToHost, s), "dRho");
    cudaCheck(cudaStreamSynchronize(s), "sensitivities");
}


void Engine::assembleHex(int order, int64_t nelem, int64_t nnodes, const double* coords, const int64_t* enodes,
                         const int64_t* dofmap, const double* E, const double* rho, double nu, int64_t n,
                         const int64_t* rowptr, const int32_t* col, double* kval, double* mval,
                         bool outputsOnDevice) {
    if (order != 1 && order != 2) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "element order must be 1 or 2");
    if (nelem <= 0 || nnodes <= 0 || n <= 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "empty mesh");
    const int nn = (order + 1) * (order + 1) * (order + 1), nd = 3 * nn;
    for (int64_t q = 0; q < nelem * nn; ++q)
        if (enodes[q] < 0 || enodes[q] >= nnodes) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "element node id out of range");
    for (int64_t q = 0; q < nelem * nd; ++q)
        if (dofmap[q] < -1 || dofmap[q] >= n) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "dofmap entry out of range");
    const int64_t nnz = rowptr[n];
    cudaCheck(cudaSetDevice(device_), "cudaSetDevice");
    cudaStream_t s = stream_;
    auto up = [&](DevBuf& b, const void* src, size_t bytes) {
        b.ensure(bytes);
        cudaCheck(cudaMemcpyAsync(b.as<char>(), src, bytes, cudaMemcpyHostToDevice, s), "assembly upload");
    };
    up(asmCoords_, coords, sizeof(double) * nnodes * 3);
    up(asmEnodes_, enodes, sizeof(int64_t) * nelem * nn);
    up(asmDof_, dofmap, sizeof(int64_t) * nelem * nd);
    up(asmE_, E, sizeof(double) * nelem);
    up(asmRho_, rho, sizeof(double) * nelem);
    up(asmRp_, rowptr, sizeof(int64_t) * (n + 1));
    up(asmCol_, col, sizeof(int32_t) * std::max<int64_t>(nnz, 1));
    double* kd = outputsOnDevice ? kval : static_cast<double*>(asmK_.ensure(sizeof(double) * std::max<int64_t>(nnz, 1)));
    double* md = outputsOnDevice ? mval : static_cast<double*>(asmM_.ensure(sizeof(double) * std::max<int64_t>(nnz, 1)));
    cudaCheck(cudaMemsetAsync(status_.as<int>(), 0, 2 * sizeof(int), s), "status");
    HexAssembleArgs a{};
    a.order = order;
    a.nelem = nelem;
    a.coords = asmCoords_.as<double>();
    a.enodes = asmEnodes_.as<int64_t>();
    a.dofmap = asmDof_.as<int64_t>();
    a.E = asmE_.as<double>();
    a.rho = asmRho_.as<double>();
    a.nu = nu;
    a.rowptr = asmRp_.as<int64_t>();
    a.col = asmCol_.as<int32_t>();
    a.nnz = nnz;
    a.kval = kd;
    a.mval = md;
    a.status = status_.as<int>();
    LAUNCH(launchHexAssemble(a, s));
    int h[2] = {0, 0};
    cudaCheck(cudaMemcpyAsync(h, status_.as<int>(), sizeof(h), cudaMemcpyDeviceToHost, s), "status");
    if (!outputsOnDevice) {
        cudaCheck(cudaMemcpyAsync(kval, kd, sizeof(double) * nnz, cudaMemcpyDeviceToHost, s), "K values");
        cudaCheck(cudaMemcpyAsync(mval, md, sizeof(double) * nnz, cudaMemcpyDeviceToHost, s), "M values");
    }
    cudaCheck(cudaStreamSynchronize(s), "assembly");
    if (h[0] == kDevBadPattern)
        throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "element " + std::to_string(h[1]) + " couples DOFs the CSR pattern lacks");
}

void Engine::finalizeVectors(const double* zt, int64_t ldz, int m, cudaStream_t s) {
    norms_.ensure(sizeof(double) * static_cast<size_t>(m) * nPencils_);
    zOut_.ensure(sizeof(double) * static_cast<size_t>(m * n_));
    LAUNCH(launchMNormSuper(supDesc_.as<SpmmSuper>(), nSup_, supCols_.as<int32_t>(), supVal_.as<double>(),
                            invDev_.as<int64_t>(), zt, m, ldz, norms_.as<double>(), nPencils_, s));
    LAUNCH(launchUnpermute(zt, ldz, m, n_, permDev_.as<int64_t>(), norms_.as<double>(), zOut_.as<double>(), s,
                           nPencils_ > 1 ? pencilDev_.as<int32_t>() : nullptr));
    cudaCheck(cudaStreamSynchronize(s), "finalize");
}

void Engine::info(int64_t* out) const {
    int64_t ft = frontTotal_;
    out[0] = static_cast<int64_t>(nodes_.size());
    out[1] = maxLevel_ + 1;
    out[2] = pA_;
    out[3] = pFinal_;
    out[4] = ft;
    size_t freeB = 0, totB = 0;
    cudaMemGetInfo(&freeB, &totB);
    out[5] = static_cast<int64_t>(totB - freeB);
    out[6] = launches_;
    out[7] = refineIters_;
    out[8] = refineNq_;
    out[9] = n_;
    out[10] = static_cast<int64_t>(sil_.size());
    out[11] = silServed_;
}

void Engine::permutation(int64_t* out) const {
    std::copy(perm_.begin(), perm_.end(), out);
}

void Engine::categoryWork(double* flops, double* bytes) const {
    for (int c = 0; c < kProfCats; ++c) {
        if (flops) flops[c] = catF_[c];
        if (bytes) bytes[c] = catB_[c];
    }
}

void Engine::work(double* out) const {
    for (int i = 0; i < AMLS_WORK_SLOTS; ++i) out[i] = work_[i];
}

}  // namespace amls_b200
