// Nested-dissection partition on the host through METIS.
//
// The METIS library is the one shipped with the CUDA toolkit
// (libmetis_static.a, METIS 5 API, 64-bit idx_t established at run time by
// METIS_SetDefaultOptions filling 40 x 8 bytes).  The graph construction and
// the recursion restate src/partition/metis_partitioner.cpp:
//   * extractGraph (:20-45): adjacency of |K|+|M| without self loops;
//   * inducedSubgraph (:48-73): neighbour lists sorted;
//   * bisect (:80-106): ComputeVertexSeparator with options seed 42
//     (metis_call.hpp).  The reference first calls PartGraphRecursive and
//     never reads its result; METIS re-seeds its generator from the options
//     at the start of every API call, so dropping that call leaves the
//     separator unchanged (checked on the benchmark pencils: identical
//     permutations) and saves its time;
//   * recursion (:110-160) and perm = post-order concatenation (:168-175).
#include "tree.hpp"

#include <dlfcn.h>
#include <spawn.h>
#include <sys/socket.h>
#include <sys/wait.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <condition_variable>
#include <csignal>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>

#include "host/metis_call.hpp"

extern char** environ;

namespace amls_b200 {

namespace {
std::mutex gMetisMutex;   // METIS keeps process-wide state: one call at a time

struct Csr {
    std::vector<int64_t> xadj, adjncy;
};

// Adjacency of |K| + |M| without self loops (the patterns are symmetric),
// neighbour lists sorted.  The reference builds the same sets through one
// std::unordered_set per vertex (metis_partitioner.cpp:20-45), but every
// graph it hands to METIS, the root's included, goes through
// inducedSubgraph, which sorts each list (:48-73); only the sets matter.
// Rows are processed in parallel over host threads.
Csr extractGraph(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp,
                 const int32_t* mc) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nt > 64) nt = 64;
    if (n < 4096) nt = 1;
    auto forRange = [&](auto&& fn) {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                const int64_t b = n * t / nt, e = n * (t + 1) / nt;
                fn(b, e);
            });
        for (auto& x : th) x.join();
    };
    std::vector<std::vector<int64_t>> lists(static_cast<size_t>(n));
    forRange([&](int64_t b, int64_t e) {
        for (int64_t v = b; v < e; ++v) {
            auto& out = lists[static_cast<size_t>(v)];
            out.clear();
            for (int64_t q = kp[v]; q < kp[v + 1]; ++q)
                if (kc[q] != v) out.push_back(kc[q]);
            for (int64_t q = mp[v]; q < mp[v + 1]; ++q)
                if (mc[q] != v) out.push_back(mc[q]);
            std::sort(out.begin(), out.end());
            out.erase(std::unique(out.begin(), out.end()), out.end());
        }
    });
    Csr g;
    g.xadj.assign(static_cast<size_t>(n) + 1, 0);
    for (int64_t i = 0; i < n; ++i)
        g.xadj[static_cast<size_t>(i) + 1] =
            g.xadj[static_cast<size_t>(i)] + static_cast<int64_t>(lists[static_cast<size_t>(i)].size());
    g.adjncy.resize(static_cast<size_t>(g.xadj.back()));
    forRange([&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i)
            std::copy(lists[static_cast<size_t>(i)].begin(), lists[static_cast<size_t>(i)].end(),
                      g.adjncy.begin() + g.xadj[static_cast<size_t>(i)]);
    });
    return g;
}

// Subgraph induced by `verts` (ascending, as every vertex set of the
// recursion is: the root's is 0..n-1 and a split keeps the order), vertices
// renumbered by their position in `verts`.  The renumbering is increasing,
// so each neighbour list stays sorted.  Large sets are counted and filled in
// parallel over host threads (the top levels of the recursion, whose calls
// are on its critical path while few other threads run).
Csr inducedSubgraph(const Csr& g, const std::vector<int64_t>& verts, std::vector<int64_t>& localOf) {
    const int64_t m = static_cast<int64_t>(verts.size());
    localOf.assign(g.xadj.size() - 1, -1);
    for (int64_t i = 0; i < m; ++i) localOf[static_cast<size_t>(verts[static_cast<size_t>(i)])] = i;
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nt > 16) nt = 16;
    if (m < 16384) nt = 1;
    auto forRange = [&](auto&& fn) {
        if (nt == 1) {
            fn(int64_t{0}, m);
            return;
        }
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t)
            th.emplace_back([&, t] { fn(m * t / nt, m * (t + 1) / nt); });
        for (auto& x : th) x.join();
    };
    Csr sub;
    sub.xadj.assign(static_cast<size_t>(m) + 1, 0);
    forRange([&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            const int64_t v = verts[static_cast<size_t>(i)];
            int64_t c = 0;
            for (int64_t p = g.xadj[static_cast<size_t>(v)]; p < g.xadj[static_cast<size_t>(v) + 1]; ++p)
                c += localOf[static_cast<size_t>(g.adjncy[static_cast<size_t>(p)])] >= 0;
            sub.xadj[static_cast<size_t>(i) + 1] = c;
        }
    });
    for (int64_t i = 0; i < m; ++i) sub.xadj[static_cast<size_t>(i) + 1] += sub.xadj[static_cast<size_t>(i)];
    sub.adjncy.resize(static_cast<size_t>(sub.xadj.back()));
    forRange([&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            const int64_t v = verts[static_cast<size_t>(i)];
            int64_t o = sub.xadj[static_cast<size_t>(i)];
            for (int64_t p = g.xadj[static_cast<size_t>(v)]; p < g.xadj[static_cast<size_t>(v) + 1]; ++p) {
                const int64_t u = localOf[static_cast<size_t>(g.adjncy[static_cast<size_t>(p)])];
                if (u >= 0) sub.adjncy[static_cast<size_t>(o++)] = u;
            }
        }
    });
    return sub;
}

// In-process separator (serialised); part[v] in {0, 1, 2}, 2 = separator.
// METIS reads the graph arrays only (its coarsening builds new graphs), so
// the caller's graph is passed as it is, without a copy.
std::vector<int64_t> bisectInProcess(const Csr& g) {
    const int64_t n = static_cast<int64_t>(g.xadj.size()) - 1;
    std::vector<int64_t> part(static_cast<size_t>(n), 0);
    if (n == 0) return part;
    int rc;
    {
        std::lock_guard<std::mutex> lock(gMetisMutex);
        rc = metisSeparator(n, const_cast<int64_t*>(g.xadj.data()), const_cast<int64_t*>(g.adjncy.data()),
                            part.data());
    }
    if (rc != kMetisOk) throw std::runtime_error("METIS_ComputeVertexSeparator failed");
    return part;
}

bool sendAll(int fd, const void* p, size_t bytes) {
    const char* c = static_cast<const char*>(p);
    while (bytes > 0) {
        const ssize_t r = send(fd, c, bytes, MSG_NOSIGNAL);
        if (r < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        c += r;
        bytes -= static_cast<size_t>(r);
    }
    return true;
}
bool recvAll(int fd, void* p, size_t bytes) {
    char* c = static_cast<char*>(p);
    while (bytes > 0) {
        const ssize_t r = recv(fd, c, bytes, 0);
        if (r == 0) return false;
        if (r < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        c += r;
        bytes -= static_cast<size_t>(r);
    }
    return true;
}

// the separator worker program sits next to this library
std::string workerPath() {
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&workerPath), &info) == 0 || !info.dli_fname) return "";
    std::string lib = info.dli_fname;
    const size_t k = lib.rfind('/');
    const std::string dir = k == std::string::npos ? "." : lib.substr(0, k);
    const std::string path = dir + "/amls_metis_worker";
    return access(path.c_str(), X_OK) == 0 ? path : "";
}

// Separator workers: `slots` concurrent METIS calls, one in this process and
// the rest in worker processes (each with its own METIS state).  A call on
// a worker that fails for any reason (no worker program, a broken socket) is
// made in this process instead; the separator is the same either way.
class SeparatorPool {
public:
    explicit SeparatorPool(int slots) {
        slots_.push_back(Slot{});              // the in-process slot
        const std::string path = slots > 1 ? workerPath() : "";
        for (int w = 1; w < slots && !path.empty(); ++w) {
            int sv[2];
            if (socketpair(AF_UNIX, SOCK_STREAM | SOCK_CLOEXEC, 0, sv) != 0) break;
            posix_spawn_file_actions_t fa;
            posix_spawn_file_actions_init(&fa);
            posix_spawn_file_actions_adddup2(&fa, sv[1], 0);
            posix_spawn_file_actions_adddup2(&fa, sv[1], 1);
            char* argv[] = {const_cast<char*>(path.c_str()), nullptr};
            pid_t pid = 0;
            const int rc = posix_spawn(&pid, path.c_str(), &fa, nullptr, argv, environ);
            posix_spawn_file_actions_destroy(&fa);
            close(sv[1]);
            if (rc != 0) {
                close(sv[0]);
                break;
            }
            Slot s;
            s.pid = pid;
            s.fd = sv[0];
            slots_.push_back(s);
        }
    }
    ~SeparatorPool() {
        for (Slot& s : slots_)
            if (s.fd >= 0) retire(s);
    }
    SeparatorPool(const SeparatorPool&) = delete;
    SeparatorPool& operator=(const SeparatorPool&) = delete;

    std::vector<int64_t> separator(const Csr& g) {
        size_t k;
        {
            std::unique_lock<std::mutex> lock(m_);
            cv_.wait(lock, [&] {
                for (const Slot& s : slots_)
                    if (!s.busy) return true;
                return false;
            });
            // this process first (the call needs no copy of the graph; the
            // root's separator, the largest call, always runs here), then
            // the workers
            k = slots_.size();
            for (size_t i = 0; i < slots_.size(); ++i)
                if (!slots_[i].busy) {
                    k = i;
                    break;
                }
            slots_[k].busy = true;
        }
        std::vector<int64_t> part;
        bool done = false;
        if (slots_[k].fd >= 0) done = remote(slots_[k], g, part);
        std::exception_ptr err;
        if (!done) {
            try {
                part = bisectInProcess(g);
            } catch (...) {
                err = std::current_exception();
            }
        }
        {
            std::lock_guard<std::mutex> lock(m_);
            slots_[k].busy = false;
        }
        cv_.notify_one();
        if (err) std::rethrow_exception(err);
        return part;
    }

private:
    struct Slot {
        pid_t pid = -1;
        int fd = -1;
        bool busy = false;
    };
    bool remote(Slot& s, const Csr& g, std::vector<int64_t>& part) {
        const int64_t n = static_cast<int64_t>(g.xadj.size()) - 1;
        const int64_t hdr[2] = {n, static_cast<int64_t>(g.adjncy.size())};
        int64_t status = 0;
        part.assign(static_cast<size_t>(n), 0);
        const bool ok = sendAll(s.fd, hdr, sizeof(hdr)) &&
                        sendAll(s.fd, g.xadj.data(), sizeof(int64_t) * g.xadj.size()) &&
                        sendAll(s.fd, g.adjncy.data(), sizeof(int64_t) * g.adjncy.size()) &&
                        recvAll(s.fd, &status, sizeof(status)) && status == kMetisOk &&
                        (n == 0 || recvAll(s.fd, part.data(), sizeof(int64_t) * static_cast<size_t>(n)));
        if (!ok) retire(s);
        return ok;
    }
    static void retire(Slot& s) {
        shutdown(s.fd, SHUT_RDWR);
        close(s.fd);
        s.fd = -1;
        if (s.pid > 0) {
            int st = 0;
            while (waitpid(s.pid, &st, 0) < 0 && errno == EINTR) {
            }
        }
        s.pid = -1;
    }
    std::mutex m_;
    std::condition_variable cv_;
    std::vector<Slot> slots_;
};
}  // namespace

int64_t SeparatorTree::addNode(NodeRole role, std::vector<int64_t> idx) {
    TreeNode nd;
    nd.id = static_cast<int64_t>(nodes_.size());
    nd.role = role;
    nd.indices = std::move(idx);
    nodes_.push_back(std::move(nd));
    return nodes_.back().id;
}

void SeparatorTree::postOrderRec(int64_t id, std::vector<int64_t>& out) const {
    for (int64_t c : node(id).children) postOrderRec(c, out);
    out.push_back(id);
}

std::vector<int64_t> SeparatorTree::postOrder() const {
    std::vector<int64_t> out;
    out.reserve(nodes_.size());
    if (!nodes_.empty()) postOrderRec(root(), out);
    return out;
}

std::vector<int64_t> SeparatorTree::ancestors(int64_t id) const {
    std::vector<int64_t> out;
    for (int64_t p = node(id).parent; p != -1; p = node(p).parent) out.push_back(p);
    return out;
}

int64_t SeparatorTree::root() const {
    for (const auto& nd : nodes_)
        if (nd.parent == -1) return nd.id;
    return -1;
}

void SeparatorTree::relabelRoot() {
    const int64_t r = root();
    if (r >= 0 && nodes_[static_cast<size_t>(r)].role == NodeRole::Separator)
        nodes_[static_cast<size_t>(r)].role = NodeRole::Root;
}

bool SeparatorTree::validate(int64_t nTotal) const {
    if (nodes_.empty()) return false;
    int roots = 0;
    for (const auto& nd : nodes_) roots += nd.parent == -1;
    if (roots != 1) return false;
    for (const auto& nd : nodes_) {
        if (nd.role == NodeRole::Leaf && !nd.children.empty()) return false;
        if (nd.role != NodeRole::Leaf && nd.children.size() != 2) return false;
        for (int64_t c : nd.children)
            if (node(c).parent != nd.id) return false;
    }
    std::vector<int64_t> all;
    for (const auto& nd : nodes_) all.insert(all.end(), nd.indices.begin(), nd.indices.end());
    if (static_cast<int64_t>(all.size()) != nTotal) return false;
    std::sort(all.begin(), all.end());
    for (int64_t i = 0; i < nTotal; ++i)
        if (all[static_cast<size_t>(i)] != i) return false;
    return true;
}

namespace {
// Result of the recursive bisection of one vertex set, built before any tree
// node is created so the two halves can run concurrently.
struct Split {
    std::vector<int64_t> verts;               // leaf: its vertices
    std::vector<int64_t> sep;                 // separator (empty for a leaf)
    std::unique_ptr<Split> left, right;
};

// The top levels run their two halves on two threads, their METIS calls in
// separate worker processes (SeparatorPool).  Every METIS call re-seeds from
// its own options, so the split of each vertex set depends on nothing but
// that vertex set: the tree is the same for any thread or worker count.

std::unique_ptr<Split> splitRec(const Csr& g, std::vector<int64_t> verts, int depth, int nLevels,
                                int64_t leafSize, SeparatorPool& pool, int parDepth) {
    auto out = std::make_unique<Split>();
    const int64_t m = static_cast<int64_t>(verts.size());
    if (m <= leafSize || depth >= nLevels || m < 4) {
        out->verts = std::move(verts);
        return out;
    }
    // the root's vertex set is all of g in order: its induced subgraph is g
    std::vector<int64_t> localOf;
    const std::vector<int64_t> part =
        depth == 0 ? pool.separator(g) : pool.separator(inducedSubgraph(g, verts, localOf));
    std::vector<int64_t> side[2], sep;
    for (int64_t i = 0; i < m; ++i) {
        const int64_t p = part[static_cast<size_t>(i)];
        if (p == 2) sep.push_back(verts[static_cast<size_t>(i)]);
        else side[p].push_back(verts[static_cast<size_t>(i)]);
    }
    const int64_t minSide = static_cast<int64_t>(std::min(side[0].size(), side[1].size()));
    if (sep.empty() || minSide < 2) {
        out->verts = std::move(verts);
        return out;
    }
    out->sep = std::move(sep);
    if (depth < parDepth) {
        std::exception_ptr err;
        std::thread t([&] {
            try {
                out->left = splitRec(g, std::move(side[0]), depth + 1, nLevels, leafSize, pool, parDepth);
            } catch (...) {
                err = std::current_exception();
            }
        });
        try {
            out->right = splitRec(g, std::move(side[1]), depth + 1, nLevels, leafSize, pool, parDepth);
        } catch (...) {
            t.join();
            throw;
        }
        t.join();
        if (err) std::rethrow_exception(err);
    } else {
        out->left = splitRec(g, std::move(side[0]), depth + 1, nLevels, leafSize, pool, parDepth);
        out->right = splitRec(g, std::move(side[1]), depth + 1, nLevels, leafSize, pool, parDepth);
    }
    return out;
}

// tree nodes in the reference's creation order: separator, then the left
// subtree, then the right one (metis_partitioner.cpp:110-160)
int64_t buildTree(SeparatorTree& tree, Split& s) {
    if (!s.left) return tree.addNode(NodeRole::Leaf, std::move(s.verts));
    const int64_t sepId = tree.addNode(NodeRole::Separator, std::move(s.sep));
    const int64_t l = buildTree(tree, *s.left);
    const int64_t r = buildTree(tree, *s.right);
    tree.setChildren(sepId, l, r);
    tree.setParent(l, sepId);
    tree.setParent(r, sepId);
    return sepId;
}
}  // namespace

PartitionResult recursiveBisection(int64_t n, const int64_t* kRowPtr, const int32_t* kCol,
                                   const int64_t* mRowPtr, const int32_t* mCol, int nLevels,
                                   int64_t leafSize, int numThreads) {
    if (n == 0) return PartitionResult();
    Csr g = extractGraph(n, kRowPtr, kCol, mRowPtr, mCol);
    return recursiveBisectionGraph(n, std::move(g.xadj), std::move(g.adjncy), nLevels, leafSize, numThreads);
}

PartitionResult recursiveBisectionGraph(int64_t n, std::vector<int64_t>&& xadj, std::vector<int64_t>&& adjncy,
                                        int nLevels, int64_t leafSize, int numThreads) {
    PartitionResult res;
    if (n == 0) return res;
    Csr g;
    g.xadj = std::move(xadj);
    g.adjncy = std::move(adjncy);
    std::vector<int64_t> all(static_cast<size_t>(n));
    std::iota(all.begin(), all.end(), 0);
    int threads = numThreads > 0 ? numThreads : static_cast<int>(std::thread::hardware_concurrency());
    threads = std::max(1, std::min(threads, 8));
    int parDepth = 0;                           // 2^parDepth concurrent subtrees
    while ((2 << parDepth) <= threads) ++parDepth;
    SeparatorPool pool(threads);
    std::unique_ptr<Split> root = splitRec(g, std::move(all), 0, nLevels, leafSize, pool, parDepth);
    buildTree(res.tree, *root);
    res.tree.relabelRoot();
    for (int64_t id : res.tree.postOrder()) {
        const auto& idx = res.tree.node(id).indices;
        res.perm.insert(res.perm.end(), idx.begin(), idx.end());
    }
    if (!res.tree.validate(n)) throw std::runtime_error("partition: tree validation failed");
    return res;
}

}  // namespace amls_b200
