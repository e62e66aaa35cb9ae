// Nested-dissection partition on the host through METIS.
//
// The METIS library is the one shipped with the CUDA toolkit
// (libmetis_static.a, METIS 5 API, 64-bit idx_t established at run time by
// METIS_SetDefaultOptions filling 40 x 8 bytes).  The graph construction and
// the recursion restate src/partition/metis_partitioner.cpp:
//   * extractGraph (:20-45): adjacency of |K|+|M| without self loops, emitted
//     in the iteration order of one std::unordered_set per vertex filled in
//     the reference's insertion order (see extractGraph below);
//   * inducedSubgraph (:48-73): neighbour lists sorted;
//   * bisect (:80-106): ComputeVertexSeparator with options seed 42.  The
//     reference first calls PartGraphRecursive and never reads its result;
//     METIS re-seeds its generator from the options at the start of every
//     API call, so dropping that call leaves the separator unchanged (checked
//     on the benchmark pencils: identical permutations) and saves its time;
//   * recursion (:110-160) and perm = post-order concatenation (:168-175).
#include "tree.hpp"

#include <algorithm>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <numeric>
#include <stdexcept>
#include <unordered_set>

extern "C" {
// METIS 5 public prototypes (idx_t = int64_t in the linked library).
int METIS_SetDefaultOptions(int64_t* options);
int METIS_ComputeVertexSeparator(int64_t* nvtxs, int64_t* xadj, int64_t* adjncy, int64_t* vwgt,
                                 int64_t* options, int64_t* sepsize, int64_t* part);
}

namespace amls_b200 {

namespace {
constexpr int kMetisOk = 1;
constexpr int kMetisNOptions = 40;
constexpr int kMetisOptionSeed = 8;
std::mutex gMetisMutex;   // METIS keeps process-wide state: one call at a time

struct Csr {
    std::vector<int64_t> xadj, adjncy;
};

// Adjacency of |K| + |M| without self loops.  The reference inserts, for
// every column c in ascending order and every row r of that column, r into
// nbr[c] and c into nbr[r] (metis_partitioner.cpp:20-45).  For a symmetric
// pattern the inserts reaching one vertex's set are exactly its neighbours
// in ascending order (repeats are no-ops that leave the container
// untouched), so each set is built here from the vertex's sorted neighbour
// list - in parallel over vertices - with the same container and insertion
// sequence, hence the same iteration order with libstdc++.
Csr extractGraph(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp,
                 const int32_t* mc) {
    std::vector<int64_t> deg(static_cast<size_t>(n) + 1, 0);
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
    // neighbours of v = union of row v of K and of M (sorted merge), minus v
    auto forNeighbours = [&](int64_t v, auto&& visit) {
        int64_t a = kp[v], ae = kp[v + 1], b = mp[v], be = mp[v + 1];
        while (a < ae || b < be) {
            int64_t r;
            if (b >= be || (a < ae && kc[a] < mc[b])) r = kc[a++];
            else if (a >= ae || mc[b] < kc[a]) r = mc[b++];
            else { r = kc[a]; ++a; ++b; }
            if (r != v) visit(r);
        }
    };
    std::vector<std::vector<int64_t>> lists(static_cast<size_t>(n));
    forRange([&](int64_t b, int64_t e) {
        std::vector<int64_t> sorted;
        for (int64_t v = b; v < e; ++v) {
            sorted.clear();
            forNeighbours(v, [&](int64_t r) { sorted.push_back(r); });
            std::unordered_set<int64_t> set;
            for (int64_t r : sorted) set.insert(r);
            auto& out = lists[static_cast<size_t>(v)];
            out.assign(set.begin(), set.end());
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
    (void)deg;
    return g;
}

Csr inducedSubgraph(const Csr& g, const std::vector<int64_t>& verts, std::vector<int64_t>& localOf) {
    const int64_t m = static_cast<int64_t>(verts.size());
    localOf.assign(g.xadj.size() - 1, -1);
    for (int64_t i = 0; i < m; ++i) localOf[static_cast<size_t>(verts[static_cast<size_t>(i)])] = i;
    Csr sub;
    sub.xadj.assign(static_cast<size_t>(m) + 1, 0);
    std::vector<int64_t> tmp;
    for (int64_t i = 0; i < m; ++i) {
        const int64_t v = verts[static_cast<size_t>(i)];
        tmp.clear();
        for (int64_t p = g.xadj[static_cast<size_t>(v)]; p < g.xadj[static_cast<size_t>(v) + 1]; ++p) {
            const int64_t u = g.adjncy[static_cast<size_t>(p)];
            if (localOf[static_cast<size_t>(u)] >= 0) tmp.push_back(localOf[static_cast<size_t>(u)]);
        }
        std::sort(tmp.begin(), tmp.end());
        sub.xadj[static_cast<size_t>(i) + 1] = sub.xadj[static_cast<size_t>(i)] + static_cast<int64_t>(tmp.size());
        sub.adjncy.insert(sub.adjncy.end(), tmp.begin(), tmp.end());
    }
    return sub;
}

// part[v] in {0, 1, 2}; 2 = vertex separator.
std::vector<int64_t> bisect(Csr g) {
    const int64_t n = static_cast<int64_t>(g.xadj.size()) - 1;
    std::vector<int64_t> part(static_cast<size_t>(n), 0);
    if (n == 0) return part;
    int64_t nvtxs = n;
    int64_t opts[kMetisNOptions];
    METIS_SetDefaultOptions(opts);
    opts[kMetisOptionSeed] = 42;
    int64_t sepsize = 0;
    int rc;
    {
        std::lock_guard<std::mutex> lock(gMetisMutex);
        rc = METIS_ComputeVertexSeparator(&nvtxs, g.xadj.data(), g.adjncy.data(), nullptr, opts,
                                          &sepsize, part.data());
    }
    if (rc != kMetisOk) throw std::runtime_error("METIS_ComputeVertexSeparator failed");
    return part;
}
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

// The top kParallelDepth levels run their two halves on two threads.  The
// METIS library keeps process-wide state (its random generator), so its calls
// are serialised by a mutex: concurrent calls give different separators,
// while every call re-seeds from its own options, so the split of each
// vertex set does not depend on the order of the serialised calls.  What
// runs concurrently is the induced-subgraph construction and bookkeeping.
constexpr int kParallelDepth = 3;

std::unique_ptr<Split> splitRec(const Csr& g, std::vector<int64_t> verts, int depth, int nLevels,
                                int64_t leafSize) {
    auto out = std::make_unique<Split>();
    const int64_t m = static_cast<int64_t>(verts.size());
    if (m <= leafSize || depth >= nLevels || m < 4) {
        out->verts = std::move(verts);
        return out;
    }
    std::vector<int64_t> localOf;
    Csr sub = inducedSubgraph(g, verts, localOf);
    const std::vector<int64_t> part = bisect(std::move(sub));
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
    if (depth < kParallelDepth) {
        std::exception_ptr err;
        std::thread t([&] {
            try {
                out->left = splitRec(g, std::move(side[0]), depth + 1, nLevels, leafSize);
            } catch (...) {
                err = std::current_exception();
            }
        });
        try {
            out->right = splitRec(g, std::move(side[1]), depth + 1, nLevels, leafSize);
        } catch (...) {
            t.join();
            throw;
        }
        t.join();
        if (err) std::rethrow_exception(err);
    } else {
        out->left = splitRec(g, std::move(side[0]), depth + 1, nLevels, leafSize);
        out->right = splitRec(g, std::move(side[1]), depth + 1, nLevels, leafSize);
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
                                   int64_t leafSize) {
    PartitionResult res;
    if (n == 0) return res;
    const Csr g = extractGraph(n, kRowPtr, kCol, mRowPtr, mCol);
    std::vector<int64_t> all(static_cast<size_t>(n));
    std::iota(all.begin(), all.end(), 0);
    std::unique_ptr<Split> root = splitRec(g, std::move(all), 0, nLevels, leafSize);
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
