// Sequential restatement of the reference's nested dissection (test
// infrastructure: pins the product's parallel partitioner).  It follows
// src/partition/metis_partitioner.cpp line by line: the graph of A = K + M
// through one std::unordered_set per vertex (:20-45), inducedSubgraph with
// sorted lists for every vertex set, the root's included (:48-73), and at
// every split METIS_PartGraphRecursive (2 parts, seed 42) followed by
// METIS_ComputeVertexSeparator with the same options (:80-106); the
// recursion with its stop rule and degenerate-split guard, the separator
// created before its left and right subtrees (:110-160), the root relabelled
// and perm = post-order concatenation (:161-178).  The METIS library is the
// one the CUDA toolkit ships (METIS 5 API, 64-bit idx_t), the same the
// product links.
#include <algorithm>
#include <cstdint>
#include <functional>
#include <unordered_set>
#include <vector>

extern "C" {
int METIS_SetDefaultOptions(int64_t* options);
int METIS_PartGraphRecursive(int64_t* nvtxs, int64_t* ncon, int64_t* xadj, int64_t* adjncy, int64_t* vwgt,
                             int64_t* vsize, int64_t* adjwgt, int64_t* nparts, void* tpwgts, void* ubvec,
                             int64_t* options, int64_t* objval, int64_t* part);
int METIS_ComputeVertexSeparator(int64_t* nvtxs, int64_t* xadj, int64_t* adjncy, int64_t* vwgt, int64_t* options,
                                 int64_t* sepsize, int64_t* part);
}

namespace {
constexpr int kNOptions = 40, kSeed = 8, kOk = 1;

struct Csr {
    std::vector<int64_t> xadj, adjncy;
};

struct Node {
    int role = 0;            // 0 leaf, 1 separator, 2 root
    std::vector<int64_t> idx, children;
    int64_t parent = -1;
};
}  // namespace

extern "C" int metis_seq_partition(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp,
                                   const int32_t* mc, int nLevels, int64_t leafSize, int64_t* perm, int64_t* nNodes,
                                   int64_t* parent, int32_t* role, int64_t* left, int64_t* right, int64_t* idxPtr,
                                   int64_t* idx) {
    // extractGraph (:20-45) of A = K + M (structural union)
    std::vector<std::unordered_set<int64_t>> nbr(static_cast<size_t>(n));
    for (int pass = 0; pass < 2; ++pass) {
        const int64_t* rp = pass ? mp : kp;
        const int32_t* ci = pass ? mc : kc;
        for (int64_t r = 0; r < n; ++r)
            for (int64_t e = rp[r]; e < rp[r + 1]; ++e) {
                const int64_t c = ci[e];
                if (r == c) continue;
                nbr[static_cast<size_t>(r)].insert(c);
                nbr[static_cast<size_t>(c)].insert(r);
            }
    }
    Csr g;
    g.xadj.assign(static_cast<size_t>(n) + 1, 0);
    for (int64_t i = 0; i < n; ++i) g.xadj[static_cast<size_t>(i) + 1] = g.xadj[static_cast<size_t>(i)] + static_cast<int64_t>(nbr[static_cast<size_t>(i)].size());
    g.adjncy.resize(static_cast<size_t>(g.xadj.back()));
    for (int64_t i = 0; i < n; ++i) {
        int64_t p = g.xadj[static_cast<size_t>(i)];
        for (int64_t j : nbr[static_cast<size_t>(i)]) g.adjncy[static_cast<size_t>(p++)] = j;
    }
    auto induced = [&](const std::vector<int64_t>& verts) {
        const int64_t m = static_cast<int64_t>(verts.size());
        std::vector<int64_t> localOf(static_cast<size_t>(n), -1);
        for (int64_t i = 0; i < m; ++i) localOf[static_cast<size_t>(verts[static_cast<size_t>(i)])] = i;
        Csr sub;
        sub.xadj.assign(static_cast<size_t>(m) + 1, 0);
        std::vector<int64_t> tmp;
        for (int64_t i = 0; i < m; ++i) {
            const int64_t v = verts[static_cast<size_t>(i)];
            tmp.clear();
            for (int64_t q = g.xadj[static_cast<size_t>(v)]; q < g.xadj[static_cast<size_t>(v) + 1]; ++q) {
                const int64_t u = g.adjncy[static_cast<size_t>(q)];
                if (localOf[static_cast<size_t>(u)] >= 0) tmp.push_back(localOf[static_cast<size_t>(u)]);
            }
            std::sort(tmp.begin(), tmp.end());
            sub.xadj[static_cast<size_t>(i) + 1] = sub.xadj[static_cast<size_t>(i)] + static_cast<int64_t>(tmp.size());
            sub.adjncy.insert(sub.adjncy.end(), tmp.begin(), tmp.end());
        }
        return sub;
    };
    // bisect (:80-106)
    auto bisect = [&](Csr sub, std::vector<int64_t>& part) {
        int64_t nv = static_cast<int64_t>(sub.xadj.size()) - 1, ncon = 1, nparts = 2, cut = 0, sepsize = 0;
        part.assign(static_cast<size_t>(nv), 0);
        if (nv == 0) return true;
        std::vector<int64_t> where(static_cast<size_t>(nv), 0);
        int64_t opts[kNOptions];
        METIS_SetDefaultOptions(opts);
        opts[kSeed] = 42;
        if (METIS_PartGraphRecursive(&nv, &ncon, sub.xadj.data(), sub.adjncy.data(), nullptr, nullptr, nullptr,
                                     &nparts, nullptr, nullptr, opts, &cut, where.data()) != kOk)
            return false;
        return METIS_ComputeVertexSeparator(&nv, sub.xadj.data(), sub.adjncy.data(), nullptr, opts, &sepsize,
                                            part.data()) == kOk;
    };
    std::vector<Node> tree;
    bool ok = true;
    std::function<int64_t(const std::vector<int64_t>&, int)> recurse = [&](const std::vector<int64_t>& verts,
                                                                           int depth) -> int64_t {
        const int64_t m = static_cast<int64_t>(verts.size());
        auto leaf = [&]() {
            Node nd;
            nd.idx = verts;
            tree.push_back(nd);
            return static_cast<int64_t>(tree.size()) - 1;
        };
        if (m <= leafSize || depth >= nLevels || m < 4) return leaf();
        std::vector<int64_t> part;
        if (!bisect(induced(verts), part)) {
            ok = false;
            return leaf();
        }
        std::vector<int64_t> side[2], sep;
        for (int64_t i = 0; i < m; ++i) {
            const int64_t p = part[static_cast<size_t>(i)];
            if (p == 2) sep.push_back(verts[static_cast<size_t>(i)]);
            else side[p].push_back(verts[static_cast<size_t>(i)]);
        }
        const int64_t minSide = static_cast<int64_t>(std::min(side[0].size(), side[1].size()));
        if (sep.empty() || minSide < 2) return leaf();
        Node s;
        s.role = 1;
        s.idx = sep;
        tree.push_back(s);
        const int64_t id = static_cast<int64_t>(tree.size()) - 1;
        const int64_t l = recurse(side[0], depth + 1);
        const int64_t r = recurse(side[1], depth + 1);
        tree[static_cast<size_t>(id)].children = {l, r};
        tree[static_cast<size_t>(l)].parent = id;
        tree[static_cast<size_t>(r)].parent = id;
        return id;
    };
    std::vector<int64_t> all(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) all[static_cast<size_t>(i)] = i;
    recurse(all, 0);
    if (!ok) return 1;
    for (auto& nd : tree)
        if (nd.parent < 0) nd.role = 2;          // relabelRoot
    std::vector<int64_t> order;
    std::function<void(int64_t)> post = [&](int64_t v) {
        for (int64_t c : tree[static_cast<size_t>(v)].children) post(c);
        order.push_back(v);
    };
    post(0);
    int64_t q = 0;
    for (int64_t id : order)
        for (int64_t v : tree[static_cast<size_t>(id)].idx) perm[q++] = v;
    *nNodes = static_cast<int64_t>(tree.size());
    idxPtr[0] = 0;
    int64_t t = 0;
    for (size_t i = 0; i < tree.size(); ++i) {
        parent[i] = tree[i].parent;
        role[i] = tree[i].role;
        left[i] = tree[i].children.empty() ? -1 : tree[i].children[0];
        right[i] = tree[i].children.empty() ? -1 : tree[i].children[1];
        for (int64_t v : tree[i].idx) idx[t++] = v;
        idxPtr[i + 1] = t;
    }
    return 0;
}
