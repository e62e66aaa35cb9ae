// Separator tree and nested-dissection partition (host side, kept on the CPU).
//
// Semantics follow the reference's SeparatorTree (src/amls/separator_tree.cpp:
// node ids in creation order, children {left, right}, post-order = children
// then self, ancestors = parent .. root) and MetisPartitioner
// (src/partition/metis_partitioner.cpp:110-179: perm[new] = old, the
// concatenation of node index lists in post-order).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace amls_b200 {

enum class NodeRole : int { Leaf = 0, Separator = 1, Root = 2 };

struct TreeNode {
    int64_t id = -1;
    NodeRole role = NodeRole::Leaf;
    std::vector<int64_t> indices;   // original row/col indices owned by the node
    std::vector<int64_t> children;  // {left, right} for separators, empty for leaves
    int64_t parent = -1;
};

class SeparatorTree {
public:
    int64_t addNode(NodeRole role, std::vector<int64_t> idx);
    void setChildren(int64_t id, int64_t l, int64_t r) { nodes_.at(id).children = {l, r}; }
    void setParent(int64_t id, int64_t p) { nodes_.at(id).parent = p; }
    int64_t nNodes() const { return static_cast<int64_t>(nodes_.size()); }
    const TreeNode& node(int64_t id) const { return nodes_.at(static_cast<size_t>(id)); }
    std::vector<int64_t> postOrder() const;
    std::vector<int64_t> ancestors(int64_t id) const;
    int64_t root() const;
    void relabelRoot();
    bool validate(int64_t nTotal) const;

private:
    std::vector<TreeNode> nodes_;
    void postOrderRec(int64_t id, std::vector<int64_t>& out) const;
};

struct PartitionResult {
    SeparatorTree tree;
    std::vector<int64_t> perm;  // perm[new] = old
};

// Recursive bisection of the graph of |K| + |M| (CSR pattern, both given),
// METIS_ComputeVertexSeparator with seed 42 at each level, stopping at
// m <= leafSize, depth >= nLevels or m < 4, or on a degenerate split.
// numThreads (0 = hardware concurrency, at most 8) bounds the concurrent
// subtrees; their METIS calls run in amls_metis_worker processes next to the
// library (in this process when the program is absent).  The tree does not
// depend on numThreads.  Throws std::runtime_error on a METIS failure.
PartitionResult recursiveBisection(int64_t n,
                                   const int64_t* kRowPtr, const int32_t* kCol,
                                   const int64_t* mRowPtr, const int32_t* mCol,
                                   int nLevels, int64_t leafSize, int numThreads = 0);
// The same from the graph of |K| + |M| without self loops (neighbour lists
// sorted), e.g. extracted on the GPU.
PartitionResult recursiveBisectionGraph(int64_t n, std::vector<int64_t>&& xadj, std::vector<int64_t>&& adjncy,
                                        int nLevels, int64_t leafSize, int numThreads = 0);

}  // namespace amls_b200
