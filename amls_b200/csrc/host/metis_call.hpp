// One METIS vertex-separator call as the reference makes it
// (src/partition/metis_partitioner.cpp:80-106): default options, seed 42,
// METIS_ComputeVertexSeparator on a graph without self loops.  Shared by the
// in-process path (partition.cpp) and the separator worker process
// (worker/metis_worker.cpp), so both produce the same separator.
#pragma once
#include <cstdint>

extern "C" {
// METIS 5 public prototypes (idx_t = int64_t in the linked library).
int METIS_SetDefaultOptions(int64_t* options);
int METIS_ComputeVertexSeparator(int64_t* nvtxs, int64_t* xadj, int64_t* adjncy, int64_t* vwgt,
                                 int64_t* options, int64_t* sepsize, int64_t* part);
}

namespace amls_b200 {

constexpr int kMetisOk = 1;
constexpr int kMetisNOptions = 40;
constexpr int kMetisOptionSeed = 8;

// part[v] in {0, 1, 2} (2 = separator); returns the METIS status code.
inline int metisSeparator(int64_t n, int64_t* xadj, int64_t* adjncy, int64_t* part) {
    int64_t nvtxs = n;
    int64_t opts[kMetisNOptions];
    METIS_SetDefaultOptions(opts);
    opts[kMetisOptionSeed] = 42;
    int64_t sepsize = 0;
    return METIS_ComputeVertexSeparator(&nvtxs, xadj, adjncy, nullptr, opts, &sepsize, part);
}

}  // namespace amls_b200
