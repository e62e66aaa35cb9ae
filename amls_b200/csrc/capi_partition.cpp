// C ABI: host-only entry points (options, errors, partition).
#include <algorithm>
#include <cstring>
#include <vector>
#include <exception>
#include <stdexcept>
#include <string>

#include "amls_b200.h"
#include "host/status.hpp"
#include "host/tree.hpp"

namespace amls_b200 {
static thread_local std::string g_last_error;
void setLastError(const std::string& msg) { g_last_error = msg; }
const char* lastError() { return g_last_error.c_str(); }
}  // namespace amls_b200

using namespace amls_b200;

extern "C" const char* amls_last_error(void) { return lastError(); }

extern "C" int amls_options_default(amls_options* opt) {
    if (!opt) return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_options_default: null options");
    std::memset(opt, 0, sizeof(*opt));
    opt->nLevels = 6;
    opt->twoPass = 1;
    opt->leafSize = 500;
    opt->thresholdFactor = 2.0;
    opt->fixedKeep = 0;
    opt->nev = 100;
    opt->denseProjectedMax = 5000;
    opt->shift = 0.0;
    opt->numThreads = 0;
    opt->recoverVectors = 1;
    opt->verbosity = 1;
    opt->refine = 0;
    opt->refineMaxIter = 60;
    opt->refineExtra = -1;
    opt->refineTol = 1e-9;
    opt->precision = AMLS_PRECISION_FP64;
    opt->silMode = 0;
    return AMLS_OK;
}

extern "C" int amls_partition(int64_t n, const int64_t* kp, const int32_t* kc, const int64_t* mp,
                              const int32_t* mc, int32_t nLevels, int64_t leafSize, int64_t* perm,
                              int64_t* n_nodes, int64_t* parent, int32_t* role, int64_t* left,
                              int64_t* right, int64_t* idx_ptr, int64_t* idx) {
    return guarded([&]() -> int {
        if (n <= 0) return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_partition: empty matrix");
        if (!kp || !kc || !mp || !mc || !perm || !n_nodes || !parent || !role || !left || !right ||
            !idx_ptr || !idx)
            return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_partition: null argument");
        PartitionResult r = recursiveBisection(n, kp, kc, mp, mc, nLevels, leafSize);
        const int64_t N = r.tree.nNodes();
        *n_nodes = N;
        for (int64_t j = 0; j < n; ++j) perm[j] = r.perm[static_cast<size_t>(j)];
        int64_t acc = 0;
        for (int64_t i = 0; i < N; ++i) {
            const TreeNode& nd = r.tree.node(i);
            parent[i] = nd.parent;
            role[i] = static_cast<int32_t>(nd.role);
            left[i] = nd.children.empty() ? -1 : nd.children[0];
            right[i] = nd.children.empty() ? -1 : nd.children[1];
            idx_ptr[i] = acc;
            for (int64_t v : nd.indices) idx[acc++] = v;
        }
        idx_ptr[N] = acc;
        return AMLS_OK;
    });
}

// CSR pattern of an element mesh: the union of the element DOF cliques
// (free DOFs only), columns sorted.  Two calls: rowptr / col NULL sets *nnz.
extern "C" int amls_element_pattern(int64_t n, int64_t nelem, int32_t ndofe, const int64_t* dofmap, int64_t* nnz,
                                    int64_t* rowptr, int32_t* col) {
    return guarded([&]() -> int {
        if (n <= 0 || nelem < 0 || ndofe <= 0 || !dofmap || !nnz)
            return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_element_pattern: bad argument");
        std::vector<std::vector<int32_t>> rows(static_cast<size_t>(n));
        for (int64_t e = 0; e < nelem; ++e) {
            const int64_t* d = dofmap + e * ndofe;
            for (int32_t a = 0; a < ndofe; ++a) {
                if (d[a] < 0) continue;
                if (d[a] >= n) return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_element_pattern: DOF out of range");
                auto& r = rows[static_cast<size_t>(d[a])];
                for (int32_t b = 0; b < ndofe; ++b)
                    if (d[b] >= 0) r.push_back(static_cast<int32_t>(d[b]));
            }
        }
        int64_t tot = 0;
        for (auto& r : rows) {
            std::sort(r.begin(), r.end());
            r.erase(std::unique(r.begin(), r.end()), r.end());
            tot += static_cast<int64_t>(r.size());
        }
        *nnz = tot;
        if (rowptr && col) {
            int64_t q = 0;
            rowptr[0] = 0;
            for (int64_t i = 0; i < n; ++i) {
                for (int32_t c : rows[static_cast<size_t>(i)]) col[q++] = c;
                rowptr[i + 1] = q;
            }
        }
        return AMLS_OK;
    });
}
