// C ABI: handle, solve and batched dense eigensolver entry points.
#include <chrono>
#include <cstring>

#include "amls_b200.h"
#include "host/engine.hpp"
#include "host/status.hpp"

using namespace amls_b200;

struct amls_handle_s {
    Engine* eng = nullptr;
};

namespace {
int checkHandle(amls_handle h) {
    if (!h || !h->eng) return fail(AMLS_ERR_INVALID_ARGUMENT, "null handle");
    return AMLS_OK;
}

int checkOptions(const amls_options* opt) {
    if (!opt) return fail(AMLS_ERR_INVALID_ARGUMENT, "null options");
    if (opt->nev <= 0) return fail(AMLS_ERR_INVALID_ARGUMENT, "nev must be positive");
    if (opt->leafSize < 1) return fail(AMLS_ERR_INVALID_ARGUMENT, "leafSize must be >= 1");
    if (opt->nLevels < 0) return fail(AMLS_ERR_INVALID_ARGUMENT, "nLevels must be >= 0");
    if (opt->silMode < -1 || opt->silMode > 1)
        return fail(AMLS_ERR_INVALID_ARGUMENT, "silMode must be -1, 0 or 1");
    return AMLS_OK;
}
}  // namespace

extern "C" int amls_create(int device, amls_handle* out) {
    return guarded([&]() -> int {
        if (!out) return fail(AMLS_ERR_INVALID_ARGUMENT, "null output handle");
        *out = nullptr;
        auto* h = new amls_handle_s;
        try {
            h->eng = new Engine(device);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return AMLS_OK;
    });
}

extern "C" int amls_destroy(amls_handle h) {
    return guarded([&]() -> int {
        if (!h) return AMLS_OK;
        delete h->eng;
        delete h;
        return AMLS_OK;
    });
}

extern "C" int amls_analyze(amls_handle h, int64_t n, const int64_t* kp, const int32_t* kc,
                            const int64_t* mp, const int32_t* mc, const amls_options* opt) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (int e = checkOptions(opt)) return e;
        if (n <= 0) return fail(AMLS_ERR_INVALID_ARGUMENT, "empty matrix");
        if (!kp || !kc || !mp || !mc) return fail(AMLS_ERR_INVALID_ARGUMENT, "null CSR array");
        h->eng->analyze(n, kp, kc, mp, mc, *opt);
        return AMLS_OK;
    });
}

extern "C" int amls_solve_values(amls_handle h, const double* kv, const double* mv,
                                 int32_t values_on_device, double* theta, double* Z,
                                 int32_t outputs_on_device, int64_t* p_out, double* timing) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!kv || !mv || !theta) return fail(AMLS_ERR_INVALID_ARGUMENT, "null argument");
        h->eng->solveValues(kv, mv, values_on_device != 0, theta, Z, outputs_on_device != 0, p_out,
                            timing);
        return AMLS_OK;
    });
}

extern "C" int amls_solve(amls_handle h, int64_t n, const int64_t* kp, const int32_t* kc,
                          const double* kv, const int64_t* mp, const int32_t* mc, const double* mv,
                          const amls_options* opt, double* theta, double* Z, int64_t* p_out,
                          double* timing) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (int e = checkOptions(opt)) return e;
        if (n <= 0) return fail(AMLS_ERR_INVALID_ARGUMENT, "empty matrix");
        if (!kp || !kc || !kv || !mp || !mc || !mv || !theta)
            return fail(AMLS_ERR_INVALID_ARGUMENT, "null argument");
        double t[AMLS_T_SLOTS] = {0};
        const auto t0 = std::chrono::steady_clock::now();
        h->eng->analyze(n, kp, kc, mp, mc, *opt);
        const auto t1 = std::chrono::steady_clock::now();
        h->eng->solveValues(kv, mv, false, theta, opt->recoverVectors ? Z : nullptr, false, p_out, t);
        t[AMLS_T_PARTITION] = std::chrono::duration<double>(t1 - t0).count();
        t[AMLS_T_TOTAL] += t[AMLS_T_PARTITION];
        if (timing) std::memcpy(timing, t, sizeof(t));
        return AMLS_OK;
    });
}

extern "C" int amls_analyze_batch(amls_handle h, int32_t batch, const int64_t* pencil_off,
                                  const int64_t* kp, const int32_t* kc, const int64_t* mp,
                                  const int32_t* mc, const amls_options* opt) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (int e = checkOptions(opt)) return e;
        if (batch < 1 || !pencil_off) return fail(AMLS_ERR_INVALID_ARGUMENT, "empty batch");
        if (pencil_off[0] != 0) return fail(AMLS_ERR_INVALID_ARGUMENT, "pencil_off[0] must be 0");
        for (int b = 0; b < batch; ++b)
            if (pencil_off[b + 1] <= pencil_off[b]) return fail(AMLS_ERR_INVALID_ARGUMENT, "empty pencil in the batch");
        if (!kp || !kc || !mp || !mc) return fail(AMLS_ERR_INVALID_ARGUMENT, "null CSR array");
        if (batch > 1 && opt->refine) return fail(AMLS_ERR_INVALID_ARGUMENT, "refinement needs a single pencil");
        h->eng->analyzeBatch(batch, pencil_off, kp, kc, mp, mc, *opt);
        return AMLS_OK;
    });
}

extern "C" int amls_solve_values_batch(amls_handle h, const double* kv, const double* mv,
                                       int32_t values_on_device, double* theta, int64_t* m, double* Z,
                                       int32_t outputs_on_device, double* timing) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!kv || !mv || !theta || !m) return fail(AMLS_ERR_INVALID_ARGUMENT, "null argument");
        h->eng->solveValues(kv, mv, values_on_device != 0, theta, Z, outputs_on_device != 0, nullptr, timing, m);
        return AMLS_OK;
    });
}

extern "C" int amls_solve_batch(amls_handle h, int32_t batch, const int64_t* pencil_off, const int64_t* kp,
                                const int32_t* kc, const double* kv, const int64_t* mp, const int32_t* mc,
                                const double* mv, const amls_options* opt, double* theta, int64_t* m,
                                double* Z, double* timing) {
    return guarded([&]() -> int {
        if (!kv || !mv || !theta || !m) return fail(AMLS_ERR_INVALID_ARGUMENT, "null argument");
        const auto t0 = std::chrono::steady_clock::now();
        if (int e = amls_analyze_batch(h, batch, pencil_off, kp, kc, mp, mc, opt)) return e;
        const auto t1 = std::chrono::steady_clock::now();
        double t[AMLS_T_SLOTS] = {0};
        h->eng->solveValues(kv, mv, false, theta, opt->recoverVectors ? Z : nullptr, false, nullptr, t, m);
        t[AMLS_T_PARTITION] = std::chrono::duration<double>(t1 - t0).count();
        t[AMLS_T_TOTAL] += t[AMLS_T_PARTITION];
        if (timing) std::memcpy(timing, t, sizeof(t));
        return AMLS_OK;
    });
}

extern "C" int amls_eliminate(amls_handle h, const double* kv, const double* mv, int32_t values_on_device) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!kv || !mv) return fail(AMLS_ERR_INVALID_ARGUMENT, "null values");
        h->eng->stageEliminate(kv, mv, values_on_device != 0);
        return AMLS_OK;
    });
}

extern "C" int amls_condense(amls_handle h, int32_t mode, int64_t k, double lambda_cut, int64_t* p) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->stageCondense(mode, static_cast<int>(k), lambda_cut, p);
        return AMLS_OK;
    });
}

extern "C" int amls_pass_modes(amls_handle h, int32_t* k_node, double* mu) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->stageModes(k_node, mu);
        return AMLS_OK;
    });
}

extern "C" int amls_reduced_eig(amls_handle h, int64_t want, int32_t vectors, double* theta, int64_t* m) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->stageReduced(static_cast<int>(want), vectors != 0, theta, m);
        return AMLS_OK;
    });
}

extern "C" int amls_backtransform(amls_handle h, double* Z, int32_t outputs_on_device, int64_t* m) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->stageBacktransform(Z, outputs_on_device != 0, m);
        return AMLS_OK;
    });
}

extern "C" int amls_refine(amls_handle h, int64_t nev, double* theta, double* Z, int32_t outputs_on_device,
                           int64_t* iters) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->stageRefine(static_cast<int>(nev), theta, Z, outputs_on_device != 0, iters);
        return AMLS_OK;
    });
}

extern "C" int amls_tree(amls_handle h, int64_t* n_nodes, int64_t* parent, int64_t* size, int32_t* level) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!h->eng->analyzed()) return fail(AMLS_ERR_INVALID_ARGUMENT, "no analysis on the handle");
        h->eng->tree(n_nodes, parent, size, level);
        return AMLS_OK;
    });
}

extern "C" int amls_hex_assemble(amls_handle h, int32_t order, int64_t nelem, int64_t nnodes, const double* coords,
                                 const int64_t* enodes, const int64_t* dofmap, const double* E, const double* rho,
                                 double nu, int64_t n, const int64_t* rowptr, const int32_t* col, double* k_val,
                                 double* m_val, int32_t outputs_on_device) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!coords || !enodes || !dofmap || !E || !rho || !rowptr || !col || !k_val || !m_val)
            return fail(AMLS_ERR_INVALID_ARGUMENT, "null argument");
        h->eng->assembleHex(order, nelem, nnodes, coords, enodes, dofmap, E, rho, nu, n, rowptr, col, k_val, m_val,
                            outputs_on_device != 0);
        return AMLS_OK;
    });
}

extern "C" int amls_info(amls_handle h, int64_t* info) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!info) return fail(AMLS_ERR_INVALID_ARGUMENT, "null info");
        for (int i = 0; i < AMLS_INFO_SLOTS; ++i) info[i] = 0;
        h->eng->info(info);
        return AMLS_OK;
    });
}

extern "C" int amls_permutation(amls_handle h, int64_t* perm) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!perm) return fail(AMLS_ERR_INVALID_ARGUMENT, "null perm");
        if (!h->eng->analyzed()) return fail(AMLS_ERR_INVALID_ARGUMENT, "no analysis on the handle");
        h->eng->permutation(perm);
        return AMLS_OK;
    });
}

extern "C" int amls_work(amls_handle h, double* work) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (!work) return fail(AMLS_ERR_INVALID_ARGUMENT, "null work");
        h->eng->work(work);
        return AMLS_OK;
    });
}

extern "C" int amls_sygvx_batched(amls_handle h, int32_t batch, const int64_t* n,
                                  const int64_t* mat_off, const double* K, const double* M,
                                  int32_t mode, int64_t il, int64_t iu, double lo, double hi,
                                  const int64_t* cap, const int64_t* w_off, double* w,
                                  const int64_t* v_off, double* V, int64_t* m) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (batch < 0 || (batch > 0 && (!n || !mat_off || !K || !M || !cap || !w_off || !w ||
                                        !v_off || !V || !m)))
            return fail(AMLS_ERR_INVALID_ARGUMENT, "null argument");
        if (mode != 0 && mode != 1) return fail(AMLS_ERR_INVALID_ARGUMENT, "mode must be 0 or 1");
        if (mode == 0 && il != 1)
            return fail(AMLS_ERR_INVALID_ARGUMENT, "index mode supports il == 1 only");
        if (mode == 1 && lo > -1e299)
            return fail(AMLS_ERR_INVALID_ARGUMENT, "interval mode supports lo = -inf only");
        h->eng->sygvxBatched(batch, n, mat_off, K, M, mode, il, iu, lo, hi, cap, w_off, w, v_off, V, m);
        return AMLS_OK;
    });
}

extern "C" int amls_set_profiling(amls_handle h, int32_t on) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->setProfiling(on != 0);
        return AMLS_OK;
    });
}

extern "C" int amls_kernel_times(amls_handle h, double* ms, int64_t* launches) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->kernelTimes(ms, launches);
        return AMLS_OK;
    });
}

extern "C" int amls_category_work(amls_handle h, double* flops, double* bytes) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        h->eng->categoryWork(flops, bytes);
        return AMLS_OK;
    });
}

extern "C" int amls_sensitivities(amls_handle h, int64_t nelem, int32_t ndofe, const int64_t* dofmap,
                                  int32_t ntypes, const int32_t* elemType,
                                  const double* Kbar, const double* Mbar, const double* weights,
                                  double gapTol, double* gE, double* gRho, double* dE, double* dRho,
                                  int32_t* simple) {
    return guarded([&]() -> int {
        if (int e = checkHandle(h)) return e;
        if (nelem <= 0 || !dofmap || !Kbar || !Mbar)
            return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_sensitivities: bad element data");
        h->eng->sensitivities(nelem, ndofe, dofmap, ntypes, elemType, Kbar, Mbar, weights, gapTol, gE,
                              gRho, dE, dRho, simple);
        return AMLS_OK;
    });
}
