// Shared pieces of the command-line programs amls_solve and amls_verify
// (host C++ over the C ABI): the reference's closed-form test pencils
// (src/io/case_generator.cpp:15-146), Matrix Market loading, the exact
// reference eigenvalues of src/reference/reference_solver.cpp:18-95 (dense
// generalized eigensolver for n <= 5000, else a tightly refined solve), and
// the error metrics of src/reference/error_metrics.cpp:7-50.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "amls_b200.h"

namespace app {

struct Csr {
    int64_t n = 0;
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> v;
};

struct Pencil {
    Csr K, M;
};

inline void check(int rc, const char* what) {
    if (rc != AMLS_OK) throw std::runtime_error(std::string(what) + ": " + amls_last_error());
}

// CSR from per-row (col, value) lists, columns sorted, duplicates summed
inline Csr fromRows(int64_t n, std::vector<std::vector<std::pair<int32_t, double>>>& rows) {
    Csr a;
    a.n = n;
    a.rp.assign(static_cast<size_t>(n + 1), 0);
    for (int64_t r = 0; r < n; ++r) {
        auto& row = rows[static_cast<size_t>(r)];
        std::sort(row.begin(), row.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (size_t t = 0; t < row.size(); ++t) {
            if (t > 0 && row[t].first == row[t - 1].first) {
                a.v.back() += row[t].second;
                continue;
            }
            a.ci.push_back(row[t].first);
            a.v.push_back(row[t].second);
        }
        a.rp[static_cast<size_t>(r + 1)] = static_cast<int64_t>(a.ci.size());
    }
    return a;
}

inline Csr identity(int64_t n) {
    std::vector<std::vector<std::pair<int32_t, double>>> rows(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) rows[static_cast<size_t>(i)].push_back({static_cast<int32_t>(i), 1.0});
    return fromRows(n, rows);
}

// pathGraph (case_generator.cpp:15-40): K = tridiag(-1, 2, -1), M = I or the
// consistent mass tridiag(1/6, 2/3, 1/6)
inline Pencil pathGraph(int64_t n, bool consistentMass) {
    std::vector<std::vector<std::pair<int32_t, double>>> k(static_cast<size_t>(n)), m(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        k[static_cast<size_t>(i)].push_back({static_cast<int32_t>(i), 2.0});
        m[static_cast<size_t>(i)].push_back({static_cast<int32_t>(i), consistentMass ? 2.0 / 3.0 : 1.0});
        if (i + 1 < n) {
            k[static_cast<size_t>(i)].push_back({static_cast<int32_t>(i + 1), -1.0});
            k[static_cast<size_t>(i + 1)].push_back({static_cast<int32_t>(i), -1.0});
            if (consistentMass) {
                m[static_cast<size_t>(i)].push_back({static_cast<int32_t>(i + 1), 1.0 / 6.0});
                m[static_cast<size_t>(i + 1)].push_back({static_cast<int32_t>(i), 1.0 / 6.0});
            }
        }
    }
    return {fromRows(n, k), fromRows(n, m)};
}

inline std::vector<double> pathGraphSpectrum(int64_t n, bool consistentMass) {
    std::vector<double> w;
    for (int64_t j = 1; j <= n; ++j) {
        const double th = M_PI * static_cast<double>(j) / static_cast<double>(n + 1);
        w.push_back(consistentMass ? 6.0 * (1.0 - std::cos(th)) / (2.0 + std::cos(th)) : 2.0 - 2.0 * std::cos(th));
    }
    std::sort(w.begin(), w.end());
    return w;
}

// gridGraph2d / 3d (:56-146): 5- / 7-point Laplacians, M = I
inline Pencil gridGraph(int64_t nx, int64_t ny, int64_t nz) {
    const int64_t n = nx * ny * nz;
    std::vector<std::vector<std::pair<int32_t, double>>> k(static_cast<size_t>(n));
    auto id = [&](int64_t i, int64_t j, int64_t l) { return static_cast<int32_t>((l * ny + j) * nx + i); };
    const double diag = nz > 1 ? 6.0 : 4.0;
    for (int64_t l = 0; l < nz; ++l)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                auto& row = k[static_cast<size_t>(id(i, j, l))];
                row.push_back({id(i, j, l), diag});
                if (i > 0) row.push_back({id(i - 1, j, l), -1.0});
                if (i + 1 < nx) row.push_back({id(i + 1, j, l), -1.0});
                if (j > 0) row.push_back({id(i, j - 1, l), -1.0});
                if (j + 1 < ny) row.push_back({id(i, j + 1, l), -1.0});
                if (l > 0) row.push_back({id(i, j, l - 1), -1.0});
                if (l + 1 < nz) row.push_back({id(i, j, l + 1), -1.0});
            }
    return {fromRows(n, k), identity(n)};
}

inline std::vector<double> gridGraphSpectrum(int64_t nx, int64_t ny, int64_t nz) {
    auto axis = [](int64_t m) {
        std::vector<double> a;
        for (int64_t j = 1; j <= m; ++j) a.push_back(2.0 - 2.0 * std::cos(M_PI * static_cast<double>(j) / static_cast<double>(m + 1)));
        return a;
    };
    const auto wx = axis(nx), wy = axis(ny), wz = nz > 1 ? axis(nz) : std::vector<double>{0.0};
    std::vector<double> w;
    for (double z : wz)
        for (double y : wy)
            for (double x : wx) w.push_back(x + y + z);
    std::sort(w.begin(), w.end());
    return w;
}

inline Csr readMtx(const std::string& path) {
    Csr a;
    int64_t nnz = 0;
    check(amls_mm_read(path.c_str(), &a.n, &nnz, nullptr, nullptr, nullptr), "amls_mm_read");
    a.rp.resize(static_cast<size_t>(a.n + 1));
    a.ci.resize(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    a.v.resize(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    check(amls_mm_read(path.c_str(), &a.n, &nnz, a.rp.data(), a.ci.data(), a.v.data()), "amls_mm_read");
    a.ci.resize(static_cast<size_t>(nnz));
    a.v.resize(static_cast<size_t>(nnz));
    return a;
}

inline std::vector<double> dense(const Csr& a) {
    std::vector<double> d(static_cast<size_t>(a.n * a.n), 0.0);
    for (int64_t r = 0; r < a.n; ++r)
        for (int64_t e = a.rp[static_cast<size_t>(r)]; e < a.rp[static_cast<size_t>(r + 1)]; ++e)
            d[static_cast<size_t>(r + a.ci[static_cast<size_t>(e)] * a.n)] += a.v[static_cast<size_t>(e)];
    return d;
}

// smallest nev eigenvalues: dense on the GPU for n <= 5000, else the AMLS
// solve refined in FP64 to 1e-12 (the reference switches to Spectra's
// shift-invert Lanczos above 5000, reference_solver.cpp:26-94)
inline std::vector<double> referenceEigenvalues(amls_handle h, const Pencil& p, int64_t nev) {
    const int64_t n = p.K.n;
    nev = std::min(nev, n);
    if (n <= 5000) {
        const std::vector<double> K = dense(p.K), M = dense(p.M);
        const int64_t nb = n, off = 0, cap = nev, wo = 0, vo = 0;
        std::vector<double> w(static_cast<size_t>(nev)), V(static_cast<size_t>(n * nev));
        int64_t m = 0;
        check(amls_sygvx_batched(h, 1, &nb, &off, K.data(), M.data(), 0, 1, nev, -1e300, 0.0, &cap, &wo, w.data(), &vo,
                                 V.data(), &m),
              "reference eigenvalues");
        w.resize(static_cast<size_t>(m));
        return w;
    }
    amls_options o;
    amls_options_default(&o);
    o.nev = nev;
    o.refine = 3;
    o.refineTol = 1e-12;
    o.recoverVectors = 0;
    o.verbosity = 0;
    std::vector<double> th(static_cast<size_t>(nev));
    int64_t pp = 0;
    check(amls_solve(h, n, p.K.rp.data(), p.K.ci.data(), p.K.v.data(), p.M.rp.data(), p.M.ci.data(), p.M.v.data(), &o,
                     th.data(), nullptr, &pp, nullptr),
          "reference eigenvalues");
    return th;
}

// ErrorMetrics::eigenvalueRelErr / frequencyRelErr (error_metrics.cpp:7-30)
inline double maxRelErr(const std::vector<double>& th, const std::vector<double>& ref) {
    double e = 0;
    for (size_t j = 0; j < th.size() && j < ref.size(); ++j)
        e = std::max(e, std::fabs(th[j] - ref[j]) / (std::fabs(ref[j]) > 0 ? std::fabs(ref[j]) : 1.0));
    return e;
}
inline double maxFreqErr(const std::vector<double>& th, const std::vector<double>& ref) {
    double e = 0;
    for (size_t j = 0; j < th.size() && j < ref.size(); ++j) {
        const double a = std::sqrt(std::max(th[j], 0.0)), b = std::sqrt(std::max(ref[j], 0.0));
        e = std::max(e, std::fabs(a - b) / (b > 0 ? b : 1.0));
    }
    return e;
}

// ||K x - theta M x|| / (||K||_inf ||x||) (ErrorMetrics::residual)
inline double residual(const Pencil& p, double theta, const double* x) {
    double knorm = 0, r2 = 0, x2 = 0;
    for (int64_t r = 0; r < p.K.n; ++r) {
        double rs = 0, kx = 0, mx = 0;
        for (int64_t e = p.K.rp[static_cast<size_t>(r)]; e < p.K.rp[static_cast<size_t>(r + 1)]; ++e) {
            rs += std::fabs(p.K.v[static_cast<size_t>(e)]);
            kx += p.K.v[static_cast<size_t>(e)] * x[p.K.ci[static_cast<size_t>(e)]];
        }
        for (int64_t e = p.M.rp[static_cast<size_t>(r)]; e < p.M.rp[static_cast<size_t>(r + 1)]; ++e)
            mx += p.M.v[static_cast<size_t>(e)] * x[p.M.ci[static_cast<size_t>(e)]];
        knorm = std::max(knorm, rs);
        r2 += (kx - theta * mx) * (kx - theta * mx);
        x2 += x[r] * x[r];
    }
    return std::sqrt(r2) / (knorm * std::sqrt(x2));
}

}  // namespace app
