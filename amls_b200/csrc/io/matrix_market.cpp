// Matrix Market input/output (host), the reference's readMatrixMarket /
// writeMatrixMarket (src/io/matrix_market.cpp:48-115): coordinate format,
// real / double / integer / pattern fields (pattern entries are 1),
// general or symmetric (the mirror of every off-diagonal entry is added),
// 1-based indices, comment and empty lines skipped, duplicate entries
// summed.  The writer emits the lower triangle of a symmetric matrix
// ("real symmetric", 17 significant digits); its size line counts the
// entries written.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "amls_b200.h"
#include "host/status.hpp"

namespace amls_b200 {

namespace {

struct Coo {
    int64_t rows = 0, cols = 0;
    std::vector<int64_t> i, j;
    std::vector<double> v;
};

Coo readCoo(const char* path) {
    std::ifstream in(path);
    if (!in) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, std::string("matrix market: cannot open ") + path);
    std::string line;
    if (!std::getline(in, line)) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: empty file");
    std::istringstream bs(line);
    std::string banner, object, format, field, symmetry;
    bs >> banner >> object >> format >> field >> symmetry;
    if (banner != "%%MatrixMarket") throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: missing banner");
    if (object != "matrix") throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: only matrix objects");
    if (format != "coordinate") throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: only coordinate format");
    if (symmetry != "symmetric" && symmetry != "general")
        throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: only symmetric / general");
    if (field != "real" && field != "double" && field != "pattern" && field != "integer")
        throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: only real / integer / pattern");
    const bool sym = symmetry == "symmetric", pattern = field == "pattern";
    Coo c;
    int64_t nnz = -1;
    c.rows = -1;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '%') continue;
        if (std::sscanf(line.c_str(), "%ld %ld %ld", &c.rows, &c.cols, &nnz) != 3)
            throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: bad size line");
        break;
    }
    if (c.rows < 0) throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: missing size line");
    c.i.reserve(static_cast<size_t>(nnz) * (sym ? 2 : 1));
    c.j.reserve(c.i.capacity());
    c.v.reserve(c.i.capacity());
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '%') continue;
        const char* p = line.c_str();
        char* e = nullptr;
        errno = 0;
        const int64_t i = std::strtoll(p, &e, 10);
        const int64_t j = std::strtoll(e, &e, 10);
        double v = 1.0;
        if (!pattern) v = std::strtod(e, &e);
        if (errno != 0 || i < 1 || j < 1 || i > c.rows || j > c.cols)
            throw AmlsError(AMLS_ERR_INVALID_ARGUMENT, "matrix market: bad entry line: " + line);
        c.i.push_back(i - 1);
        c.j.push_back(j - 1);
        c.v.push_back(v);
        if (sym && i != j) {
            c.i.push_back(j - 1);
            c.j.push_back(i - 1);
            c.v.push_back(v);
        }
    }
    return c;
}

// CSR with sorted columns and duplicates summed (setFromTriplets)
void toCsr(const Coo& c, std::vector<int64_t>& rp, std::vector<int32_t>& ci, std::vector<double>& v) {
    const int64_t n = c.rows;
    rp.assign(static_cast<size_t>(n + 1), 0);
    for (int64_t r : c.i) ++rp[static_cast<size_t>(r + 1)];
    for (int64_t r = 0; r < n; ++r) rp[static_cast<size_t>(r + 1)] += rp[static_cast<size_t>(r)];
    std::vector<int64_t> pos(rp.begin(), rp.end() - 1);
    std::vector<int32_t> cc(c.i.size());
    std::vector<double> vv(c.i.size());
    for (size_t t = 0; t < c.i.size(); ++t) {
        const int64_t q = pos[static_cast<size_t>(c.i[t])]++;
        cc[static_cast<size_t>(q)] = static_cast<int32_t>(c.j[t]);
        vv[static_cast<size_t>(q)] = c.v[t];
    }
    ci.clear();
    v.clear();
    std::vector<int64_t> out(static_cast<size_t>(n + 1), 0);
    std::vector<std::pair<int32_t, double>> row;
    for (int64_t r = 0; r < n; ++r) {
        row.clear();
        for (int64_t q = rp[static_cast<size_t>(r)]; q < rp[static_cast<size_t>(r + 1)]; ++q)
            row.push_back({cc[static_cast<size_t>(q)], vv[static_cast<size_t>(q)]});
        std::stable_sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t t = 0; t < row.size(); ++t) {
            if (!ci.empty() && static_cast<int64_t>(ci.size()) > out[static_cast<size_t>(r)] && ci.back() == row[t].first)
                v.back() += row[t].second;
            else {
                ci.push_back(row[t].first);
                v.push_back(row[t].second);
            }
        }
        out[static_cast<size_t>(r + 1)] = static_cast<int64_t>(ci.size());
    }
    rp.swap(out);
}

}  // namespace
}  // namespace amls_b200

using namespace amls_b200;

extern "C" int amls_mm_read(const char* path, int64_t* n, int64_t* nnz, int64_t* rowptr, int32_t* col,
                            double* val) {
    return guarded([&]() -> int {
        if (!path || !n || !nnz) return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_mm_read: null argument");
        const Coo c = readCoo(path);
        if (c.rows != c.cols) return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_mm_read: matrix is not square");
        std::vector<int64_t> rp;
        std::vector<int32_t> ci;
        std::vector<double> v;
        toCsr(c, rp, ci, v);
        *n = c.rows;
        *nnz = static_cast<int64_t>(ci.size());
        if (rowptr) std::memcpy(rowptr, rp.data(), sizeof(int64_t) * rp.size());
        if (col) std::memcpy(col, ci.data(), sizeof(int32_t) * ci.size());
        if (val) std::memcpy(val, v.data(), sizeof(double) * v.size());
        return AMLS_OK;
    });
}

extern "C" int amls_mm_write(const char* path, int64_t n, const int64_t* rowptr, const int32_t* col,
                             const double* val) {
    return guarded([&]() -> int {
        if (!path || n < 0 || !rowptr || !col || !val) return fail(AMLS_ERR_INVALID_ARGUMENT, "amls_mm_write: null argument");
        FILE* f = std::fopen(path, "w");
        if (!f) return fail(AMLS_ERR_INVALID_ARGUMENT, std::string("amls_mm_write: cannot write ") + path);
        int64_t lower = 0;
        for (int64_t r = 0; r < n; ++r)
            for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) lower += col[e] <= r;
        std::fprintf(f, "%%%%MatrixMarket matrix coordinate real symmetric\n");
        std::fprintf(f, "%ld %ld %ld\n", static_cast<long>(n), static_cast<long>(n), static_cast<long>(lower));
        for (int64_t r = 0; r < n; ++r)
            for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e)
                if (col[e] <= r) std::fprintf(f, "%ld %ld %.17g\n", static_cast<long>(r + 1), static_cast<long>(col[e] + 1), val[e]);
        const bool ok = std::fclose(f) == 0;
        return ok ? AMLS_OK : fail(AMLS_ERR_INVALID_ARGUMENT, "amls_mm_write: write failed");
    });
}
