// amls_verify: the reference's verification sweep (src/apps/amls_verify.cpp:
// 43-279) on the GPU solver.  Suites:
//   closed  closed-form spectra: path 2000 (eta sweep), path 2000 with the
//           consistent mass, grid 64 x 64 with leafSize 1000 (eta sweep),
//           path 500 (nLevels sweep 2..6)
//   hb      Harwell-Boeing pencils bcsstk01/08/09/13 with their bcsstm mass
//           matrices from --matrices DIR (an M that is not positive definite
//           is replaced by the identity, as the reference does)
//   nd      nd3k / nd6k from --matrices DIR with M = I
// Each case passes when the largest relative eigenvalue error is <= 4 %.
// Reference eigenvalues: closed forms, else the dense GPU eigensolver for
// n <= 5000 and the FP64-refined solve above.  Writes
// OUTDIR/verify_results.csv and OUTDIR/verify_report.md.  Exit code 0 when
// every case passed.
#include <sys/stat.h>

#include <fstream>
#include <iostream>
#include <tuple>

#include "apps/app_common.hpp"

namespace {

struct Row {
    std::string caseName;
    double eta = 0;
    int nLevels = 0;
    int64_t p = 0;
    double maxRelErr = -1, maxFreqErr = -1, phase1 = 0, phase2 = 0, back = 0, partition = 0;
    bool pass = false;
};
std::vector<Row> rows;

void runCase(amls_handle h, const std::string& name, const app::Pencil& pc, const std::vector<double>& ref,
             int64_t nev, double eta, int nLevels, int64_t leafSize = 500) {
    amls_options o;
    amls_options_default(&o);
    o.nev = nev;
    o.thresholdFactor = eta;
    o.nLevels = nLevels;
    o.leafSize = leafSize;
    o.verbosity = 0;
    o.recoverVectors = 1;
    Row r;
    r.caseName = name;
    r.eta = eta;
    r.nLevels = nLevels;
    const int64_t n = pc.K.n, ne = std::min(nev, n);
    std::vector<double> th(static_cast<size_t>(ne)), Z(static_cast<size_t>(n * ne));
    double t[AMLS_T_SLOTS] = {0};
    if (amls_solve(h, n, pc.K.rp.data(), pc.K.ci.data(), pc.K.v.data(), pc.M.rp.data(), pc.M.ci.data(), pc.M.v.data(),
                   &o, th.data(), Z.data(), &r.p, t) == AMLS_OK) {
        r.maxRelErr = app::maxRelErr(th, ref);
        r.maxFreqErr = app::maxFreqErr(th, ref);
        r.phase1 = t[AMLS_T_ELIMINATION] + t[AMLS_T_CONDENSE];
        r.phase2 = t[AMLS_T_REDUCED];
        r.back = t[AMLS_T_BACKTRANSFORM];
        r.partition = t[AMLS_T_PARTITION];
        r.pass = r.maxRelErr <= 0.04;
    } else {
        std::cerr << "[verify] " << name << " eta=" << eta << " L=" << nLevels << " failed: " << amls_last_error() << "\n";
    }
    rows.push_back(r);
    std::cout << "[verify] " << name << " eta=" << eta << " L=" << nLevels << " p=" << r.p
              << " maxRelErr=" << r.maxRelErr << (r.pass ? " PASS" : " FAIL") << "\n";
}

// M numerically positive definite: positive diagonal and a Cholesky that
// succeeds (the dense GPU factorisation for n <= 5000)
bool numericallySpd(amls_handle h, const app::Csr& M) {
    for (int64_t r = 0; r < M.n; ++r) {
        bool diag = false;
        for (int64_t e = M.rp[static_cast<size_t>(r)]; e < M.rp[static_cast<size_t>(r + 1)]; ++e)
            if (M.ci[static_cast<size_t>(e)] == r) diag = M.v[static_cast<size_t>(e)] > 0;
        if (!diag) return false;
    }
    if (M.n > 5000) return true;
    const std::vector<double> Md = app::dense(M);
    std::vector<double> I(static_cast<size_t>(M.n * M.n), 0.0);
    for (int64_t i = 0; i < M.n; ++i) I[static_cast<size_t>(i + i * M.n)] = 1.0;
    const int64_t nb = M.n, off = 0, cap = 1, wo = 0, vo = 0;
    double w = 0;
    std::vector<double> V(static_cast<size_t>(M.n));
    int64_t m = 0;
    return amls_sygvx_batched(h, 1, &nb, &off, I.data(), Md.data(), 0, 1, 1, -1e300, 0.0, &cap, &wo, &w, &vo, V.data(),
                              &m) == AMLS_OK;
}

app::Pencil loadPair(amls_handle h, const std::string& k, const std::string& m, bool identityM) {
    app::Pencil p;
    p.K = app::readMtx(k);
    p.M = (!identityM && !m.empty()) ? app::readMtx(m) : app::identity(p.K.n);
    if (!numericallySpd(h, p.M)) {
        std::cout << "[verify] note: the M of " << k << " is not positive definite, using the identity\n";
        p.M = app::identity(p.K.n);
    }
    return p;
}

void writeReport(const std::string& dir) {
    mkdir(dir.c_str(), 0755);
    {
        std::ofstream csv(dir + "/verify_results.csv");
        csv << "case,eta,nLevels,p,maxRelErr,maxFreqErr,phase1_s,phase2_s,back_s,partition_s,pass\n";
        for (const auto& r : rows)
            csv << r.caseName << "," << r.eta << "," << r.nLevels << "," << r.p << "," << r.maxRelErr << ","
                << r.maxFreqErr << "," << r.phase1 << "," << r.phase2 << "," << r.back << "," << r.partition << ","
                << (r.pass ? 1 : 0) << "\n";
    }
    std::ofstream md(dir + "/verify_report.md");
    md << "# AMLS verification report\n\nAcceptance: relative eigenvalue error <= 4 % (frequency error <= 2 %).\n\n";
    md << "| case | eta | levels | p | max rel err | max freq err | phase1 (s) | pass |\n|---|---|---|---|---|---|---|---|\n";
    int pass = 0;
    for (const auto& r : rows) {
        pass += r.pass;
        md << "| " << r.caseName << " | " << r.eta << " | " << r.nLevels << " | " << r.p << " | " << r.maxRelErr
           << " | " << r.maxFreqErr << " | " << r.phase1 << " | " << (r.pass ? "yes" : "no") << " |\n";
    }
    md << "\npassed " << pass << "/" << rows.size() << ".\n";
}

}  // namespace

int main(int argc, char** argv) {
    std::string suite = "all", outdir = "verify_out", matrixDir = "tests/matrices";
    int64_t nev = 50;
    bool quick = false;
    int device = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string s = argv[i];
        auto next = [&]() -> std::string {
            if (++i >= argc) {
                std::cerr << "missing argument value\n";
                std::exit(2);
            }
            return argv[i];
        };
        if (s == "--suite") suite = next();
        else if (s == "--outdir") outdir = next();
        else if (s == "--nev") nev = std::stoll(next());
        else if (s == "--matrices") matrixDir = next();
        else if (s == "--quick") quick = true;
        else if (s == "--device") device = std::stoi(next());
        else {
            std::cerr << "unknown argument " << s << "\n";
            return 2;
        }
    }
    amls_handle h = nullptr;
    if (amls_create(device, &h) != AMLS_OK) {
        std::cerr << "[verify] " << amls_last_error() << "\n";
        return 1;
    }
    const std::vector<double> etas = quick ? std::vector<double>{2.0} : std::vector<double>{1.2, 1.5, 2.0, 3.0, 4.0};
    const std::vector<int> levels = quick ? std::vector<int>{4} : std::vector<int>{2, 3, 4, 5, 6};
    if (suite == "all" || suite == "closed") {
        {
            const auto p = app::pathGraph(2000, false);
            const auto ref = app::pathGraphSpectrum(2000, false);
            for (double eta : etas) runCase(h, "path2000", p, ref, nev, eta, 4);
        }
        {
            const auto p = app::pathGraph(2000, true);
            runCase(h, "path2000-consM", p, app::pathGraphSpectrum(2000, true), nev, 2.0, 4);
        }
        {
            const auto p = app::gridGraph(64, 64, 1);
            const auto ref = app::gridGraphSpectrum(64, 64, 1);
            for (double eta : etas) runCase(h, "grid64x64", p, ref, nev, eta, 4, 1000);
        }
        {
            const auto p = app::pathGraph(500, false);
            const auto ref = app::pathGraphSpectrum(500, false);
            for (int L : levels) runCase(h, "path500", p, ref, nev, 2.0, L);
        }
    }
    if (suite == "all" || suite == "hb") {
        const std::vector<std::tuple<std::string, std::string, std::vector<double>>> pairs = {
            {"bcsstk01/bcsstk01.mtx", "bcsstm01/bcsstm01.mtx", {}},
            {"bcsstk08/bcsstk08.mtx", "bcsstm08/bcsstm08.mtx", {}},
            {"bcsstk09/bcsstk09.mtx", "bcsstm09/bcsstm09.mtx", {2.0, 3.0, 4.0, 8.0}},
            {"bcsstk13/bcsstk13.mtx", "bcsstm13/bcsstm13.mtx", {}},
        };
        for (const auto& [k, m, etasM] : pairs) {
            try {
                const auto p = loadPair(h, matrixDir + "/" + k, matrixDir + "/" + m, false);
                const auto ref = app::referenceEigenvalues(h, p, nev);
                const auto& useEtas = !etasM.empty() ? etasM : (quick ? std::vector<double>{2.0} : etas);
                for (double eta : useEtas) runCase(h, k.substr(0, k.find('/')), p, ref, nev, eta, p.K.n > 2000 ? 4 : 3);
            } catch (const std::exception& e) {
                std::cerr << "[verify] skipping " << k << ": " << e.what() << "\n";
            }
        }
    }
    if (suite == "all" || suite == "nd") {
        const std::vector<std::string> names = quick ? std::vector<std::string>{"nd3k"}
                                                     : std::vector<std::string>{"nd3k", "nd6k"};
        for (const auto& nm : names) {
            try {
                const auto p = loadPair(h, matrixDir + "/" + nm + "/" + nm + ".mtx", "", true);
                std::cout << "[verify] " << nm << ": no M, using the identity\n";
                const auto ref = app::referenceEigenvalues(h, p, nev);
                for (double eta : (quick ? std::vector<double>{2.0} : etas)) runCase(h, nm, p, ref, nev, eta, 5);
            } catch (const std::exception& e) {
                std::cerr << "[verify] skipping " << nm << ": " << e.what() << "\n";
            }
        }
    }
    writeReport(outdir);
    int pass = 0;
    for (const auto& r : rows) pass += r.pass;
    std::cout << "[verify] done: " << pass << "/" << rows.size() << " passed; report in " << outdir << "/\n";
    amls_destroy(h);
    return pass == static_cast<int>(rows.size()) ? 0 : 1;
}
