// amls_solve: command-line AMLS solve on the GPU with the flags of the
// reference's amls_solve (src/apps/amls_solve.cpp:31-85):
//   amls_solve --case path:N [--consistent-mass] | --case grid:NX,NY |
//              --case grid3d:N | --K K.mtx [--M M.mtx]
//   options: --nev K --nlevels L --eta H --shift S --fixed-keep K0
//            --leaf-size S --threads T --no-recover --quiet --out FILE
//   B200 options: --device D --refine K --precision fp64|mixed --sil-mode M
// Prints the size, reduced dimension, phase times, the first ten Ritz values
// (with the closed-form reference and relative error for the generated
// cases) and the residuals of the first and last pair; --out writes
// "j theta_j" lines.  Exit code 1 on a solver error, 2 on bad usage.
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>

#include "apps/app_common.hpp"

namespace {
[[noreturn]] void usage() {
    std::cerr << "usage:\n"
                 "  amls_solve --case path:N [--consistent-mass] [options]\n"
                 "  amls_solve --case grid:NX,NY [options]\n"
                 "  amls_solve --case grid3d:N [options]\n"
                 "  amls_solve --K K.mtx [--M M.mtx] [options]\n"
                 "options: --nev K --nlevels L --eta H --shift S --fixed-keep K0\n"
                 "         --leaf-size S --threads T --no-recover --quiet --out FILE\n"
                 "         --device D --refine K --precision fp64|mixed --sil-mode -1|0|1\n";
    std::exit(2);
}
}  // namespace

int main(int argc, char** argv) {
    std::string kFile, mFile, caseType, outFile;
    int64_t caseN = 0, caseNy = 0;
    bool consistentMass = false;
    int device = 0;
    amls_options opt;
    amls_options_default(&opt);
    for (int i = 1; i < argc; ++i) {
        const std::string s = argv[i];
        auto next = [&]() -> std::string {
            if (++i >= argc) usage();
            return argv[i];
        };
        try {
            if (s == "--K") kFile = next();
            else if (s == "--M") mFile = next();
            else if (s == "--case") {
                const std::string c = next();
                const auto colon = c.find(':');
                if (colon == std::string::npos) usage();
                caseType = c.substr(0, colon);
                const std::string rest = c.substr(colon + 1);
                const auto comma = rest.find(',');
                caseN = std::stoll(rest.substr(0, comma));
                if (comma != std::string::npos) caseNy = std::stoll(rest.substr(comma + 1));
            } else if (s == "--consistent-mass") consistentMass = true;
            else if (s == "--nev") opt.nev = std::stoll(next());
            else if (s == "--nlevels") opt.nLevels = std::stoi(next());
            else if (s == "--eta") opt.thresholdFactor = std::stod(next());
            else if (s == "--shift") opt.shift = std::stod(next());
            else if (s == "--fixed-keep") opt.fixedKeep = std::stoll(next());
            else if (s == "--leaf-size") opt.leafSize = std::stoll(next());
            else if (s == "--threads") opt.numThreads = std::stoi(next());
            else if (s == "--no-recover") opt.recoverVectors = 0;
            else if (s == "--quiet") opt.verbosity = 0;
            else if (s == "--out") outFile = next();
            else if (s == "--device") device = std::stoi(next());
            else if (s == "--refine") opt.refine = std::stoi(next());
            else if (s == "--precision") {
                const std::string v = next();
                if (v == "fp64") opt.precision = AMLS_PRECISION_FP64;
                else if (v == "mixed") opt.precision = AMLS_PRECISION_MIXED;
                else usage();
            } else if (s == "--sil-mode") opt.silMode = std::stoi(next());
            else usage();
        } catch (const std::logic_error&) {
            usage();
        }
    }
    if (kFile.empty() && caseType.empty()) usage();
    app::Pencil p;
    std::vector<double> ref;
    try {
        if (!caseType.empty()) {
            if (caseType == "path") {
                p = app::pathGraph(caseN, consistentMass);
                ref = app::pathGraphSpectrum(caseN, consistentMass);
            } else if (caseType == "grid") {
                p = app::gridGraph(caseN, caseNy, 1);
                ref = app::gridGraphSpectrum(caseN, caseNy, 1);
            } else if (caseType == "grid3d") {
                p = app::gridGraph(caseN, caseN, caseN);
                ref = app::gridGraphSpectrum(caseN, caseN, caseN);
            } else {
                std::cerr << "unknown case type: " << caseType << "\n";
                usage();
            }
        } else {
            p.K = app::readMtx(kFile);
            if (!mFile.empty()) p.M = app::readMtx(mFile);
            else {
                p.M = app::identity(p.K.n);
                std::cerr << "[amls_solve] note: no M given, using the identity\n";
            }
        }
    } catch (const std::exception& e) {
        std::cerr << "[amls_solve] input failed: " << e.what() << "\n";
        return 1;
    }
    const int64_t n = p.K.n;
    const int64_t nev = std::min<int64_t>(opt.nev, n);
    std::vector<double> theta(static_cast<size_t>(std::max<int64_t>(nev, 1)));
    std::vector<double> Z(opt.recoverVectors ? static_cast<size_t>(n * nev) : 0);
    double timing[AMLS_T_SLOTS] = {0};
    int64_t pOut = 0, info[AMLS_INFO_SLOTS] = {0};
    amls_handle h = nullptr;
    if (amls_create(device, &h) != AMLS_OK) {
        std::cerr << "[amls_solve] " << amls_last_error() << "\n";
        return 1;
    }
    const int rc = amls_solve(h, n, p.K.rp.data(), p.K.ci.data(), p.K.v.data(), p.M.rp.data(), p.M.ci.data(),
                              p.M.v.data(), &opt, theta.data(), opt.recoverVectors ? Z.data() : nullptr, &pOut,
                              timing);
    if (rc != AMLS_OK) {
        std::cerr << "[amls_solve] solve failed: " << amls_last_error() << "\n";
        amls_destroy(h);
        return 1;
    }
    amls_info(h, info);
    if (!outFile.empty()) {
        std::ofstream out(outFile);
        out.precision(17);
        for (int64_t j = 0; j < nev; ++j) out << j + 1 << " " << theta[static_cast<size_t>(j)] << "\n";
    }
    std::cout.precision(10);
    std::cout << "# AMLS solve n=" << n << " nev=" << opt.nev << " p=" << pOut << " tree nodes=" << info[0] << "\n";
    const char* names[AMLS_T_SLOTS] = {"partition", "upload", "elimination", "condense", "reduced",
                                       "backtransform", "total", "device"};
    std::cout << "# timing (s): ";
    for (int t = 0; t < AMLS_T_SLOTS; ++t) std::cout << names[t] << "=" << timing[t] << " ";
    std::cout << "\n";
    for (int64_t j = 0; j < nev && j < 10; ++j) {
        std::cout << j + 1 << "\t" << theta[static_cast<size_t>(j)];
        if (static_cast<int64_t>(ref.size()) > j) {
            const double r = ref[static_cast<size_t>(j)];
            std::cout << "\tref=" << r << "\trelerr=" << std::fabs(theta[static_cast<size_t>(j)] - r) / (std::fabs(r) > 0 ? std::fabs(r) : 1.0);
        }
        std::cout << "\n";
    }
    if (nev > 10) std::cout << "... (" << nev << " values)\n";
    if (opt.recoverVectors && nev > 0)
        std::cout << "# residuals: first=" << app::residual(p, theta[0], Z.data())
                  << " last=" << app::residual(p, theta[static_cast<size_t>(nev - 1)], Z.data() + (nev - 1) * n) << "\n";
    amls_destroy(h);
    return 0;
}
