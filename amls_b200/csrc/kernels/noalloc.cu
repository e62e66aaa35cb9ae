// Allocation-free variant of the dense generalized eigensolver.
//
// Some callers cannot call cudaMalloc at all: a host application whose own
// memory pool owns every device allocation and forbids allocations from
// outside it, or a real-time loop that must never enter the driver's
// allocator (an allocation can block on the device and take milliseconds).
// amls_sygvx_lowest_noalloc serves them: the caller passes device pointers
// for the inputs and outputs, and every intermediate (factor, reduced
// matrix, tridiagonal form, eigenvector workspace, launch tables, status
// word) lives in the file-scope device array below, of fixed size.  The
// array exists on every GPU that loads this library and stays allocated
// until the process exits.
//
// Host code may not use `g_noallocScratch` as a device address (in host code
// the name is a host-side stand-in); its device address is obtained once per
// device (per CUDA context on it) with cudaGetSymbolAddress, with that device
// current, the first time the entry point runs there.  If the context is torn
// down and created again (cudaDeviceReset), the module is loaded again and the
// array may move: the address is looked up again when the context changes.
//
// The call is synchronous: it ends by reading the status word back and
// synchronising the caller's stream.
//
// All calls share the one array and it keeps the last call's contents:
// everything that must start at zero is cleared by each call, and calls that
// overlap on the GPU (different streams, or different host threads) race on
// the array - serialise them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "amls_b200.h"
#include "kernels/launch.hpp"

namespace amls_b200 {

namespace {

constexpr int kMaxN = AMLS_NOALLOC_MAX_N;            // largest accepted order
constexpr int64_t kN2 = int64_t(kMaxN) * kMaxN;
// doubles: F, G, E (n^2 each), Y and Yt (n*k <= n^2 each), work (6 n k),
// d, e, tau, w (n each)
constexpr int64_t kScratchDoubles = 3 * kN2 + 2 * kN2 + 6 * kN2 + 4 * kMaxN;
constexpr int64_t kTableBytes = 64 * 1024;            // descriptor tables
constexpr int64_t kScratchBytes = kScratchDoubles * 8 + kTableBytes + 256;

}  // namespace

// The scratch of amls_sygvx_lowest_noalloc (see the file comment).
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

namespace {

std::mutex g_setupMutex;
struct ScratchSlot {
    void* addr = nullptr;
    unsigned long long ctxId = 0;   // context the address belongs to
};
ScratchSlot g_scratch[64];          // per device ordinal

// Unique id of the current CUDA context (cuCtxGetId through the runtime's
// driver entry points, so the library needs no link against libcuda).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
bool currentContextId(unsigned long long* id) {
    static CtxGetCurrentFn getCurrent = nullptr;
    static CtxGetIdFn getId = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getCurrent = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getId = reinterpret_cast<CtxGetIdFn>(f);
    }
    if (!getCurrent || !getId) return false;
    CUcontext c = nullptr;
    if (getCurrent(&c) != CUDA_SUCCESS || !c) return false;
    return getId(c, id) == CUDA_SUCCESS;
}

// Device address of the scratch array on the current device: looked up once
// per device and context, with that device current.
cudaError_t scratchAddress(int dev, unsigned char** out) {
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_setupMutex);
    // make the device's primary context current (and initialised)
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return e;
    unsigned long long id = 0;
    const bool haveId = currentContextId(&id);
    ScratchSlot& slot = g_scratch[dev];
    if (!slot.addr || !haveId || slot.ctxId != id) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess) return e;
        slot.addr = p;
        slot.ctxId = haveId ? id : 0;
    }
    *out = static_cast<unsigned char*>(slot.addr);
    return cudaSuccess;
}

struct TableBuilder {
    unsigned char host[kTableBytes];
    size_t used = 0;
    template <class T>
    size_t add(const T* p, size_t count) {
        size_t off = (used + 15) & ~size_t(15);
        if (off + sizeof(T) * count > sizeof(host)) return size_t(-1);
        std::memcpy(host + off, p, sizeof(T) * count);
        used = off + sizeof(T) * count;
        return off;
    }
};

}  // namespace

}  // namespace amls_b200

using namespace amls_b200;

extern "C" int amls_sygvx_lowest_noalloc(int64_t n, const double* K, const double* M, int64_t k,
                                         double* w, double* V, int64_t* m, void* stream) {
    if (n < 1 || n > kMaxN || k < 1 || k > n || !K || !M || !w || !V || !m)
        return AMLS_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return AMLS_ERR_NO_DEVICE;
    unsigned char* base = nullptr;
    if (scratchAddress(dev, &base) != cudaSuccess) return AMLS_ERR_CUDA;

    // scratch carve-up (doubles)
    double* dbl = reinterpret_cast<double*>(base);
    const int64_t n2 = n * n, nk = n * k;
    double* F = dbl;              // M, then its Cholesky factor
    double* G = F + n2;           // K L^-T
    double* E = G + n2;           // C = L^-1 K L^-T, then Householder vectors
    double* Y = E + n2;           // eigenvectors of C
    double* Yt = Y + nk;          // Y^T, then Y^T L^-1
    double* work = Yt + nk;       // inverse iteration (6 n k)
    double* d = work + 6 * nk;
    double* e = d + n;
    double* tau = e + n;
    double* wv = tau + n;
    unsigned char* tables = base + kScratchDoubles * 8;
    int* status = reinterpret_cast<int*>(base + kScratchDoubles * 8 + kTableBytes);  // [code, where, kOut]

    const int32_t ni = static_cast<int32_t>(n), ki = static_cast<int32_t>(k);
    TableBuilder tb;
    FrontDesc f{F, n, ni, ni, 0, 0};
    FrontDesc fe{E, n, ni, ni, 0, 0};
    TrsmDesc t1{F, n, G, n, ni, ni, 0, 0};            // G <- G L^-T
    TrsmDesc t2{F, n, E, n, ni, ni, 0, 0};            // E <- E L^-T
    TrsmDesc t3{F, n, Yt, k, ni, ki, 0, 1};           // Yt <- Yt L^-1
    CopyDesc c1{G, n, E, n, ni, ni};                  // E = G^T
    CopyDesc c2{Y, n, Yt, k, ni, ki};                 // Yt = Y^T
    CopyDesc c3{Yt, k, V, n, ki, ni};                 // V = Yt^T
    EigDesc ed{};
    ed.A = E;
    ed.lda = n;
    ed.d = d;
    ed.e = e;
    ed.tau = tau;
    ed.n = ni;
    ed.w = wv;
    ed.Y = Y;
    ed.ldy = n;
    ed.kcap = ki;
    ed.kOut = status + 2;
    ed.work = work;
    TileRef rowTiles[kMaxN / kTrsmRows + 1];
    int nRow = 0;
    for (int r = 0; r < ni; r += kTrsmRows) rowTiles[nRow++] = {0, r, 0, 0};
    TileRef kTiles[kMaxN / kTrsmRows + 1];
    int nK = 0;
    for (int r = 0; r < ki; r += kTrsmRows) kTiles[nK++] = {0, r, 0, 0};
    TileRef sq[(kMaxN / 32 + 1) * (kMaxN / 32 + 1)], yk[(kMaxN / 32 + 1) * (kMaxN / 32 + 1)],
        ky[(kMaxN / 32 + 1) * (kMaxN / 32 + 1)];
    int nSq = 0, nYk = 0, nKy = 0;
    for (int j = 0; j < ni; j += 32)
        for (int i = 0; i < ni; i += 32) sq[nSq++] = {0, i, j, 0};
    for (int j = 0; j < ki; j += 32)
        for (int i = 0; i < ni; i += 32) yk[nYk++] = {0, i, j, 0};
    for (int j = 0; j < ni; j += 32)
        for (int i = 0; i < ki; i += 32) ky[nKy++] = {0, i, j, 0};
    const size_t oF = tb.add(&f, 1), oFe = tb.add(&fe, 1), oT1 = tb.add(&t1, 1),
                 oT2 = tb.add(&t2, 1), oT3 = tb.add(&t3, 1), oC1 = tb.add(&c1, 1),
                 oC2 = tb.add(&c2, 1), oC3 = tb.add(&c3, 1), oE = tb.add(&ed, 1),
                 oRow = tb.add(rowTiles, nRow), oK = tb.add(kTiles, nK), oSq = tb.add(sq, nSq),
                 oYk = tb.add(yk, nYk), oKy = tb.add(ky, nKy);
    if (oKy == size_t(-1)) return AMLS_ERR_INVALID_ARGUMENT;
    auto T = [&](size_t off) { return tables + off; };

    cudaError_t err = cudaSuccess;
    auto run = [&](cudaError_t x) {
        if (err == cudaSuccess && x != cudaSuccess) err = x;
    };
    run(cudaMemcpyAsync(tables, tb.host, tb.used, cudaMemcpyHostToDevice, s));
    run(cudaMemsetAsync(status, 0, 3 * sizeof(int), s));
    run(cudaMemcpyAsync(F, M, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
    run(cudaMemcpyAsync(G, K, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
    const FrontDesc* dF = reinterpret_cast<const FrontDesc*>(T(oF));
    for (int jb = 0; jb * kCholBlock < ni; ++jb) {
        run(launchCholDiag(dF, 1, jb, status, s));
        run(launchCholPanel(dF, 1, jb, (ni + kTrsmRows - 1) / kTrsmRows, s));
    }
    run(launchTrsmRows(reinterpret_cast<const TrsmDesc*>(T(oT1)),
                       reinterpret_cast<const TileRef*>(T(oRow)), nRow, s));
    run(launchTransposeBatched(reinterpret_cast<const CopyDesc*>(T(oC1)),
                               reinterpret_cast<const TileRef*>(T(oSq)), nSq, s));
    run(launchTrsmRows(reinterpret_cast<const TrsmDesc*>(T(oT2)),
                       reinterpret_cast<const TileRef*>(T(oRow)), nRow, s));
    run(launchSymmetrize(reinterpret_cast<const FrontDesc*>(T(oFe)), 1, s));
    const EigDesc* dE = reinterpret_cast<const EigDesc*>(T(oE));
    run(launchTridiagSmall(dE, 1, s));
    run(launchBisect(dE, 1, 2, ki, 0.0, ki, status, s));
    run(launchInverseIter(dE, 1, ki, status, s));
    run(launchBackTransform(dE, 1, ki, s));
    run(launchTransposeBatched(reinterpret_cast<const CopyDesc*>(T(oC2)),
                               reinterpret_cast<const TileRef*>(T(oYk)), nYk, s));
    run(launchTrsmRows(reinterpret_cast<const TrsmDesc*>(T(oT3)),
                       reinterpret_cast<const TileRef*>(T(oK)), nK, s));
    run(launchTransposeBatched(reinterpret_cast<const CopyDesc*>(T(oC3)),
                               reinterpret_cast<const TileRef*>(T(oKy)), nKy, s));
    run(cudaMemcpyAsync(w, wv, sizeof(double) * k, cudaMemcpyDeviceToDevice, s));
    int hs[3] = {0, 0, 0};
    run(cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, s));
    run(cudaStreamSynchronize(s));
    if (err != cudaSuccess) {
        cudaGetLastError();
        return err == cudaErrorMemoryAllocation ? AMLS_ERR_OOM : AMLS_ERR_CUDA;
    }
    switch (hs[0]) {
        case kDevOk: break;
        case kDevNotSpd: return AMLS_ERR_NOT_SPD;
        case kDevIterCap: return AMLS_ERR_ITERATION;
        case kDevTimeout: return AMLS_ERR_TIMEOUT;
        default: return AMLS_ERR_NUMERIC;
    }
    *m = hs[2];
    return AMLS_OK;
}
