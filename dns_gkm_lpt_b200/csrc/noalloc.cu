// gkm_spline_build_noalloc: the velocity-spline build for callers that cannot
// allocate device memory.
//
// Who needs it: a host program that has already given the GPU's memory to its
// own pool allocator (a cudaMalloc from a library would fail or fragment that
// pool), and a program that must not stall other streams (cudaMalloc and
// cudaFree may synchronise the whole device).  Such a caller owns the state W
// and the coefficient array and passes both in; the intermediate line-solve
// results, which the handle-based path keeps in its own allocation, live here
// in a fixed-size array compiled into the library.
//
// The array is a file-scope __device__ object: every GPU that loads this
// library holds it (kScratchBytes plus the small table block) until the
// process exits.  In host code its name only stands for the device object, it
// is not a device address, so the address is looked up once per device with
// cudaGetSymbolAddress while that device is current, and that address is what
// the kernels receive.  The solver tables are filled by a one-thread kernel on
// the caller's stream, so a call launches kernels only: no allocation and no
// host-to-device copy.  All calls share both arrays; calls that overlap on the
// GPU (on one stream or several) race, so order them on one stream or
// serialise them.
#include "gkm.h"
#include "gkm_internal.h"

#include <cstdio>
#include <mutex>
#include <vector>

namespace {

constexpr long long kScratchDoubles = 4LL * 1024 * 1024;   // 32 MiB of intermediate coefficients
constexpr int kMaxLine = 1024;                                // longest spline line (points per axis)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];
static __device__ __align__(256) double g_noalloc_tables[3 * (kMaxLine + 1)];

struct DeviceSymbols {
    double* scratch = nullptr;
    double* tables = nullptr;
};

std::mutex g_mutex;
DeviceSymbols g_symbols[kMaxDevices];

// Thomas tables of the line solves: natural dp_1 = 4, m_i = 1/dp_{i-1},
// dp_i = 4 - m_i; periodic (Sherman-Morrison, gamma = -4) dp_0 = 8,
// dp_i = b_i - m_i with b_{N-1} = 4.25 and z = B^-1 (-4, 0, .., 0, 1).
// One thread fills the table array in device memory, so a call copies nothing
// from the host; every operation is rounded on its own (no fused multiply-add),
// which gives the same values as the handle path's host-built tables.
__global__ void line_tables_kernel(int N, int periodic, double* __restrict__ t)
{
    double* mt = t;
    double* dp = t + (N + 1);
    double* z = t + 2 * (N + 1);
    for (int i = 0; i <= N; i++) mt[i] = dp[i] = z[i] = 0.0;
    if (!periodic) {
        dp[1] = 4.0;
        for (int i = 2; i <= N - 2; i++) {
            mt[i] = __ddiv_rn(1.0, dp[i - 1]);
            dp[i] = __dsub_rn(4.0, mt[i]);
        }
        return;
    }
    dp[0] = 8.0;
    for (int i = 1; i < N; i++) {
        mt[i] = __ddiv_rn(1.0, dp[i - 1]);
        dp[i] = __dsub_rn((i == N - 1) ? 4.25 : 4.0, mt[i]);
    }
    double rp = -4.0;
    z[0] = rp;
    for (int i = 1; i < N; i++) {
        const double r = (i == N - 1) ? 1.0 : 0.0;
        rp = __dsub_rn(r, __dmul_rn(mt[i], rp));
        z[i] = rp;
    }
    z[N - 1] = __ddiv_rn(z[N - 1], dp[N - 1]);
    for (int i = N - 2; i >= 0; i--) z[i] = __ddiv_rn(__dsub_rn(z[i], z[i + 1]), dp[i]);
}

// Once per device, with that device current: the device addresses of the two
// static arrays.  The first call on a device performs this lookup and the
// addresses are kept for the life of the process; they stay valid as long as
// the device's primary context does, so a caller that destroys it
// (cudaDeviceReset) must not call this entry point afterwards.
cudaError_t device_symbols(DeviceSymbols& out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceSymbols& s = g_symbols[dev];
    if (!s.scratch) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        void* q = nullptr;
        e = cudaGetSymbolAddress(&q, g_noalloc_tables);
        if (e != cudaSuccess) return e;
        s.scratch = static_cast<double*>(p);
        s.tables = static_cast<double*>(q);
    }
    out = s;
    return cudaSuccess;
}

}  // namespace

extern "C" gkm_status gkm_spline_build_noalloc(const double* W, int32_t n, int32_t spline_mode, int32_t component,
                                                double* coefs, void* stream)
{
    if (!W || !coefs || n < 4 || component < 1 || component > 3 || spline_mode < 0 || spline_mode > 1)
        return GKM_ERR_ARG;
    const int periodic = spline_mode == GKM_SPLINE_PERIODIC;
    const long long nt = (long long)n + 6;
    const long long N = periodic ? n : nt;
    const long long M = N + (periodic ? 3 : 2);
    const long long need = M * M * N;
    if (N > kMaxLine || need > kScratchDoubles) {
        std::fprintf(stderr,
                     "gkm_spline_build_noalloc: n = %d needs %lld doubles of scratch; the static buffer holds %lld "
                     "(lines up to %d points)\n",
                     n, need, kScratchDoubles, kMaxLine);
        return GKM_ERR_CONFIG;
    }
    DeviceSymbols sym;
    cudaError_t e = device_symbols(sym);
    if (e != cudaSuccess) return GKM_ERR_CUDA;

    // the periodic Sherman-Morrison denominator is a kernel argument: the host computes it with the
    // same recurrences (it only needs the scalars, nothing is copied to the device)
    double denom = 0.0;
    if (periodic) {
        std::vector<double> mt(N + 1), dp(N + 1), z(N + 1);
        gkm::spline_line_tables((int)N, periodic, mt.data(), dp.data(), z.data(), &denom);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    line_tables_kernel<<<1, 1, 0, s>>>((int)N, periodic, sym.tables);
    e = cudaGetLastError();
    if (e != cudaSuccess) return GKM_ERR_CUDA;

    gkm::FieldConst fc{};
    fc.n = n;
    fc.nt = (int)nt;
    fc.nt3 = nt * nt * nt;
    gkm::SplineGrid g{};
    g.npts = (int)N;
    g.pad = periodic ? 3 : 2;
    g.periodic = periodic;
    const long long N1 = N + 1;
    gkm::SplineTables tb{sym.tables, sym.tables + N1, sym.tables + 2 * N1, denom};
    e = gkm::launch_spline_component(W, fc, g, tb, component, coefs, sym.scratch, s);
    return e == cudaSuccess ? GKM_OK : GKM_ERR_CUDA;
}
