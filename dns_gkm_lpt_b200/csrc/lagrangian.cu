// Lagrangian side of the step on sm_100a: velocity splines, tricubic
// evaluation, Heun advection and the PrintStats reductions.
//
// Reference path replaced: generateSplines (src/update.cpp:1235-1247) ->
// get_bsplinep (src/Interpolation.cpp:3-31) -> einspline; Particle::
// updatePosition / track (src/ParticleTrack.cpp:42-73); the velocity part of
// getParticleProp (:99-113); PrintStats (src/update.cpp:688-842).
//
// Splines are uniform cubic B-splines built as batched 1-D line solves along
// each axis (axis 0 = y first, then x, then z).  Two end conditions:
//   natural_ghost3: the reference's grid (nt points from -3dx+dx/2, f''=0 at
//                   both ends), coefficients c_{-1}..c_{N} (N+2 per axis);
//   periodic:       the n interior cell centres, cyclic rows, stored N+3 per
//                   axis with wrapped copies so a 4-point window never wraps.
// The line solve and the evaluation use rounding-explicit intrinsics in the
// order of the CPU oracle, so both produce the same bits.
#include "gkm_internal.h"

namespace gkm {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// One line: f (N points, stride fs) -> c (N+pad values, stride cs).
// The recurrences are sequential, but their inputs are not: the loops fetch U inputs ahead (data
// in the forward sweeps, the forward results in the backward sweeps) so that many loads are in
// flight per thread; the arithmetic and its order are unchanged.  Measured: U = 8 for the
// component-batched launches (fewer lines per component, more inputs in flight pay), U = 4 for
// the one-component launches of large grids (their lines already fill the GPU).
constexpr int kLineBatchBatched = 8, kLineBatchSingle = 4;
// the component-batched pass kernels hold six 128-thread CTAs per SM (80 registers): more lines
// in flight than the compiler's own choice (96-112 registers; 256^3 splines 1.57 -> 1.49 ms),
// where eight (64 registers) spill the fetch-ahead values
constexpr int kPassCtasPerSm = 6;

template <int U, class Src>
__device__ void line_solve(const Src& f, int N, int periodic, const SplineTables& tb, double* c, long long cs)
{
    if (!periodic) {
        const double c0 = f(0), cl = f(N - 1);
        double rp = 0.0;
        auto fwd = [&](int i, double fi) {
            double r = mul(6.0, fi);
            if (i == 1) r = sub(r, c0);
            if (i == N - 2) r = sub(r, cl);
            rp = (i == 1) ? r : sub(r, mul(tb.mt[i], rp));
            c[(long long)(i + 1) * cs] = rp;
        };
        int i = 1;
        for (; i + U - 1 <= N - 2; i += U) {
            double fv[U];
#pragma unroll
            for (int u = 0; u < U; u++) fv[u] = f(i + u);
#pragma unroll
            for (int u = 0; u < U; u++) fwd(i + u, fv[u]);
        }
        for (; i <= N - 2; i++) fwd(i, f(i));
        double x = __ddiv_rn(c[(long long)(N - 1) * cs], tb.dp[N - 2]);
        c[(long long)(N - 1) * cs] = x;
        i = N - 3;
        for (; i - U + 1 >= 1; i -= U) {
            double cv[U];
#pragma unroll
            for (int u = 0; u < U; u++) cv[u] = c[(long long)(i - u + 1) * cs];
#pragma unroll
            for (int u = 0; u < U; u++) {
                x = __ddiv_rn(sub(cv[u], x), tb.dp[i - u]);
                c[(long long)(i - u + 1) * cs] = x;
            }
        }
        for (; i >= 1; i--) {
            x = __ddiv_rn(sub(c[(long long)(i + 1) * cs], x), tb.dp[i]);
            c[(long long)(i + 1) * cs] = x;
        }
        // x now holds c_1 (or c_{N-2} when N == 3)
        const double x1 = (N - 2 >= 1) ? c[2 * cs] : cl;
        const double xl2 = (N - 2 >= 1) ? c[(long long)(N - 1) * cs] : c0;
        c[cs] = c0;
        c[(long long)N * cs] = cl;
        c[0] = sub(2.0 * c0, x1);
        c[(long long)(N + 1) * cs] = sub(2.0 * cl, xl2);
    } else {
        // y = B^-1 (6 f) stored in slots 1..N
        double rp = mul(6.0, f(0));
        c[cs] = rp;
        int i = 1;
        for (; i + U - 1 <= N - 1; i += U) {
            double fv[U];
#pragma unroll
            for (int u = 0; u < U; u++) fv[u] = f(i + u);
#pragma unroll
            for (int u = 0; u < U; u++) {
                rp = sub(mul(6.0, fv[u]), mul(tb.mt[i + u], rp));
                c[(long long)(i + u + 1) * cs] = rp;
            }
        }
        for (; i < N; i++) {
            rp = sub(mul(6.0, f(i)), mul(tb.mt[i], rp));
            c[(long long)(i + 1) * cs] = rp;
        }
        double x = __ddiv_rn(c[(long long)N * cs], tb.dp[N - 1]);
        c[(long long)N * cs] = x;
        i = N - 2;
        for (; i - U + 1 >= 0; i -= U) {
            double cv[U];
#pragma unroll
            for (int u = 0; u < U; u++) cv[u] = c[(long long)(i - u + 1) * cs];
#pragma unroll
            for (int u = 0; u < U; u++) {
                x = __ddiv_rn(sub(cv[u], x), tb.dp[i - u]);
                c[(long long)(i - u + 1) * cs] = x;
            }
        }
        for (; i >= 0; i--) {
            x = __ddiv_rn(sub(c[(long long)(i + 1) * cs], x), tb.dp[i]);
            c[(long long)(i + 1) * cs] = x;
        }
        const double fac = __ddiv_rn(add(c[cs], mul(-0.25, c[(long long)N * cs])), tb.denom);
        for (int i = 0; i < N; i++) c[(long long)(i + 1) * cs] = sub(c[(long long)(i + 1) * cs], mul(fac, tb.z[i]));
        c[0] = c[(long long)N * cs];
        c[(long long)(N + 1) * cs] = c[cs];
        c[(long long)(N + 2) * cs] = c[2 * cs];
    }
}

// line_solve with the intermediate results stored one slot lower (the forward value of point i in
// slot i, where the input of point i was), so the line may be solved in place: c may be the
// storage f reads (same stride), as long as slots N .. N+pad-1 exist past the N inputs.  The
// arithmetic and its order are those of line_solve, so the coefficients are identical.
template <int U, class Src>
__device__ void line_solve_ip(const Src& f, int N, int periodic, const SplineTables& tb, double* c, long long cs)
{
    if (!periodic) {
        const double c0 = f(0), cl = f(N - 1);
        double rp = 0.0;
        auto fwd = [&](int i, double fi) {
            double r = mul(6.0, fi);
            if (i == 1) r = sub(r, c0);
            if (i == N - 2) r = sub(r, cl);
            rp = (i == 1) ? r : sub(r, mul(tb.mt[i], rp));
            c[(long long)i * cs] = rp;
        };
        int i = 1;
        for (; i + U - 1 <= N - 2; i += U) {
            double fv[U];
#pragma unroll
            for (int u = 0; u < U; u++) fv[u] = f(i + u);
#pragma unroll
            for (int u = 0; u < U; u++) fwd(i + u, fv[u]);
        }
        for (; i <= N - 2; i++) fwd(i, f(i));
        double x = __ddiv_rn(c[(long long)(N - 2) * cs], tb.dp[N - 2]);
        c[(long long)(N - 1) * cs] = x;
        i = N - 3;
        for (; i - U + 1 >= 1; i -= U) {
            double cv[U];
#pragma unroll
            for (int u = 0; u < U; u++) cv[u] = c[(long long)(i - u) * cs];
#pragma unroll
            for (int u = 0; u < U; u++) {
                x = __ddiv_rn(sub(cv[u], x), tb.dp[i - u]);
                c[(long long)(i - u + 1) * cs] = x;
            }
        }
        for (; i >= 1; i--) {
            x = __ddiv_rn(sub(c[(long long)i * cs], x), tb.dp[i]);
            c[(long long)(i + 1) * cs] = x;
        }
        const double x1 = (N - 2 >= 1) ? c[2 * cs] : cl;
        const double xl2 = (N - 2 >= 1) ? c[(long long)(N - 1) * cs] : c0;
        c[cs] = c0;
        c[(long long)N * cs] = cl;
        c[0] = sub(2.0 * c0, x1);
        c[(long long)(N + 1) * cs] = sub(2.0 * cl, xl2);
    } else {
        double rp = mul(6.0, f(0));
        c[0] = rp;
        int i = 1;
        for (; i + U - 1 <= N - 1; i += U) {
            double fv[U];
#pragma unroll
            for (int u = 0; u < U; u++) fv[u] = f(i + u);
#pragma unroll
            for (int u = 0; u < U; u++) {
                rp = sub(mul(6.0, fv[u]), mul(tb.mt[i + u], rp));
                c[(long long)(i + u) * cs] = rp;
            }
        }
        for (; i < N; i++) {
            rp = sub(mul(6.0, f(i)), mul(tb.mt[i], rp));
            c[(long long)i * cs] = rp;
        }
        double x = __ddiv_rn(c[(long long)(N - 1) * cs], tb.dp[N - 1]);
        c[(long long)N * cs] = x;
        i = N - 2;
        for (; i - U + 1 >= 0; i -= U) {
            double cv[U];
#pragma unroll
            for (int u = 0; u < U; u++) cv[u] = c[(long long)(i - u) * cs];
#pragma unroll
            for (int u = 0; u < U; u++) {
                x = __ddiv_rn(sub(cv[u], x), tb.dp[i - u]);
                c[(long long)(i - u + 1) * cs] = x;
            }
        }
        for (; i >= 0; i--) {
            x = __ddiv_rn(sub(c[(long long)i * cs], x), tb.dp[i]);
            c[(long long)(i + 1) * cs] = x;
        }
        const double fac = __ddiv_rn(add(c[cs], mul(-0.25, c[(long long)N * cs])), tb.denom);
        for (int i = 0; i < N; i++) c[(long long)(i + 1) * cs] = sub(c[(long long)(i + 1) * cs], mul(fac, tb.z[i]));
        c[0] = c[(long long)N * cs];
        c[(long long)(N + 1) * cs] = c[cs];
        c[(long long)(N + 2) * cs] = c[2 * cs];
    }
}

// Data of a spline at ghost-layout cell idx (generateSplines, src/update.cpp:1200-1210,1239-1241):
// q = 1..3 velocity rho u_q / rho; q = kSrcDensity rho; q = kSrcPressure
// (rho (gam-1)) (rho E / rho - |u|^2 / 2); q = kSrcPlain the array itself (one nt^3 component).
constexpr int kSrcDensity = 0, kSrcPressure = 4, kSrcPlain = 5;

__device__ __forceinline__ double spline_source(const double* __restrict__ W, long long nt3, double gm1, int q,
                                                long long idx)
{
    if (q == kSrcDensity || q == kSrcPlain) return W[idx];
    const double d = W[idx];
    if (q != kSrcPressure) return __ddiv_rn(W[q * nt3 + idx], d);
    const double u = __ddiv_rn(W[nt3 + idx], d), v = __ddiv_rn(W[2 * nt3 + idx], d), w = __ddiv_rn(W[3 * nt3 + idx], d);
    const double vs = add(add(mul(u, u), mul(v, v)), mul(w, w));
    return mul(mul(d, gm1), sub(__ddiv_rn(W[4 * nt3 + idx], d), mul(0.5, vs)));
}

// pass 0: the data of source q along axis 0 (y) -> out [M0][N1][N2]; one line (i, k)
template <int U>
__device__ __forceinline__ void pass0_line(const double* __restrict__ W, const FieldConst& fc, const SplineGrid& g,
                                           const SplineTables& tb, int q, double* __restrict__ out, long long L,
                                           long long stride = 0)
{
    const int N = g.npts;
    const long long lines = stride ? stride : (long long)N * N;   // output stride along axis 0
    const long long nt3 = fc.nt3;
    const int nt = fc.nt;
    const int off = g.periodic ? 3 : 0;
    const int i = (int)(L / N), k = (int)(L - (long long)i * N);
    const long long base = (long long)(i + off) * nt + (k + off);
    const long long sj = (long long)nt * nt;
    auto f = [&](int j) { return spline_source(W, nt3, fc.gm1, q, (long long)(j + off) * sj + base); };
    line_solve<U>(f, N, g.periodic, tb, out + L, lines);
}

__global__ void spline_pass0(const double* __restrict__ W, FieldConst fc, SplineGrid g, SplineTables tb, int q,
                             double* __restrict__ out)
{
    const long long lines = (long long)g.npts * g.npts;
    for (long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x; L < lines; L += (long long)gridDim.x * blockDim.x)
        pass0_line<kLineBatchSingle>(W, fc, g, tb, q, out, L);
}

// pass 1: [M0][N1][N2] along axis 1 -> [M0][M1][N2]; one line (a, k)
template <int U>
__device__ __forceinline__ void pass1_line(const double* __restrict__ in, const SplineGrid& g, const SplineTables& tb,
                                           double* __restrict__ out, long long L)
{
    const int N = g.npts, M = N + g.pad;
    const int a = (int)(L / N), k = (int)(L - (long long)a * N);
    const double* src = in + (long long)a * N * N + k;
    auto f = [&](int i) { return src[(long long)i * N]; };
    line_solve<U>(f, N, g.periodic, tb, out + (long long)a * M * N + k, N);
}

__global__ void spline_pass1(const double* __restrict__ in, SplineGrid g, SplineTables tb, double* __restrict__ out)
{
    const long long lines = (long long)(g.npts + g.pad) * g.npts;
    for (long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x; L < lines; L += (long long)gridDim.x * blockDim.x)
        pass1_line<kLineBatchSingle>(in, g, tb, out, L);
}

// pass 2: [M0][M1][N2] along axis 2 -> [M0][M1][M2].  Lines are contiguous,
// so a thread per line would read 32 scattered addresses per warp access.
// Instead each warp owns 32 lines and moves 32-value chunks of them through
// shared memory (coalesced 256 B rows); lane j then runs line j's recurrence on
// its staged row.  The arithmetic per line is the one of line_solve, in the
// same order, so the coefficients are identical.
constexpr int kLineChunk = 32;
constexpr int kPass2Warps = 4;

// lines [L0, L0 + 32) of a pass-2 input (lines total), by one warp with its staging rows sm.
// Chunks are 32 output slots [s0, s0 + 32), holding values s0 - 1 .. s0 + 30 of the line (value i
// lands in slot i + 1): the copies out, and the backward sweep's copies back in, then cover whole
// 32-byte sectors of the output rows (2,112 bytes, a multiple of 32) instead of starting 8 bytes
// into one.
__device__ __forceinline__ void pass2_group(const double* __restrict__ in, const SplineGrid& g, const SplineTables& tb,
                                            double* __restrict__ out, long long L0, long long lines,
                                            double (*sm)[kLineChunk + 1])
{
    const int N = g.npts, M = N + g.pad;
    const int lane = threadIdx.x & 31;
    const int nl = (int)min(32LL, lines - L0);   // lines of this warp
    const long long myL = L0 + lane;
    const bool mine = lane < nl;
    // values s0 - 1 + lane of the warp's lines from the input rows (N values each)
    auto load_in = [&](int s0) {
        const int e = s0 - 1 + lane;
        if (e >= 0 && e < N)
            for (int j = 0; j < nl; j++) sm[j][lane] = in[(L0 + j) * N + e];
        __syncwarp();
    };
    // slots s0 + lane (1..N) of the warp's output rows, in and out
    auto load_out = [&](int s0) {
        const int sl = s0 + lane;
        if (sl >= 1 && sl <= N)
            for (int j = 0; j < nl; j++) sm[j][lane] = out[(L0 + j) * M + sl];
        __syncwarp();
    };
    auto store_out = [&](int s0) {
        __syncwarp();
        const int sl = s0 + lane;
        if (sl >= 1 && sl <= N)
            for (int j = 0; j < nl; j++) out[(L0 + j) * M + sl] = sm[j][lane];
        __syncwarp();
    };
    const int s_last = (N / kLineChunk) * kLineChunk;   // the chunk holding slot N
    const double* src = in + myL * N;
    double* dst = out + myL * M;
    if (!g.periodic) {
        const double c0 = mine ? src[0] : 0.0, cl = mine ? src[N - 1] : 0.0;
        // forward elimination: slot i+1 <- rp_i for i = 1..N-2 (values 0 and N-1 land in slots 1, N)
        double rp = 0.0;
        for (int s0 = 0; s0 <= s_last; s0 += kLineChunk) {
            load_in(s0);
            if (mine)
                for (int t = 0; t < kLineChunk; t++) {
                    const int i = s0 - 1 + t;
                    if (i < 1 || i > N - 2) continue;
                    double r = mul(6.0, sm[lane][t]);
                    if (i == 1) r = sub(r, c0);
                    if (i == N - 2) r = sub(r, cl);
                    rp = (i == 1) ? r : sub(r, mul(tb.mt[i], rp));
                    sm[lane][t] = rp;
                }
            store_out(s0);
        }
        // back substitution, chunks in descending order
        double x = 0.0, x1 = 0.0, xl2 = 0.0;
        for (int s0 = s_last; s0 >= 0; s0 -= kLineChunk) {
            load_out(s0);
            if (mine)
                for (int t = kLineChunk - 1; t >= 0; t--) {
                    const int i = s0 - 1 + t;
                    if (i < 1 || i > N - 2) continue;
                    x = (i == N - 2) ? __ddiv_rn(sm[lane][t], tb.dp[N - 2]) : __ddiv_rn(sub(sm[lane][t], x), tb.dp[i]);
                    sm[lane][t] = x;
                    if (i == N - 2) xl2 = x;
                    if (i == 1) x1 = x;
                }
            store_out(s0);
        }
        if (mine) {
            dst[1] = c0;
            dst[N] = cl;
            dst[0] = sub(2.0 * c0, x1);
            dst[N + 1] = sub(2.0 * cl, xl2);
        }
    } else {
        double rp = 0.0;
        for (int s0 = 0; s0 <= s_last; s0 += kLineChunk) {
            load_in(s0);
            if (mine)
                for (int t = 0; t < kLineChunk; t++) {
                    const int i = s0 - 1 + t;
                    if (i < 0 || i > N - 1) continue;
                    rp = (i == 0) ? mul(6.0, sm[lane][t]) : sub(mul(6.0, sm[lane][t]), mul(tb.mt[i], rp));
                    sm[lane][t] = rp;
                }
            store_out(s0);
        }
        double x = 0.0, x0 = 0.0, xl = 0.0;
        for (int s0 = s_last; s0 >= 0; s0 -= kLineChunk) {
            load_out(s0);
            if (mine)
                for (int t = kLineChunk - 1; t >= 0; t--) {
                    const int i = s0 - 1 + t;
                    if (i < 0 || i > N - 1) continue;
                    x = (i == N - 1) ? __ddiv_rn(sm[lane][t], tb.dp[N - 1]) : __ddiv_rn(sub(sm[lane][t], x), tb.dp[i]);
                    sm[lane][t] = x;
                    if (i == N - 1) xl = x;
                    if (i == 0) x0 = x;
                }
            store_out(s0);
        }
        const double fac = mine ? __ddiv_rn(add(x0, mul(-0.25, xl)), tb.denom) : 0.0;
        double y0 = 0.0, y1 = 0.0, yl = 0.0;
        for (int s0 = 0; s0 <= s_last; s0 += kLineChunk) {
            load_out(s0);
            if (mine)
                for (int t = 0; t < kLineChunk; t++) {
                    const int i = s0 - 1 + t;
                    if (i < 0 || i > N - 1) continue;
                    const double v = sub(sm[lane][t], mul(fac, tb.z[i]));
                    sm[lane][t] = v;
                    if (i == 0) y0 = v;
                    if (i == 1) y1 = v;
                    if (i == N - 1) yl = v;
                }
            store_out(s0);
        }
        if (mine) {
            dst[0] = yl;
            dst[N + 1] = y0;
            dst[N + 2] = y1;
        }
    }
}

__global__ void __launch_bounds__(32 * kPass2Warps) spline_pass2(const double* __restrict__ in, SplineGrid g,
                                                                 SplineTables tb, double* __restrict__ out)
{
    __shared__ double stage[kPass2Warps][32][kLineChunk + 1];
    const int M = g.npts + g.pad;
    const long long lines = (long long)M * M;
    const int warp = threadIdx.x >> 5;
    const long long nwarps = (long long)gridDim.x * kPass2Warps;
    for (long long L0 = ((long long)blockIdx.x * kPass2Warps + warp) * 32; L0 < lines; L0 += nwarps * 32)
        pass2_group(in, g, tb, out, L0, lines, stage[warp]);
}

// ---- velocity splines with FP32 coefficients: the same FP64 line solves, only the stored
// coefficients are rounded to single precision.  Pass 0 writes [M0][M1][N2] with room along axis
// 1, pass 1 solves in place there, pass 2 solves each of its lines in place and writes the rounded
// coefficients: one FP64 buffer of M^2 N values serves all three components (instead of that
// scratch plus three FP64 coefficient arrays of M^3).
__global__ void spline_pass0_room(const double* __restrict__ W, FieldConst fc, SplineGrid g, SplineTables tb, int q,
                                  double* __restrict__ out)
{
    const long long lines = (long long)g.npts * g.npts;
    const long long stride = (long long)(g.npts + g.pad) * g.npts;
    for (long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x; L < lines; L += (long long)gridDim.x * blockDim.x)
        pass0_line<kLineBatchSingle>(W, fc, g, tb, q, out, L, stride);
}

// pass 1 in place on [M0][M1][N2]: line (a, k) reads rows 0..N-1 and writes rows 0..M-1
__global__ void spline_pass1_inplace(double* buf, SplineGrid g, SplineTables tb)
{
    const int N = g.npts, M = N + g.pad;
    const long long lines = (long long)M * N;
    for (long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x; L < lines; L += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(L / N), k = (int)(L - (long long)a * N);
        double* line = buf + (long long)a * M * N + k;
        auto f = [&](int i) { return line[(long long)i * N]; };
        line_solve_ip<kLineBatchSingle>(f, N, g.periodic, tb, line, N);
    }
}

// pass 2 with FP32 output: the lines of [M0][M1][N2] along axis 2, 32 per warp through shared
// memory as pass2_group, the forward values stored in the line's own slots (slot i); natural ends:
// the backward sweep writes each solution rounded as its coefficient; periodic: the solution of
// point i goes to slot i+1 (i <= N-2; the last one stays in a register) for the correction sweep,
// which writes the rounded coefficients.  Output [M0][M1][M2] floats.
__device__ __forceinline__ void pass2_group_f32(double* in, const SplineGrid& g, const SplineTables& tb,
                                                float* __restrict__ out, long long L0, long long lines,
                                                double (*sm)[kLineChunk + 1])
{
    const int N = g.npts, M = N + g.pad;
    const int lane = threadIdx.x & 31;
    const int nl = (int)min(32LL, lines - L0);
    const long long myL = L0 + lane;
    const bool mine = lane < nl;
    auto load = [&](int k0) {
        for (int j = 0; j < nl; j++) {
            const int k = k0 + lane;
            if (k < N) sm[j][lane] = in[(L0 + j) * N + k];
        }
        __syncwarp();
    };
    // staged values of points k (k < kmax) into slots k + off of their lines
    auto store = [&](int k0, int off, int kmax) {
        __syncwarp();
        for (int j = 0; j < nl; j++) {
            const int k = k0 + lane;
            if (k < kmax) in[(L0 + j) * N + k + off] = sm[j][lane];
        }
        __syncwarp();
    };
    // staged values of slots k (kmin <= k < kmax) rounded into coefficients k + off
    auto emit = [&](int k0, int kmin, int kmax, int off) {
        __syncwarp();
        for (int j = 0; j < nl; j++) {
            const int k = k0 + lane;
            if (k >= kmin && k < kmax) out[(L0 + j) * M + k + off] = (float)sm[j][lane];
        }
        __syncwarp();
    };
    const double* src = in + myL * N;
    float* dst = out + myL * M;
    const int top = ((N - 1) / kLineChunk) * kLineChunk;
    if (!g.periodic) {
        const double c0 = mine ? src[0] : 0.0, cl = mine ? src[N - 1] : 0.0;
        double rp = 0.0;
        for (int k0 = 0; k0 < N; k0 += kLineChunk) {
            load(k0);
            if (mine)
                for (int t = 0; t < kLineChunk && k0 + t < N; t++) {
                    const int i = k0 + t;
                    if (i < 1 || i > N - 2) continue;
                    double r = mul(6.0, sm[lane][t]);
                    if (i == 1) r = sub(r, c0);
                    if (i == N - 2) r = sub(r, cl);
                    rp = (i == 1) ? r : sub(r, mul(tb.mt[i], rp));
                    sm[lane][t] = rp;
                }
            store(k0, 0, N);
        }
        double x = 0.0, x1 = 0.0, xl2 = 0.0;
        for (int k0 = top; k0 >= 0; k0 -= kLineChunk) {
            load(k0);
            if (mine)
                for (int t = kLineChunk - 1; t >= 0; t--) {
                    const int i = k0 + t;
                    if (i < 1 || i > N - 2) continue;
                    x = (i == N - 2) ? __ddiv_rn(sm[lane][t], tb.dp[N - 2]) : __ddiv_rn(sub(sm[lane][t], x), tb.dp[i]);
                    sm[lane][t] = x;
                    if (i == N - 2) xl2 = x;
                    if (i == 1) x1 = x;
                }
            emit(k0, 1, N - 1, 1);   // the solution of point i is coefficient i + 1 (1 <= i <= N-2)
        }
        if (mine) {
            dst[1] = (float)c0;
            dst[0] = (float)sub(2.0 * c0, x1);
            dst[N] = (float)cl;
            dst[N + 1] = (float)sub(2.0 * cl, xl2);
        }
    } else {
        double rp = 0.0;
        for (int k0 = 0; k0 < N; k0 += kLineChunk) {
            load(k0);
            if (mine)
                for (int t = 0; t < kLineChunk && k0 + t < N; t++) {
                    const int i = k0 + t;
                    rp = (i == 0) ? mul(6.0, sm[lane][t]) : sub(mul(6.0, sm[lane][t]), mul(tb.mt[i], rp));
                    sm[lane][t] = rp;
                }
            store(k0, 0, N);
        }
        double x = 0.0, x0 = 0.0, xl = 0.0;
        for (int k0 = top; k0 >= 0; k0 -= kLineChunk) {
            load(k0);
            if (mine)
                for (int t = kLineChunk - 1; t >= 0; t--) {
                    const int i = k0 + t;
                    if (i > N - 1) continue;
                    x = (i == N - 1) ? __ddiv_rn(sm[lane][t], tb.dp[N - 1]) : __ddiv_rn(sub(sm[lane][t], x), tb.dp[i]);
                    sm[lane][t] = x;
                    if (i == N - 1) xl = x;
                    if (i == 0) x0 = x;
                }
            store(k0, 1, N - 1);
        }
        const double fac = mine ? __ddiv_rn(add(x0, mul(-0.25, xl)), tb.denom) : 0.0;
        double y0 = 0.0, y1 = 0.0;
        for (int k0 = 0; k0 < N; k0 += kLineChunk) {
            load(k0);
            if (mine)
                for (int t = 0; t < kLineChunk && k0 + t < N; t++) {
                    const int s = k0 + t;   // slot s holds point s-1
                    if (s < 1) continue;
                    const double v = sub(sm[lane][t], mul(fac, tb.z[s - 1]));
                    sm[lane][t] = v;
                    if (s == 1) y0 = v;
                    if (s == 2) y1 = v;
                }
            emit(k0, 1, N, 0);
        }
        if (mine) {
            const double yl = sub(xl, mul(fac, tb.z[N - 1]));
            dst[N] = (float)yl;
            dst[0] = (float)yl;
            dst[N + 1] = (float)y0;
            dst[N + 2] = (float)y1;
        }
    }
}

__global__ void __launch_bounds__(32 * kPass2Warps) spline_pass2_f32(double* in, SplineGrid g, SplineTables tb,
                                                                     float* __restrict__ out)
{
    __shared__ double stage[kPass2Warps][32][kLineChunk + 1];
    const int M = g.npts + g.pad;
    const long long lines = (long long)M * M;
    const int warp = threadIdx.x >> 5;
    const long long nwarps = (long long)gridDim.x * kPass2Warps;
    for (long long L0 = ((long long)blockIdx.x * kPass2Warps + warp) * 32; L0 < lines; L0 += nwarps * 32)
        pass2_group_f32(in, g, tb, out, L0, lines, stage[warp]);
}

struct Basis {
    double w[4];
};

__device__ __forceinline__ int locate(const SplineGrid& g, double x, double& t)
{
    const double u = mul(sub(x, g.start), g.dinv);
    const double fl = floor(u);
    int i = (int)fl;
    if (g.periodic) {
        t = sub(u, fl);
        i %= g.npts;
        if (i < 0) i += g.npts;
        return i;
    }
    if (i < 0) i = 0;
    if (i > g.npts - 2) i = g.npts - 2;
    t = sub(u, (double)i);
    return i;
}

__device__ __forceinline__ Basis basis(double t)
{
    const double t2 = mul(t, t), t3 = mul(t2, t), s = sub(1.0, t);
    const double c = 1.0 / 6.0;
    Basis b;
    b.w[0] = mul(c, mul(mul(s, s), s));
    b.w[1] = mul(c, add(sub(mul(3.0, t3), mul(6.0, t2)), 4.0));
    b.w[2] = mul(c, add(add(add(mul(-3.0, t3), mul(3.0, t2)), mul(3.0, t)), 1.0));
    b.w[3] = mul(c, t3);
    return b;
}

// value of one spline at a point (the oracle's contraction order: z, then x, then y); CT is the
// type the coefficients are stored in (double, or float for the FP32 velocity splines), the
// arithmetic is FP64
template <class CT>
__device__ __forceinline__ double spline_value(const CT* __restrict__ C, const SplineGrid& g, int ia, int ib, int ic,
                                               const Basis& A, const Basis& B, const Basis& Cz)
{
    const long long M = g.npts + g.pad;
    double v = 0.0;
#pragma unroll
    for (int x = 0; x < 4; x++) {
        double bw = 0.0;
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const CT* row = C + ((long long)(ia + x) * M + (ib + y)) * M + ic;
            const double cw = add(add(add(mul(Cz.w[0], (double)row[0]), mul(Cz.w[1], (double)row[1])),
                                      mul(Cz.w[2], (double)row[2])),
                                  mul(Cz.w[3], (double)row[3]));
            bw = (y == 0) ? mul(B.w[0], cw) : add(bw, mul(B.w[y], cw));
        }
        v = add(v, mul(A.w[x], bw));
    }
    return v;
}

template <class CT>
__device__ __forceinline__ void eval3(const CT* const* coefs, const SplineGrid& g, double a, double b, double c,
                                      double out[3])
{
    double ta, tb, tc;
    const int ia = locate(g, a, ta), ib = locate(g, b, tb), ic = locate(g, c, tc);
    const Basis A = basis(ta), B = basis(tb), Cz = basis(tc);
#pragma unroll
    for (int f = 0; f < 3; f++) out[f] = spline_value<CT>(coefs[f], g, ia, ib, ic, A, B, Cz);
}

template <class CT>
struct Coefs3T {
    const CT* c[3];
};
using Coefs3 = Coefs3T<double>;

// ---------------------------------------------- values, gradients, Hessians --
// eval_UBspline_3d_d_vg / _vgl / _vgh as the CPU oracle evaluates them: basis
// weights w, first derivatives d and second derivatives h per axis, the 4x4x4
// window contracted along axis 2, then 1, then 0, every sum left to right.
struct BasisFull {
    double w[4], d[4], h[4];
};

__device__ __forceinline__ BasisFull basis_full(double t, double dinv)
{
    const double t2 = mul(t, t), t3 = mul(t2, t), s = sub(1.0, t);
    const double c = 1.0 / 6.0;
    BasisFull b;
    b.w[0] = mul(c, mul(mul(s, s), s));
    b.w[1] = mul(c, add(sub(mul(3.0, t3), mul(6.0, t2)), 4.0));
    b.w[2] = mul(c, add(add(add(mul(-3.0, t3), mul(3.0, t2)), mul(3.0, t)), 1.0));
    b.w[3] = mul(c, t3);
    b.d[0] = mul(mul(-0.5, mul(s, s)), dinv);
    b.d[1] = mul(mul(0.5, sub(mul(3.0, t2), mul(4.0, t))), dinv);
    b.d[2] = mul(mul(0.5, add(add(mul(-3.0, t2), mul(2.0, t)), 1.0)), dinv);
    b.d[3] = mul(mul(0.5, t2), dinv);
    const double d2 = mul(dinv, dinv);
    b.h[0] = mul(s, d2);
    b.h[1] = mul(sub(mul(3.0, t), 2.0), d2);
    b.h[2] = mul(add(mul(-3.0, t), 1.0), d2);
    b.h[3] = mul(t, d2);
    return b;
}

__device__ __forceinline__ double dot4(const double a[4], const double* r)
{
    return add(add(add(mul(a[0], r[0]), mul(a[1], r[1])), mul(a[2], r[2])), mul(a[3], r[3]));
}

__device__ __forceinline__ double dot4(const double a[4], double r0, double r1, double r2, double r3)
{
    return add(add(add(mul(a[0], r0), mul(a[1], r1)), mul(a[2], r2)), mul(a[3], r3));
}

struct SplineVal {
    double v, g[3], lap, h[6];   // h: 00 01 02 11 12 22
};

// WHAT 1: value + gradient; 2: + Laplacian; 3: + Hessian
template <int WHAT>
__device__ __forceinline__ SplineVal spline_eval(const double* __restrict__ C, const SplineGrid& g, double a, double b,
                                                 double c)
{
    double ta, tb, tc;
    const int ia = locate(g, a, ta), ib = locate(g, b, tb), ic = locate(g, c, tc);
    const BasisFull A = basis_full(ta, g.dinv), B = basis_full(tb, g.dinv), Z = basis_full(tc, g.dinv);
    const long long M = g.npts + g.pad;
    double v = 0, g0 = 0, g1 = 0, g2 = 0, h00 = 0, h01 = 0, h02 = 0, h11 = 0, h12 = 0, h22 = 0;
#pragma unroll
    for (int x = 0; x < 4; x++) {
        double cw[4], cd[4], ch[4];
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const double* row = C + ((long long)(ia + x) * M + (ib + y)) * M + ic;
            const double r0 = row[0], r1 = row[1], r2 = row[2], r3 = row[3];
            cw[y] = dot4(Z.w, r0, r1, r2, r3);
            cd[y] = dot4(Z.d, r0, r1, r2, r3);
            ch[y] = (WHAT >= 2) ? dot4(Z.h, r0, r1, r2, r3) : 0.0;
        }
        const double bw = dot4(B.w, cw), bd = dot4(B.d, cw), bwd = dot4(B.w, cd);
        v = add(v, mul(A.w[x], bw));
        g0 = add(g0, mul(A.d[x], bw));
        g1 = add(g1, mul(A.w[x], bd));
        g2 = add(g2, mul(A.w[x], bwd));
        if (WHAT >= 2) {
            const double bh = dot4(B.h, cw), bwh = dot4(B.w, ch);
            h00 = add(h00, mul(A.h[x], bw));
            h11 = add(h11, mul(A.w[x], bh));
            h22 = add(h22, mul(A.w[x], bwh));
        }
        if (WHAT == 3) {
            const double bdd = dot4(B.d, cd);
            h01 = add(h01, mul(A.d[x], bd));
            h02 = add(h02, mul(A.d[x], bwd));
            h12 = add(h12, mul(A.w[x], bdd));
        }
    }
    SplineVal r;
    r.v = v;
    r.g[0] = g0;
    r.g[1] = g1;
    r.g[2] = g2;
    r.lap = (WHAT == 2) ? add(add(h00, h11), h22) : 0.0;
    r.h[0] = h00;
    r.h[1] = h01;
    r.h[2] = h02;
    r.h[3] = h11;
    r.h[4] = h12;
    r.h[5] = h22;
    return r;
}

// Laplacian of a velocity spline at every spline node, written at the node's
// ghost-layout cell (generateSplines, src/update.cpp:1217-1228): node (j, i, k)
// sits at ((j - 3) dx + dx/2, ...) on the reference grid.  The reference's
// loops visit interior nodes only; its ghost nodes keep the zeros of a fresh
// allocation and are splined as zeros, which this reproduces.
__global__ void lap_nodes_kernel(const double* __restrict__ C, SplineGrid g, FieldConst fc, double* __restrict__ out)
{
    const int N = g.npts, nt = fc.nt, off = g.periodic ? 3 : 0;
    const long long total = (long long)N * N * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / ((long long)N * N)), i = (int)((e / N) % N), k = (int)(e % N);
        const int J = j + off, I = i + off, K = k + off;
        const long long o = ((long long)J * nt + I) * nt + K;
        if (J < 3 || J >= nt - 3 || I < 3 || I >= nt - 3 || K < 3 || K >= nt - 3) {
            out[o] = 0.0;
            continue;
        }
        const double hx = mul(0.5, fc.dx);
        const double y = add(mul((double)(J - 3), fc.dx), hx);
        const double x = add(mul((double)(I - 3), fc.dx), hx);
        const double z = add(mul((double)(K - 3), fc.dx), hx);
        out[o] = spline_eval<2>(C, g, y, x, z).lap;
    }
}

struct Coefs8 {
    const double* c[8];   // rho, u, v, w, p, lap u, lap v, lap w
};

// getParticleProp (src/ParticleTrack.cpp:99-113) for every particle; props is
// SoA [kPropCount][np] in the order of the property table of include/gkm.h.
__global__ void particle_props_kernel(Coefs8 cf, SplineGrid g, long long np, const double* __restrict__ py,
                                      const double* __restrict__ px, const double* __restrict__ pz,
                                      double* __restrict__ props)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        const double a = py[p], b = px[p], c = pz[p];
        double* o = props + p;
        auto put = [&](int slot, double v) { o[(long long)slot * np] = v; };
        const SplineVal d = spline_eval<1>(cf.c[0], g, a, b, c);
        put(0, d.v);
        for (int q = 0; q < 3; q++) put(1 + q, d.g[q]);
        for (int f = 0; f < 3; f++) {
            const SplineVal u = spline_eval<1>(cf.c[1 + f], g, a, b, c);
            put(4 + f, u.v);
            for (int q = 0; q < 3; q++) put(7 + 3 * f + q, u.g[q]);
        }
        const SplineVal P = spline_eval<3>(cf.c[4], g, a, b, c);
        put(16, P.v);
        for (int q = 0; q < 3; q++) put(17 + q, P.g[q]);
        const int hmap[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int q = 0; q < 9; q++) put(20 + q, P.h[hmap[q]]);
        for (int f = 0; f < 3; f++) {
            const SplineVal l = spline_eval<1>(cf.c[5 + f], g, a, b, c);
            put(29 + f, l.v);
            for (int q = 0; q < 3; q++) put(32 + 3 * f + q, l.g[q]);
        }
    }
}

// GetParticleStats (src/update.cpp:1111-1162): per-CTA sums of U.U, S_ij S_ij,
// (du/dx)^2, (du/dx)^3, (dw/dz)^2, (dw/dz)^3 over the particles (gradients are
// (d/dy, d/dx, d/dz) in the property table)
__global__ void particle_stats_kernel(const double* __restrict__ props, long long np, StatsPartial* __restrict__ part)
{
    __shared__ double red[6][32];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        auto P = [&](int slot) { return props[(long long)slot * np + p]; };
        const double U0 = P(4), U1 = P(5), U2 = P(6);
        const double dudx = P(8), dvdx = P(11), dwdx = P(14);
        const double dudy = P(7), dvdy = P(10), dwdy = P(13);
        const double dudz = P(9), dvdz = P(12), dwdz = P(15);
        acc[0] += U0 * U0 + U1 * U1 + U2 * U2;
        acc[1] += dudx * dudx + 0.5 * ((dudy + dvdx) * (dudy + dvdx)) + 0.5 * ((dudz + dwdx) * (dudz + dwdx)) +
                  0.5 * ((dwdy + dvdz) * (dwdy + dvdz)) + dvdy * dvdy + dwdz * dwdz;
        acc[2] += dudx * dudx;
        acc[3] += dudx * dudx * dudx;
        acc[4] += dwdz * dwdz;
        acc[5] += dwdz * dwdz * dwdz;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < 6; s++) {
        double v = acc[s];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[s][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 16) {
        double v = 0.0;
        if (threadIdx.x < 6)
            for (int w2 = 0; w2 < (int)(blockDim.x >> 5); w2++) v += red[threadIdx.x][w2];
        part[blockIdx.x].v[threadIdx.x] = v;
    }
}

__global__ void particle_stats_finish(const StatsPartial* __restrict__ part, int nblocks, double* __restrict__ out)
{
    const int s = threadIdx.x;
    if (s >= 6) return;
    double v = 0.0;
    for (int b = 0; b < nblocks; b++) v += part[b].v[s];
    out[s] = v;
}

template <class CT>
__global__ void particles_eval_kernel(Coefs3T<CT> cf, SplineGrid g, long long np, const double* __restrict__ py,
                                      const double* __restrict__ px, const double* __restrict__ pz,
                                      double* __restrict__ Uu, double* __restrict__ Uv, double* __restrict__ Uw)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        double U[3];
        eval3<CT>(cf.c, g, py[p], px[p], pz[p], U);
        Uu[p] = U[0];
        Uv[p] = U[1];
        Uw[p] = U[2];
    }
}

// Heun step (src/ParticleTrack.cpp:48-73): U from the previous evaluation,
// U2 from the new spline at pos + U dt (pos is (y, x, z), U is (u, v, w)),
// pos += (U + U2) dt / 2, periodic wrap, then U at the new position for the
// next step's predictor (the reference's getParticleProp at loop start).
// particle p read from src and written to dst (the same arrays, or the sorted copy and the
// particle arrays); arrays y, x, z, u, v, w
template <class CT>
__device__ __forceinline__ void heun_particle(const Coefs3T<CT>& cf, const SplineGrid& g, double dt, long long p,
                                              const ParticleArrays& src, const ParticleArrays& dst)
{
    const double twopi = 2.0 * 3.14159265358979311600;   // 2 * atan(1)*4 in double
    double pos[3] = {src.a[0][p], src.a[1][p], src.a[2][p]};
    const double U[3] = {src.a[3][p], src.a[4][p], src.a[5][p]};
    double U2[3];
    eval3<CT>(cf.c, g, add(pos[0], mul(U[1], dt)), add(pos[1], mul(U[0], dt)), add(pos[2], mul(U[2], dt)), U2);
    pos[0] = add(pos[0], mul(mul(0.5, add(U[1], U2[1])), dt));
    pos[1] = add(pos[1], mul(mul(0.5, add(U[0], U2[0])), dt));
    pos[2] = add(pos[2], mul(mul(0.5, add(U[2], U2[2])), dt));
#pragma unroll
    for (int q = 0; q < 3; q++) {
        if (pos[q] > twopi) pos[q] = fmod(pos[q], twopi);
        if (pos[q] < 0) pos[q] = sub(twopi, fmod(-pos[q], twopi));
    }
    double Un[3];
    eval3<CT>(cf.c, g, pos[0], pos[1], pos[2], Un);
    dst.a[0][p] = pos[0];
    dst.a[1][p] = pos[1];
    dst.a[2][p] = pos[2];
    dst.a[3][p] = Un[0];
    dst.a[4][p] = Un[1];
    dst.a[5][p] = Un[2];
}

// Heun step (src/ParticleTrack.cpp:48-73): U from the previous evaluation,
// U2 from the new spline at pos + U dt (pos is (y, x, z), U is (u, v, w)),
// pos += (U + U2) dt / 2, periodic wrap, then U at the new position for the
// next step's predictor (the reference's getParticleProp at loop start).
// With tag_src the particles come from the sorted copy and their tags move with them.
template <class CT>
__global__ void particles_heun_kernel(Coefs3T<CT> cf, SplineGrid g, const DevClock* __restrict__ clock, long long np,
                                      ParticleArrays src, ParticleArrays dst, const long long* __restrict__ tag_src,
                                      long long* __restrict__ tag_dst)
{
    const double dt = clock->dt;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        heun_particle<CT>(cf, g, dt, p, src, dst);
        if (tag_src) tag_dst[p] = tag_src[p];
    }
}

// ------------------------------------------------------- particle ordering --
// Particles are kept ordered by blocks of 8^3 spline cells (y-major, z fastest,
// the coefficient layout), so the 4x4x4 windows that a warp gathers overlap
// in L1/L2.  A counting sort: keys and counts, an exclusive scan of the
// counts, a scatter into the second particle arrays.  Each particle's
// arithmetic is independent of the order.
__global__ void particle_keys_kernel(SplineGrid g, int nb, long long np, ParticleArrays P, unsigned* __restrict__ keys,
                                     unsigned* __restrict__ counts)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        double t;
        const int a = locate(g, P.a[0][p], t) >> 3, b = locate(g, P.a[1][p], t) >> 3, c = locate(g, P.a[2][p], t) >> 3;
        const unsigned key = ((unsigned)a * nb + b) * nb + c;
        keys[p] = key;
        atomicAdd(&counts[key], 1u);
    }
}

constexpr int kScanChunk = 1024;   // elements per CTA of the scan (256 threads x 4)

// exclusive scan of data[0, n) in chunks of kScanChunk; chunk totals to sums (if given)
__global__ void __launch_bounds__(256) scan_chunks_kernel(unsigned* __restrict__ data, long long n,
                                                          unsigned* __restrict__ sums)
{
    __shared__ unsigned warp_tot[8];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const long long base = (long long)blockIdx.x * kScanChunk + 4LL * tid;
    unsigned v[4], run = 0;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        v[e] = (base + e < n) ? data[base + e] : 0u;
        run += v[e];
    }
    unsigned x = run;   // inclusive scan of the threads' totals within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned t = lane < 8 ? warp_tot[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < 8) warp_tot[lane] = t;
    }
    __syncthreads();
    unsigned excl = x - run + (wid ? warp_tot[wid - 1] : 0u);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        if (base + e < n) data[base + e] = excl;
        excl += v[e];
    }
    if (sums && tid == 0) sums[blockIdx.x] = warp_tot[7];
}

__global__ void scan_add_kernel(unsigned* __restrict__ data, long long n, const unsigned* __restrict__ sums)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        data[i] += sums[i / kScanChunk];
}

__global__ void particle_scatter_kernel(long long np, const unsigned* __restrict__ keys, unsigned* __restrict__ offsets,
                                        ParticleArrays src, ParticleArrays dst, const long long* __restrict__ tag_src,
                                        long long* __restrict__ tag_dst)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        const unsigned d = atomicAdd(&offsets[keys[p]], 1u);
#pragma unroll
        for (int c = 0; c < 6; c++) dst.a[c][d] = src.a[c][p];
        tag_dst[d] = tag_src[p];
    }
}

// ---------------------------------------------------------------- stats --
// PrintStats (src/update.cpp:688-842) on the device.  At a node the spline
// value equals the data (interpolation), so rho and u come from the cell; the
// gradients come from the coefficients: per axis the node weights are
// (1, 4, 1)/6 for values and (-1, 0, 1)/2 * dinv for the derivative.
template <class CT>
__device__ __forceinline__ void node_grad(const CT* __restrict__ C, long long M, int a, int b, int c, double dinv,
                                          double g[3])
{
    const double w[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
    const double d[3] = {-0.5 * dinv, 0.0, 0.5 * dinv};
    double g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
    for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = 0; y < 3; y++) {
            const CT* row = C + ((long long)(a + x) * M + (b + y)) * M + c;
            const double r0 = (double)row[0], r1 = (double)row[1], r2 = (double)row[2];
            const double cw = w[0] * r0 + w[1] * r1 + w[2] * r2;
            const double cd = d[0] * r0 + d[2] * r2;
            g0 += d[x] * w[y] * cw;
            g1 += w[x] * d[y] * cw;
            g2 += w[x] * w[y] * cd;
        }
    g[0] = g0;
    g[1] = g1;
    g[2] = g2;
}

__device__ __forceinline__ double visc(const FieldConst& fc, double T)
{
    double x = T / fc.T0;
    if (fc.visc == 1) return fc.mu0 * pow(x, 0.76);
    return fc.mu0 * pow(x, 1.5) * (fc.T0 + 110.4) / (T + 110.4);
}

__device__ __forceinline__ void cell_c2p(const double* W, long long nt3, long long idx, double gm1, double& d, double& u,
                                         double& v, double& w, double& P, double& T)
{
    d = W[idx];
    u = W[nt3 + idx] / d;
    v = W[2 * nt3 + idx] / d;
    w = W[3 * nt3 + idx] / d;
    const double vs = u * u + v * v + w * w;
    P = (d * gm1) * (W[4 * nt3 + idx] / d - 0.5 * vs);
    T = P / (287.0 * d);
}

template <int PASS, class CT>
__global__ void stats_kernel(const double* __restrict__ W, FieldConst fc, SplineGrid g, Coefs3T<CT> cf,
                             const double* __restrict__ means, StatsPartial* __restrict__ part)
{
    __shared__ double red[16][32];
    const int n = fc.n, nt = fc.nt;
    const long long nt3 = fc.nt3, total = (long long)n * n * n;
    const long long M = g.npts + g.pad;
    const int off = g.periodic ? 0 : 3;   // coefficient window start of interior cell m
    double acc[16];
#pragma unroll
    for (int s = 0; s < 16; s++) acc[s] = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / ((long long)n * n)), i = (int)((e / n) % n), k = (int)(e % n);
        const long long idx = ((long long)(j + 3) * nt + (i + 3)) * nt + (k + 3);
        double d, u, v, w, P, T;
        cell_c2p(W, nt3, idx, fc.gm1, d, u, v, w, P, T);
        if (PASS == 0) {
            double gu[3], gv[3], gw[3];
            node_grad<CT>(cf.c[0], M, j + off, i + off, k + off, g.dinv, gu);
            node_grad<CT>(cf.c[1], M, j + off, i + off, k + off, g.dinv, gv);
            node_grad<CT>(cf.c[2], M, j + off, i + off, k + off, g.dinv, gw);
            const double dudx = gu[1], dudy = gu[0], dudz = gu[2];
            const double dvdx = gv[1], dvdy = gv[0], dvdz = gv[2];
            const double dwdx = gw[1], dwdy = gw[0], dwdz = gw[2];
            const double a2 = dudx * dudx + dudy * dudy + dudz * dudz + dvdx * dvdx + dvdy * dvdy + dvdz * dvdz +
                              dwdx * dwdx + dwdy * dwdy + dwdz * dwdz;
            acc[0] += d * (u * u + v * v + w * w);                      // TKE
            acc[1] += visc(fc, T) * a2;                                 // Diss
            acc[2] += dudx * dudx + 0.5 * (dudy + dvdx) * (dudy + dvdx) + 0.5 * (dudz + dwdx) * (dudz + dwdx) +
                      0.5 * (dwdy + dvdz) * (dwdy + dvdz) + dvdy * dvdy + dwdz * dwdz;   // SijSij
            acc[3] += dudx * dudx;
            acc[4] += dudx * dudx * dudx;
            acc[5] += dudx * dudx * dudx * dudx;
            acc[6] += dvdy * dvdy;
            acc[7] += dvdy * dvdy * dvdy;
            acc[8] += dvdy * dvdy * dvdy * dvdy;
            acc[9] += dwdz * dwdz;
            acc[10] += dwdz * dwdz * dwdz;
            acc[11] += dwdz * dwdz * dwdz * dwdz;
            acc[12] += P;
            acc[13] += T;
            acc[14] += 1.0 / d;
        } else {
            acc[0] += (means[0] - P) * (means[0] - P);
            acc[1] += (means[1] - T) * (means[1] - T);
            acc[2] += (means[2] - 1.0 / d) * (means[2] - 1.0 / d);
        }
    }
    // deterministic block reduction: warp shuffles, then warp partials in fixed order
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < 16; s++) {
        double v = acc[s];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[s][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 16) {
        double v = 0.0;
        for (int w2 = 0; w2 < (int)(blockDim.x >> 5); w2++) v += red[threadIdx.x][w2];
        part[blockIdx.x].v[threadIdx.x] = v;
    }
}

// sums partials in block order (deterministic); PASS 0 also forms the means for pass 1
__global__ void stats_finish(const StatsPartial* __restrict__ part, int nblocks, double ncells, int pass,
                             double* __restrict__ out)
{
    const int s = threadIdx.x;
    if (s >= 16) return;
    double v = 0.0;
    for (int b = 0; b < nblocks; b++) v += part[b].v[s];
    if (pass == 0) out[s] = v / ncells;
    else if (s < 3) out[16 + s] = sqrt(v / ncells);
}

template <class K, class... Args>
cudaError_t grid_launch(K kernel, long long work, int threads, cudaStream_t s, Args... args)
{
    long long b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    kernel<<<(unsigned)b, threads, 0, s>>>(args...);
    return cudaGetLastError();
}

// ---- ensemble forms: one launch per pass over every member's lines / particles
__global__ void __launch_bounds__(128, kPassCtasPerSm) ensemble_pass0_kernel(const MemberDev* __restrict__ mem, const long long* __restrict__ off, int nm,
                                      int buf)
{
    const long long total = off[nm];
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
        const int m = find_member(off, nm, x);
        const MemberDev& md = mem[m];
        const long long local = x - off[m];
        const long long lines = (long long)md.grid.npts * md.grid.npts;
        const int q = (int)(local / lines);
        pass0_line<kLineBatchBatched>(md.buf[buf], md.fc, md.grid, md.tb, q + 1, md.coef[q], local - q * lines);
    }
}

__global__ void __launch_bounds__(128, kPassCtasPerSm) ensemble_pass1_kernel(const MemberDev* __restrict__ mem, const long long* __restrict__ off, int nm)
{
    const long long total = off[nm];
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
        const int m = find_member(off, nm, x);
        const MemberDev& md = mem[m];
        const long long local = x - off[m];
        const long long lines = (long long)(md.grid.npts + md.grid.pad) * md.grid.npts;
        const int q = (int)(local / lines);
        pass1_line<kLineBatchBatched>(md.coef[q], md.grid, md.tb, md.scratch[q], local - q * lines);
    }
}

__global__ void __launch_bounds__(32 * kPass2Warps, kPassCtasPerSm)
    ensemble_pass2_kernel(const MemberDev* __restrict__ mem, const long long* __restrict__ off, int nm)
{
    __shared__ double stage[kPass2Warps][32][kLineChunk + 1];
    const int warp = threadIdx.x >> 5;
    const long long total = off[nm];
    for (long long w = (long long)blockIdx.x * kPass2Warps + warp; w < total; w += (long long)gridDim.x * kPass2Warps) {
        const int m = find_member(off, nm, w);
        const MemberDev& md = mem[m];
        const long long local = w - off[m];
        const long long M = md.grid.npts + md.grid.pad;
        const long long lines = M * M, groups = (lines + 31) / 32;
        const int q = (int)(local / groups);
        pass2_group(md.scratch[q], md.grid, md.tb, md.coef[q], (local - q * groups) * 32, lines, stage[warp]);
    }
}

__global__ void ensemble_heun_kernel(const MemberDev* __restrict__ mem, const long long* __restrict__ off, int nm)
{
    const long long total = off[nm];
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
        const int m = find_member(off, nm, x);
        const MemberDev& md = mem[m];
        const Coefs3 cf{{md.coef[0], md.coef[1], md.coef[2]}};
        const ParticleArrays P{{md.P[0], md.P[1], md.P[2], md.P[3], md.P[4], md.P[5]}};
        heun_particle<double>(cf, md.grid, md.clock->dt, x - off[m], P, P);
    }
}

cudaError_t launch_pass2(const double* in, const SplineGrid& g, const SplineTables& tb, double* out, cudaStream_t s)
{
    const long long M = g.npts + g.pad;
    long long b = (M * M + 32 * kPass2Warps - 1) / (32 * kPass2Warps);
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    spline_pass2<<<(unsigned)b, 32 * kPass2Warps, 0, s>>>(in, g, tb, out);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_spline_build(const double* W, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                double* coef_u, double* coef_v, double* coef_w, double* scratch, cudaStream_t s)
{
    double* outs[3] = {coef_u, coef_v, coef_w};
    const long long N = g.npts, M = N + g.pad;
    for (int f = 0; f < 3; f++) {
        cudaError_t e = grid_launch(spline_pass0, N * N, 128, s, W, fc, g, tb, f + 1, outs[f]);
        if (e != cudaSuccess) return e;
        e = grid_launch(spline_pass1, M * N, 128, s, (const double*)outs[f], g, tb, scratch);
        if (e != cudaSuccess) return e;
        e = launch_pass2((const double*)scratch, g, tb, outs[f], s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// one velocity component (1 = u, 2 = v, 3 = w) with caller-provided scratch and tables
cudaError_t launch_spline_component(const double* W, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                    int component, double* coef, double* scratch, cudaStream_t s)
{
    const long long N = g.npts, M = N + g.pad;
    cudaError_t e = grid_launch(spline_pass0, N * N, 128, s, W, fc, g, tb, component, coef);
    if (e != cudaSuccess) return e;
    e = grid_launch(spline_pass1, M * N, 128, s, (const double*)coef, g, tb, scratch);
    if (e != cudaSuccess) return e;
    return launch_pass2((const double*)scratch, g, tb, coef, s);
}

cudaError_t launch_ensemble_splines(const MemberDev* mem, const EnsembleWork& w, const long long totals[3], int nm,
                                    int buf, cudaStream_t s)
{
    cudaError_t e = grid_launch(ensemble_pass0_kernel, totals[0], 128, s, mem, w.line0, nm, buf);
    if (e != cudaSuccess) return e;
    e = grid_launch(ensemble_pass1_kernel, totals[1], 128, s, mem, w.line1, nm);
    if (e != cudaSuccess) return e;
    long long b = (totals[2] + kPass2Warps - 1) / kPass2Warps;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    ensemble_pass2_kernel<<<(unsigned)b, 32 * kPass2Warps, 0, s>>>(mem, w.warp2, nm);
    return cudaGetLastError();
}

cudaError_t launch_ensemble_heun(const MemberDev* mem, const long long* off, int nm, long long total, cudaStream_t s)
{
    if (total <= 0) return cudaSuccess;
    return grid_launch(ensemble_heun_kernel, total, 128, s, mem, off, nm);
}

// spline of an arbitrary source (spline_source kinds) with caller scratch
cudaError_t launch_spline_source(const double* src, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                 int kind, double* coef, double* scratch, cudaStream_t s)
{
    return launch_spline_component(src, fc, g, tb, kind, coef, scratch, s);
}

cudaError_t launch_lap_nodes(const double* coef, const SplineGrid& g, const FieldConst& fc, double* out, cudaStream_t s)
{
    const long long N = g.npts;
    return grid_launch(lap_nodes_kernel, N * N * N, 128, s, coef, g, fc, out);
}

cudaError_t launch_particle_props(const double* const coefs[8], const SplineGrid& g, long long np, const double* py,
                                  const double* px, const double* pz, double* props, cudaStream_t s)
{
    if (np <= 0) return cudaSuccess;
    Coefs8 cf;
    for (int q = 0; q < 8; q++) cf.c[q] = coefs[q];
    return grid_launch(particle_props_kernel, np, 128, s, cf, g, np, py, px, pz, props);
}

cudaError_t launch_particle_stats(const double* props, long long np, StatsPartial* partials, int nblocks, double* out6,
                                  cudaStream_t s)
{
    particle_stats_kernel<<<nblocks, 256, 0, s>>>(props, np, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    particle_stats_finish<<<1, 32, 0, s>>>(partials, nblocks, out6);
    return cudaGetLastError();
}

template <class CT>
static cudaError_t particles_eval_t(const CT* const coefs[3], const SplineGrid& g, long long np, const double* py,
                                    const double* px, const double* pz, double* Uu, double* Uv, double* Uw,
                                    cudaStream_t s)
{
    if (np <= 0) return cudaSuccess;
    Coefs3T<CT> cf{{coefs[0], coefs[1], coefs[2]}};
    return grid_launch(particles_eval_kernel<CT>, np, 128, s, cf, g, np, py, px, pz, Uu, Uv, Uw);
}

cudaError_t launch_particles_eval(const double* const coefs[3], const SplineGrid& g, long long np, const double* py,
                                  const double* px, const double* pz, double* Uu, double* Uv, double* Uw,
                                  cudaStream_t s)
{
    return particles_eval_t<double>(coefs, g, np, py, px, pz, Uu, Uv, Uw, s);
}

cudaError_t launch_particles_eval(const float* const coefs[3], const SplineGrid& g, long long np, const double* py,
                                  const double* px, const double* pz, double* Uu, double* Uv, double* Uw,
                                  cudaStream_t s)
{
    return particles_eval_t<float>(coefs, g, np, py, px, pz, Uu, Uv, Uw, s);
}

template <class CT>
static cudaError_t particles_heun_t(const CT* const coefs[3], const SplineGrid& g, const DevClock* clock, long long np,
                                    const ParticleArrays& src, const ParticleArrays& dst, const long long* tag_src,
                                    long long* tag_dst, cudaStream_t s)
{
    if (np <= 0) return cudaSuccess;
    Coefs3T<CT> cf{{coefs[0], coefs[1], coefs[2]}};
    return grid_launch(particles_heun_kernel<CT>, np, 128, s, cf, g, clock, np, src, dst, tag_src, tag_dst);
}

cudaError_t launch_particles_heun(const double* const coefs[3], const SplineGrid& g, const DevClock* clock, long long np,
                                  const ParticleArrays& src, const ParticleArrays& dst, const long long* tag_src,
                                  long long* tag_dst, cudaStream_t s)
{
    return particles_heun_t<double>(coefs, g, clock, np, src, dst, tag_src, tag_dst, s);
}

cudaError_t launch_particles_heun(const float* const coefs[3], const SplineGrid& g, const DevClock* clock, long long np,
                                  const ParticleArrays& src, const ParticleArrays& dst, const long long* tag_src,
                                  long long* tag_dst, cudaStream_t s)
{
    return particles_heun_t<float>(coefs, g, clock, np, src, dst, tag_src, tag_dst, s);
}

int scan_temp_size(long long n)
{
    long long total = 0;
    for (long long m = (n + kScanChunk - 1) / kScanChunk; m > 1; m = (m + kScanChunk - 1) / kScanChunk) total += m;
    return (int)(total + 1);
}

// exclusive scan of data[0, n) in place; temp holds scan_temp_size(n) values
static cudaError_t scan_exclusive(unsigned* data, long long n, unsigned* temp, int* launches, cudaStream_t s)
{
    const long long chunks = (n + kScanChunk - 1) / kScanChunk;
    if (chunks <= 1) {
        scan_chunks_kernel<<<1, 256, 0, s>>>(data, n, nullptr);
        *launches += 1;
        return cudaGetLastError();
    }
    scan_chunks_kernel<<<(unsigned)chunks, 256, 0, s>>>(data, n, temp);
    *launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = scan_exclusive(temp, chunks, temp + chunks, launches, s);
    if (e != cudaSuccess) return e;
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    scan_add_kernel<<<(unsigned)b, 256, 0, s>>>(data, n, temp);
    *launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_particle_sort(const SplineGrid& g, long long np, const ParticleArrays& src, const ParticleArrays& dst,
                                 const long long* tag_src, long long* tag_dst, unsigned* keys, unsigned* counts,
                                 unsigned* temp, int* launches, cudaStream_t s)
{
    if (np <= 0) return cudaSuccess;
    const int nb = (g.npts + 7) / 8;
    const long long nkeys = (long long)nb * nb * nb;
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned) * (size_t)nkeys, s);
    if (e != cudaSuccess) return e;
    e = grid_launch(particle_keys_kernel, np, 256, s, g, nb, np, src, keys, counts);
    if (e != cudaSuccess) return e;
    *launches += 1;   // the memset is a copy-engine operation, not a kernel
    e = scan_exclusive(counts, nkeys, temp, launches, s);
    if (e != cudaSuccess) return e;
    return grid_launch(particle_scatter_kernel, np, 256, s, np, (const unsigned*)keys, counts, src, dst, tag_src, tag_dst);
}

template <class CT>
static cudaError_t stats_t(const double* W, const FieldConst& fc, const SplineGrid& g, const CT* const coefs[3],
                           StatsPartial* partials, int nblocks, double* out, cudaStream_t s)
{
    Coefs3T<CT> cf{{coefs[0], coefs[1], coefs[2]}};
    const double ncells = (double)fc.n * fc.n * fc.n;
    stats_kernel<0, CT><<<nblocks, 256, 0, s>>>(W, fc, g, cf, nullptr, partials);
    stats_finish<<<1, 32, 0, s>>>(partials, nblocks, ncells, 0, out);
    // means of p, T, 1/rho sit in out[12..14]
    stats_kernel<1, CT><<<nblocks, 256, 0, s>>>(W, fc, g, cf, out + 12, partials);
    stats_finish<<<1, 32, 0, s>>>(partials, nblocks, ncells, 1, out);
    return cudaGetLastError();
}

cudaError_t launch_stats(const double* W, const FieldConst& fc, const SplineGrid& g, const double* const coefs[3],
                         StatsPartial* partials, int nblocks, double* out, cudaStream_t s)
{
    return stats_t<double>(W, fc, g, coefs, partials, nblocks, out, s);
}

cudaError_t launch_stats(const double* W, const FieldConst& fc, const SplineGrid& g, const float* const coefs[3],
                         StatsPartial* partials, int nblocks, double* out, cudaStream_t s)
{
    return stats_t<float>(W, fc, g, coefs, partials, nblocks, out, s);
}

cudaError_t launch_spline_build_f32(const double* W, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                    float* coef_u, float* coef_v, float* coef_w, double* buf, cudaStream_t s)
{
    float* outs[3] = {coef_u, coef_v, coef_w};
    const long long N = g.npts, M = N + g.pad;
    for (int f = 0; f < 3; f++) {
        cudaError_t e = grid_launch(spline_pass0_room, N * N, 128, s, W, fc, g, tb, f + 1, buf);
        if (e != cudaSuccess) return e;
        e = grid_launch(spline_pass1_inplace, M * N, 128, s, buf, g, tb);
        if (e != cudaSuccess) return e;
        long long b = (M * M + 32 * kPass2Warps - 1) / (32 * kPass2Warps);
        if (b < 1) b = 1;
        if (b > 148 * 16) b = 148 * 16;
        spline_pass2_f32<<<(unsigned)b, 32 * kPass2Warps, 0, s>>>(buf, g, tb, outs[f]);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace gkm
