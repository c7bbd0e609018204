// Eulerian step on sm_100a: fused WENO reconstruction + gas-kinetic flux +
// conservative update, one sweep kernel per direction, plus the periodic halo
// wrap and the max(|u|+c) reduction that sets the next dt.
//
// Reference path replaced: evolveEulerian -> derivsX/Y/Z -> flux -> update
// (src/update.cpp:206-516), HaloTransfer (:855-1029), timestep (:1031-1054).
//
// Layout: the reference's own arrays, 5 components of nt^3 doubles (nt = n+6,
// index (j*nt + i)*nt + k, z fastest), ghosts refreshed on the device after
// every step, so every stencil read is in bounds and host<->device copies are
// plain memcpys of the reference's W[5].
//
// Per step: x sweep writes A = Fx(i) - Fx(i-1); y sweep A = (A + Fy(j)) - Fy(j-1);
// z sweep W' = W - (1/dx) ((A + Fz(k)) - Fz(k-1)) into A; the halo kernel
// wraps A's ghosts and the caller swaps W and A.  The additions run in the
// reference's left-to-right order with rounding-explicit intrinsics.
#include "gkm_internal.h"
#include "gkm_numerics.cuh"

namespace gkm {
namespace {

template <int DIR>
__device__ __forceinline__ int perm(int q)
{
    // face frame: slot 1 holds the normal momentum (y: swap 1<->2, z: swap 1<->3),
    // src/update.cpp:352-382 and :461-491
    if (DIR == 1) return q == 1 ? 2 : (q == 2 ? 1 : q);
    if (DIR == 2) return q == 1 ? 3 : (q == 3 ? 1 : q);
    return q;
}

struct Strides {
    long long sn, sA, sB;
};

template <int DIR>
__device__ __forceinline__ Strides strides(int nt)
{
    const long long nt2 = (long long)nt * nt;
    if (DIR == 0) return {nt, nt2, 1};   // normal i; window (j, k)
    if (DIR == 1) return {nt2, nt, 1};   // normal j; window (i, k)
    return {1, nt2, nt};                 // normal k; window (j, i)
}

// Tangential neighbour faces in window coordinates (da, db) and the scale of
// the first tangential slope.  "N/S" feed the y-slot slope and "F/B" the
// z-slot slope, as the reference pairs them (src/update.cpp:231-257,303-329,412-438).
template <int DIR>
struct Neigh {
    static constexpr int Na = DIR == 0 ? 1 : (DIR == 1 ? -1 : 0);
    static constexpr int Nb = DIR == 2 ? 1 : 0;
    static constexpr int Fa = DIR == 2 ? 1 : 0;
    static constexpr int Fb = DIR == 2 ? 0 : 1;
    static constexpr double ys = DIR == 1 ? -0.5 : 0.5;
};

template <int DIR>
struct SmemFace {
    const double* __restrict__ wf;   // slab of the left cell (6 comps x kWC)
    const double* __restrict__ wf1;  // slab of the right cell
    const double* __restrict__ rec;  // reconstructions: Wl comps 0..4, Wr comps 5..9
    int c, cN, cS, cF, cB;
    double inv_dx;
    __device__ __forceinline__ double WL(int q) const { return wf[perm<DIR>(q) * kWC + c]; }
    __device__ __forceinline__ double WR(int q) const { return wf1[perm<DIR>(q) * kWC + c]; }
    __device__ __forceinline__ double Wl(int q) const { return rec[perm<DIR>(q) * kWC + c]; }
    __device__ __forceinline__ double Wr(int q) const { return rec[(5 + perm<DIR>(q)) * kWC + c]; }
    __device__ __forceinline__ double DW(int v, int q) const
    {
        const int p = perm<DIR>(q);
        const double* l = rec + p * kWC;
        const double* r = rec + (5 + p) * kWC;
        switch (v) {
            case 0: return 2.0 * (l[c] - wf[p * kWC + c]) * inv_dx;
            case 1: return 2.0 * (wf1[p * kWC + c] - r[c]) * inv_dx;
            case 2: return Neigh<DIR>::ys * (l[cN] - l[cS]) * inv_dx;
            case 3: return Neigh<DIR>::ys * (r[cN] - r[cS]) * inv_dx;
            case 4: return 0.5 * (l[cF] - l[cB]) * inv_dx;
            default: return 0.5 * (r[cF] - r[cB]) * inv_dx;
        }
    }
};

__device__ __forceinline__ double viscosity(const FieldConst& fc, double T)
{
    double x = T / fc.T0;
    if (fc.visc == 1) return fc.mu0 * pow(x, 0.76);
    return fc.mu0 * (x * sqrt(x)) * (fc.T0 + 110.4) / (T + 110.4);   // Sutherland, src/update.cpp:277
}

// max(|u| + c) term of one cell with the reference's rounding (src/update.cpp:844-853,1041-1048)
__device__ __forceinline__ double wave_speed(const double w[5], double gam, double gm1)
{
    double d = w[0];
    double u = __ddiv_rn(w[1], d), v = __ddiv_rn(w[2], d), x = __ddiv_rn(w[3], d);
    double vs = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(x, x));
    double p = __dmul_rn(__dmul_rn(d, gm1), __dsub_rn(__ddiv_rn(w[4], d), __dmul_rn(0.5, vs)));
    return __dadd_rn(__dsqrt_rn(vs), __dsqrt_rn(__ddiv_rn(__dmul_rn(gam, p), d)));
}

__device__ __forceinline__ double step_dt(const SweepArgs& a)
{
    if (a.dt_fixed_mode) return a.dt_fixed;
    double mw = __longlong_as_double((long long)a.clock->wave[a.parity]);
    return __ddiv_rn(__dmul_rn(a.fc.cfl, a.fc.dx), mw);   // dt = cfl*dx/maxVAL, src/update.cpp:1053
}

__device__ __forceinline__ double block_max(double v, double* red)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < (int)((blockDim.x * blockDim.y + 31) / 32); w++) v = fmax(v, red[w]);
    }
    return v;
}

template <int DIR>
__global__ void __launch_bounds__(kSweepThreads, 2) sweep_kernel(SweepArgs a)
{
    extern __shared__ double smem[];
    double* ring = smem;                               // [kRing][kSlabComps][kWC]
    double* rec = smem + kRing * kSlabComps * kWC;     // [10][kWC]
    const FieldConst& fc = a.fc;
    const int n = fc.n, nt = fc.nt;
    const long long nt3 = fc.nt3;
    const Strides st = strides<DIR>(nt);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTB + tx;
    const int b0 = blockIdx.x * kTB, a0 = blockIdx.y * kTA;
    const int f_begin = blockIdx.z * a.seg_len;
    const int f_end = min(f_begin + a.seg_len, n);
    const double dt = step_dt(a);
    const Phys<double> ph{fc.gam, fc.gm1, kR, fc.K};
    const double* __restrict__ W = a.W;

    if (DIR == 0 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && tid == 0) {
        a.clock->wave[a.parity ^ 1] = 0ull;   // the z sweep of this step reduces into it
        a.clock->dt = dt;
    }
    if (f_begin >= n) return;

    auto slot = [&](int f) { return ring + ((f + 12) % kRing) * (kSlabComps * kWC); };
    auto load_slab = [&](int f) {
        double* s = slot(f);
        for (int c = tid; c < kWC; c += kSweepThreads) {
            const int aa = c / kWB, bb = c - aa * kWB;
            const int A = a0 + aa - 1, B = b0 + bb - 1;
            if (A > n || B > n) continue;
            const long long idx = (A + 3) * st.sA + (B + 3) * st.sB + (long long)(f + 3) * st.sn;
            const double r = W[idx], m1 = W[nt3 + idx], m2 = W[2 * nt3 + idx], m3 = W[3 * nt3 + idx],
                         E = W[4 * nt3 + idx];
            s[0 * kWC + c] = r;
            s[1 * kWC + c] = m1;
            s[2 * kWC + c] = m2;
            s[3 * kWC + c] = m3;
            s[4 * kWC + c] = E;
            s[5 * kWC + c] = temperature<double>(r, m1, m2, m3, E, ph);
        }
    };

    for (int f = f_begin - 3; f < f_begin + 2; f++) load_slab(f);

    const bool active = (a0 + ty < n) && (b0 + tx < n);
    const int cc = (ty + 1) * kWB + (tx + 1);
    const long long cell0 = (a0 + ty + 3) * st.sA + (b0 + tx + 3) * st.sB;
    double Fprev[5] = {0, 0, 0, 0, 0};
    double wmax = 0.0;
    bool bad = false;

    for (int f = f_begin - 1; f < f_end; f++) {
        load_slab(f + 3);
        __syncthreads();
        // reconstruct every face of the window once (the reference repeats this 5x per face)
        {
            const double* s0 = slot(f - 2);
            const double* s1 = slot(f - 1);
            const double* s2 = slot(f);
            const double* s3 = slot(f + 1);
            const double* s4 = slot(f + 2);
            const double* s5 = slot(f + 3);
            for (int c = tid; c < kWC; c += kSweepThreads) {
                const int aa = c / kWB, bb = c - aa * kWB;
                if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
                double l[5], r[5];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int o = q * kWC + c;
                    weno_scalar<double>(s0[o], s1[o], s2[o], s3[o], s4[o], s5[o], kWenoEps, l[q], r[q]);
                }
                double Tl, Tr;
                {
                    const int o = 5 * kWC + c;
                    weno_scalar<double>(s0[o], s1[o], s2[o], s3[o], s4[o], s5[o], kWenoEps, Tl, Tr);
                }
                l[4] = face_energy<double>(l[0], l[1], l[2], l[3], Tl, ph);
                r[4] = face_energy<double>(r[0], r[1], r[2], r[3], Tr, ph);
#pragma unroll
                for (int q = 0; q < 5; q++) {
                    rec[q * kWC + c] = l[q];
                    rec[(5 + q) * kWC + c] = r[q];
                }
            }
        }
        __syncthreads();
        if (active) {
            SmemFace<DIR> pv;
            pv.wf = slot(f);
            pv.wf1 = slot(f + 1);
            pv.rec = rec;
            pv.c = cc;
            pv.cN = cc + Neigh<DIR>::Na * kWB + Neigh<DIR>::Nb;
            pv.cS = cc - Neigh<DIR>::Na * kWB - Neigh<DIR>::Nb;
            pv.cF = cc + Neigh<DIR>::Fa * kWB + Neigh<DIR>::Fb;
            pv.cB = cc - Neigh<DIR>::Fa * kWB - Neigh<DIR>::Fb;
            pv.inv_dx = fc.inv_dx;
            // collision time of the left cell, mu(T)/p (src/update.cpp:276-278)
            const double* wl = slot(f);
            double tau0;
            {
                double d = wl[cc], id = 1.0 / d;
                double u = wl[kWC + cc] * id, v = wl[2 * kWC + cc] * id, w = wl[3 * kWC + cc] * id;
                double p = (d * fc.gm1) * (wl[4 * kWC + cc] * id - 0.5 * (u * u + v * v + w * w));
                double T = p / (kR * d);
                tau0 = viscosity(fc, T) / p;
            }
            double Fr[5];
            gks_flux<double>(pv, tau0, dt, fc.dx, ph, Fr);
            double F[5];
#pragma unroll
            for (int q = 0; q < 5; q++) F[perm<DIR>(q)] = Fr[q];
            if (f >= f_begin) {
                const long long ci = cell0 + (long long)(f + 3) * st.sn;
                if (DIR == 0) {
#pragma unroll
                    for (int q = 0; q < 5; q++) a.A[q * nt3 + ci] = __dsub_rn(F[q], Fprev[q]);
                } else if (DIR == 1) {
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        double acc = a.A[q * nt3 + ci];
                        a.A[q * nt3 + ci] = __dsub_rn(__dadd_rn(acc, F[q]), Fprev[q]);
                    }
                } else {
                    double wn[5];
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        double acc = a.A[q * nt3 + ci];
                        double s = __dsub_rn(__dadd_rn(acc, F[q]), Fprev[q]);
                        wn[q] = __dsub_rn(W[q * nt3 + ci], __dmul_rn(fc.inv_dx, s));
                        a.A[q * nt3 + ci] = wn[q];
                    }
                    double ws = wave_speed(wn, fc.gam, fc.gm1);
                    if (!isfinite(ws) || !(wn[0] > 0.0)) bad = true;
                    else wmax = ws > wmax ? ws : wmax;
                }
            }
#pragma unroll
            for (int q = 0; q < 5; q++) Fprev[q] = F[q];
        }
    }
    if (DIR == 2) {
        double m = block_max(wmax, rec);
        if (tid == 0 && m > 0.0) atomicMax(&a.clock->wave[a.parity ^ 1], (unsigned long long)__double_as_longlong(m));
        if (bad) atomicOr(&a.clock->status, 1);
    }
}

// Periodic ghost refresh: every ghost cell takes the interior cell at the
// wrapped index (what HaloTransfer produces on a 1x1x1 periodic topology).
__global__ void halo_kernel(double* __restrict__ W, FieldConst fc, DevClock* clock, int finish_step)
{
    const int n = fc.n, nt = fc.nt;
    const long long nt2 = (long long)nt * nt, nt3 = fc.nt3;
    const long long r1 = 6 * nt2, r2 = (long long)n * 6 * nt, r3 = (long long)n * n * 6;
    const long long total = r1 + r2 + r3;
    if (finish_step && blockIdx.x == 0 && threadIdx.x == 0) {
        clock->t += clock->dt;   // src/update.cpp:168-169
        clock->iter += 1;
    }
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        int j, i, k;
        if (g < r1) {
            long long m = g / nt2, rem = g - m * nt2;
            j = m < 3 ? (int)m : n + (int)m;
            i = (int)(rem / nt);
            k = (int)(rem - (long long)i * nt);
        } else if (g < r1 + r2) {
            long long h = g - r1;
            long long per = 6LL * nt;
            j = 3 + (int)(h / per);
            long long rem = h - (long long)(j - 3) * per;
            int m = (int)(rem / nt);
            i = m < 3 ? m : n + m;
            k = (int)(rem - (long long)m * nt);
        } else {
            long long h = g - r1 - r2;
            long long per = 6LL * n;
            j = 3 + (int)(h / per);
            long long rem = h - (long long)(j - 3) * per;
            i = 3 + (int)(rem / 6);
            int m = (int)(rem - (long long)(i - 3) * 6);
            k = m < 3 ? m : n + m;
        }
        auto wrap = [n](int x) { return x < 3 ? x + n : (x >= n + 3 ? x - n : x); };
        const long long dst = ((long long)j * nt + i) * nt + k;
        const long long src = ((long long)wrap(j) * nt + wrap(i)) * nt + wrap(k);
#pragma unroll
        for (int q = 0; q < 5; q++) W[q * nt3 + dst] = W[q * nt3 + src];
    }
}

__global__ void wave_reduce_kernel(const double* __restrict__ W, FieldConst fc, DevClock* clock, int slot)
{
    __shared__ double red[32];
    const int n = fc.n, nt = fc.nt;
    const long long nt3 = fc.nt3, total = (long long)n * n * n;
    double m = 0.0;
    bool bad = false;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(g / ((long long)n * n)), i = (int)((g / n) % n), k = (int)(g % n);
        const long long idx = ((long long)(j + 3) * nt + (i + 3)) * nt + (k + 3);
        double w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) w[q] = W[q * nt3 + idx];
        double ws = wave_speed(w, fc.gam, fc.gm1);
        if (!isfinite(ws) || !(w[0] > 0.0)) bad = true;
        else m = ws > m ? ws : m;
    }
    m = block_max(m, red);
    if (threadIdx.x == 0 && m > 0.0) atomicMax(&clock->wave[slot], (unsigned long long)__double_as_longlong(m));
    if (bad) atomicOr(&clock->status, 1);
}

// Single-face entry with the same math as the sweep: per face 51 inputs
// WL[5] WR[5] Wl[5] Wr[5] DWxl DWxr DWyl DWyr DWzl DWzr [6x5] tau0.
__global__ void flux_faces_kernel(const double* __restrict__ in, long long nf, Phys<double> ph, double dt, double dx,
                                  double* __restrict__ F)
{
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const double* p = in + f * 51;
    FaceInput<double> fi;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        fi.WL_[q] = p[q];
        fi.WR_[q] = p[5 + q];
        fi.Wl_[q] = p[10 + q];
        fi.Wr_[q] = p[15 + q];
    }
#pragma unroll
    for (int v = 0; v < 6; v++)
#pragma unroll
        for (int q = 0; q < 5; q++) fi.DW_[v][q] = p[20 + 5 * v + q];
    double out[5];
    gks_flux<double>(fi, p[50], dt, dx, ph, out);
#pragma unroll
    for (int q = 0; q < 5; q++) F[f * 5 + q] = out[q];
}

__global__ void weno_faces_kernel(const double* __restrict__ s, long long n, Phys<double> ph, double* __restrict__ Wl,
                                  double* __restrict__ Wr)
{
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= n) return;
    const double* p = s + f * 30;   // 6 cells x 5 components
    double l[5], r[5], T[6];
#pragma unroll
    for (int o = 0; o < 6; o++) T[o] = temperature<double>(p[5 * o], p[5 * o + 1], p[5 * o + 2], p[5 * o + 3], p[5 * o + 4], ph);
#pragma unroll
    for (int q = 0; q < 4; q++)
        weno_scalar<double>(p[q], p[5 + q], p[10 + q], p[15 + q], p[20 + q], p[25 + q], kWenoEps, l[q], r[q]);
    double Tl, Tr;
    weno_scalar<double>(T[0], T[1], T[2], T[3], T[4], T[5], kWenoEps, Tl, Tr);
    l[4] = face_energy<double>(l[0], l[1], l[2], l[3], Tl, ph);
    r[4] = face_energy<double>(r[0], r[1], r[2], r[3], Tr, ph);
#pragma unroll
    for (int q = 0; q < 5; q++) {
        Wl[f * 5 + q] = l[q];
        Wr[f * 5 + q] = r[q];
    }
}

template <int DIR>
cudaError_t launch_one(const SweepArgs& a, int nseg, cudaStream_t s)
{
    dim3 grid((a.fc.n + kTB - 1) / kTB, (a.fc.n + kTA - 1) / kTA, nseg);
    dim3 block(kTB, kTA);
    sweep_kernel<DIR><<<grid, block, kSweepSmem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t sweep_prepare()
{
    cudaError_t e = cudaFuncSetAttribute(sweep_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSweepSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sweep_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSweepSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sweep_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSweepSmem);
    return e;
}

cudaError_t launch_sweep(int dir, const SweepArgs& a, int nseg, cudaStream_t s)
{
    if (dir == 0) return launch_one<0>(a, nseg, s);
    if (dir == 1) return launch_one<1>(a, nseg, s);
    return launch_one<2>(a, nseg, s);
}

cudaError_t launch_halo(double* W, const FieldConst& fc, DevClock* clock, int finish_step, cudaStream_t s)
{
    long long total = (long long)fc.nt * fc.nt * fc.nt - (long long)fc.n * fc.n * fc.n;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    halo_kernel<<<blocks, 256, 0, s>>>(W, fc, clock, finish_step);
    return cudaGetLastError();
}

cudaError_t launch_wave_reduce(const double* W, const FieldConst& fc, DevClock* clock, int slot, cudaStream_t s)
{
    long long total = (long long)fc.n * fc.n * fc.n;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    wave_reduce_kernel<<<blocks, 256, 0, s>>>(W, fc, clock, slot);
    return cudaGetLastError();
}

cudaError_t launch_flux_faces(const double* in, long long nfaces, double gam, int K, double dt, double dx, double* F,
                              cudaStream_t s)
{
    if (nfaces <= 0) return cudaSuccess;
    Phys<double> ph{gam, gam - 1.0, kR, K};
    flux_faces_kernel<<<(unsigned)((nfaces + 63) / 64), 64, 0, s>>>(in, nfaces, ph, dt, dx, F);
    return cudaGetLastError();
}

cudaError_t launch_weno_faces(const double* stencils, long long n, double gam, double* Wl, double* Wr, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    Phys<double> ph{gam, gam - 1.0, kR, 2};
    weno_faces_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(stencils, n, ph, Wl, Wr);
    return cudaGetLastError();
}

}  // namespace gkm
