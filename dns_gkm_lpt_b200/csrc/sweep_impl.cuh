// The fused sweep kernel, templated on the face normal DIR and on the type T
// the reconstruction and the flux run in.  Instantiated for T = double in
// sweep.cu (the FP64 drop-in) and for T = float in sweep_mixed.cu (the
// mixed-precision form).  Both read and write the FP64 state and FP64
// accumulator; the float form converts to non-dimensional single precision
// when a slab enters shared memory (rho / rho0, m / (rho0 us), E / p0,
// T / T0 with us = sqrt(p0 / rho0), lengths in dx) and converts each face
// flux back to dimensional FP64 before the flux difference is accumulated.
//
// Reference path: derivsX/Y/Z (src/update.cpp:214-503) -> flux
// (src/GKMflux.cpp:11-229) -> update (src/update.cpp:505-516), timestep
// (src/update.cpp:1031-1054).
#pragma once

#include "gkm_internal.h"
#include "gkm_numerics.cuh"

namespace gkm {
namespace sweep_detail {

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

template <int DIR, class T, int kWC>
struct SmemFace {
    const T* __restrict__ wf;   // slab of the left cell (6 comps x kWC)
    const T* __restrict__ wf1;  // slab of the right cell
    const T* __restrict__ rec;  // reconstructions: Wl comps 0..4, Wr comps 5..9
    int c, cN, cS, cF, cB;
    T inv_dx;
    __device__ __forceinline__ T WL(int q) const { return wf[perm<DIR>(q) * kWC + c]; }
    __device__ __forceinline__ T WR(int q) const { return wf1[perm<DIR>(q) * kWC + c]; }
    __device__ __forceinline__ T Wl(int q) const { return rec[perm<DIR>(q) * kWC + c]; }
    __device__ __forceinline__ T Wr(int q) const { return rec[(5 + perm<DIR>(q)) * kWC + c]; }
    __device__ __forceinline__ T DW(int v, int q) const
    {
        const int p = perm<DIR>(q);
        const T* l = rec + p * kWC;
        const T* r = rec + (5 + p) * kWC;
        const T ys = T(Neigh<DIR>::ys);
        switch (v) {
            case 0: return T(2) * (l[c] - wf[p * kWC + c]) * inv_dx;
            case 1: return T(2) * (wf1[p * kWC + c] - r[c]) * inv_dx;
            case 2: return ys * (l[cN] - l[cS]) * inv_dx;
            case 3: return ys * (r[cN] - r[cS]) * inv_dx;
            case 4: return T(0.5) * (l[cF] - l[cB]) * inv_dx;
            default: return T(0.5) * (r[cF] - r[cB]) * inv_dx;
        }
    }
};

// tau0 = mu(T) / p of a cell (src/update.cpp:276-278) with one division: Sutherland
// mu0 x^(3/2) (T0 + 110.4) / (T + 110.4), x = T / T0, or the power law mu0 x^0.76
__device__ __forceinline__ double collision_time(const FieldConst& fc, double T, double p)
{
    const double x = T * fc.inv_T0;
    if (fc.visc == 1) return fc.mu0 * pow(x, 0.76) / p;
    return fc.mu0 * (x * sqrt(x)) * (fc.T0 + 110.4) / ((T + 110.4) * p);
}

// |u| + c of a conserved state in FP64: with one reciprocal of rho (the z sweeps' reduction
// for the next step's dt, within an ulp or two of the reference's), and with the reference's
// divisions (src/update.cpp:1039-1046 via c2p; the stand-alone timestep, whose dt equals the
// reference's bit for bit).
__device__ __forceinline__ double wave_speed_recip(const double w[5], double gam, double gm1)
{
    const double d = w[0], id = 1.0 / d;
    const double u = w[1] * id, v = w[2] * id, x = w[3] * id;
    const double vs = u * u + v * v + x * x;
    const double p = (d * gm1) * (w[4] * id - 0.5 * vs);
    return sqrt(vs) + sqrt(gam * p * id);
}

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
    return cfl_dt(a.fc, a.clock, a.parity, a.dt_fixed_mode, a.dt_fixed);
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

// elements of one ring slot: kSlabComps x WC values, padded to a multiple of 128 bytes
template <class T, class Tile>
__host__ __device__ constexpr int slot_elems()
{
    return (int)((kSlabComps * Tile::WC * sizeof(T) + 127) / 128 * 128 / sizeof(T));
}

template <class T, class Tile>
__host__ __device__ constexpr size_t sweep_ring_bytes()
{
    // 128 bytes of slack to align the ring (a bulk tensor copy lands on a 128-byte boundary),
    // the ring of padded slots, the reconstructions
    return (128 + sizeof(T) * (size_t)(kRing * slot_elems<T, Tile>() + 10 * Tile::WC) + 15) / 16 * 16;
}

// ring + reconstructions, then a per-thread FP64 staging area [5][threads] for the
// accumulator of the thread's cell, fetched asynchronously while the flux is computed.
// The mixed x sweep (and a mixed sweep without tensor maps) keeps its FP32 ring unaligned and
// has no staging area.
template <class T, int DIR>
__host__ __device__ constexpr bool sweep_lean()
{
    return sizeof(T) == 4 && DIR != 1;
}

// FP64 z sweep: the accumulator of two consecutive k-cells of the window moves as one brick, a
// box (2, TB, TA, 5) of the (k, i, j, q) tensor, loaded and stored by bulk tensor copies; two
// bricks in flight.  The staging area of the other sweeps shares their space.  The slabs arrive the
// same way, two planes of the window and its halo (a box (2, WB, WA, 5)) in a landing area.
template <class Tile>
__host__ __device__ constexpr int zbrick_elems()
{
    return 5 * Tile::TA * Tile::TB * 2;
}
template <class Tile>
__host__ __device__ constexpr int zland_elems()
{
    return 5 * Tile::WC * 2;
}

template <class T, int DIR>
__host__ __device__ constexpr bool sweep_zpairs()
{
    return DIR == 2;
}
// mixed x and y sweeps: each new slab lands in FP64 by one bulk tensor copy in a landing area, and the
// threads convert it into the FP32 ring
template <class T, int DIR>
__host__ __device__ constexpr bool sweep_mland()
{
    return sizeof(T) == 4 && DIR != 2;
}
// the mixed z sweep's FP64 state of the updated cells (its ring holds FP32 copies) comes as bricks
// too, else by direct loads
template <class T>
__host__ __device__ constexpr bool sweep_state_bricks()
{
    return sizeof(T) == 4;
}
// brick buffers of the z sweep: two (the next pair's brick requested one cell before the current
// pair's store), or one (requested after that store has read it) where shared memory decides how
// many CTAs an SM holds (the mixed form: three CTAs per SM instead of two)
template <class T>
__host__ __device__ constexpr int sweep_zbufs()
{
    return sizeof(T) == 4 ? 1 : 2;
}

template <class T, class Tile, int DIR = 1>
__host__ __device__ constexpr size_t sweep_smem_bytes()
{
    // z sweep: ring + reconstructions, 128 bytes of slack to align the bricks, two accumulator
    // bricks, two bricks of the FP64 state (mixed form), the slab landing area, three mbarriers
    if (sweep_zpairs<T, DIR>())
        return (sweep_ring_bytes<T, Tile>() + 128 +
                sizeof(double) * ((sweep_state_bricks<T>() ? 2 : 1) * sweep_zbufs<T>() * zbrick_elems<Tile>() +
                                  zland_elems<Tile>()) +
                24 + 15) /
               16 * 16;
    // mixed x, y: ring + reconstructions, the y sweep's accumulator staging, slack, the landing area,
    // one mbarrier
    if (sweep_mland<T, DIR>())
        return sweep_ring_bytes<T, Tile>() + (DIR == 1 ? sizeof(double) * 5 * (size_t)Tile::threads : 0) + 128 +
               sizeof(double) * 5 * (size_t)Tile::WC + 16;
    if (sweep_lean<T, DIR>()) return sizeof(T) * (size_t)(kRing * slot_elems<T, Tile>() + 10 * Tile::WC);
    return sweep_ring_bytes<T, Tile>() + sizeof(double) * 5 * (size_t)Tile::threads + 16;   // + mbarrier
}

// cp.async: 8-byte global -> shared copies that land while the thread keeps computing
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Bulk tensor copies (TMA) completing on an mbarrier.  The waits are bounded: a copy that has not
// landed after ~2^24 polls raises bit 1 of the clock's status word and the kernel carries on,
// so a failure is reported to the host and never hangs the GPU.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void tma_slab_load(unsigned dst, const void* tmap, int c0, int c1, int c2, unsigned bytes,
                                              unsigned bar)
{
    // shared-memory writes of the generic proxy (the slot's previous contents) before the copy's
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(dst),
        "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(0), "r"(bar)
        : "memory");
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, int polls = 1 << 24)
{
    for (int it = 0; it < polls; it++) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// global -> shared bulk tensor copy completing on a barrier phase whose expected bytes were
// already announced (by the tma_slab_load of the same phase)
__device__ __forceinline__ void tma_box_load(unsigned dst, const void* tmap, int c0, int c1, int c2, unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(dst),
        "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(0), "r"(bar)
        : "memory");
}
// shared -> global bulk tensor copy of a box whose origin (c0, c1, c2, 0) is inside the tensor
// (elements beyond its extent are not written), and the waits on such copies: until each has read
// its shared-memory source, and until each has completed
__device__ __forceinline__ void tma_box_store(const void* tmap, int c0, int c1, int c2, unsigned src)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];\n" ::"l"(tmap),
                 "r"(c0), "r"(c1), "r"(c2), "r"(0), "r"(src)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// generic-proxy shared-memory writes of this thread, ordered before later bulk copies that read them
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// retire `bytes` of a barrier phase's expected transaction count without a copy (the failure-detection
// test hook takes back the bytes it added beyond what its copy delivers)
__device__ __forceinline__ void mbar_complete_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// the test hook's extra expected bytes and its short poll count
constexpr unsigned kProbeExtraBytes = 16;
constexpr int kProbePolls = 256;

}  // namespace sweep_detail

// Periodic ghost refresh of ghost cell g (0 <= g < nt^3 - n^3): the ghost
// takes the interior cell at the wrapped index (what HaloTransfer produces on
// a 1x1x1 periodic topology).  Ghost cells are enumerated as the 6 ghost
// y-planes, then the 6 ghost x-rows of the interior y-planes, then the 6
// ghost z-cells of the interior (y, x) rows.
__device__ __forceinline__ void halo_cell(double* __restrict__ W, const FieldConst& fc, long long g)
{
    const int n = fc.n, nt = fc.nt;
    const long long nt2 = (long long)nt * nt, nt3 = fc.nt3;
    const long long r1 = 6 * nt2, r2 = (long long)n * 6 * nt;
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

// Which data movement a sweep kernel is compiled for: tensor copies (the handle has tensor maps)
// or per-element copies (odd nt).  The single-cube launches pick the form by the maps a launch
// carries, so each kernel holds only its own path; the ensemble's persistent kernel serves
// members with and without maps and decides per item.
constexpr int kMapsRuntime = 0, kMapsOn = 1, kMapsOff = 2;

// One CTA's work: the window (bx, by) of faces, segment bz along the normal.
// Called once per CTA by sweep_kernel and once per work item by the
// persistent ensemble kernel; every thread of the CTA takes the same path.
template <int DIR, class T, class Tile, int MM = kMapsRuntime>
__device__ __forceinline__ void sweep_block(const SweepArgs& a, int bx, int by, int bz, unsigned char* smem_raw)
{
    using namespace sweep_detail;
    constexpr int kTB = Tile::TB, kTA = Tile::TA, kWB = Tile::WB, kWC = Tile::WC;
    constexpr int kSweepThreads = Tile::threads;
    constexpr bool kMixed = sizeof(T) == 4;
    constexpr int kSlot = slot_elems<T, Tile>();
    // ring [kRing][kSlot] (slot: kSlabComps x kWC values), reconstructions [10][kWC], then the
    // accumulator staging [5][threads] and one mbarrier
    T* ring = sweep_lean<T, DIR>() ? reinterpret_cast<T*>(smem_raw)
                                   : reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    T* rec = ring + kRing * kSlot;
    constexpr bool kZPairs = sweep_zpairs<T, DIR>();
    constexpr int kZB = zbrick_elems<Tile>();
    // z sweep: two accumulator bricks (128-byte aligned for the bulk copies), whose space also
    // serves as the FP64 staging area, in the mixed form two bricks of the FP64 state, the slab
    // landing area [q][a][b][2], then three mbarriers (the two bricks', the landing area's)
    double* stage =
        kZPairs ? reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(smem_raw + sweep_ring_bytes<T, Tile>()) + 127) &
                                            ~uintptr_t(127))
                : reinterpret_cast<double*>(smem_raw + sweep_ring_bytes<T, Tile>());   // [5][threads]
    // every area a bulk tensor copy writes starts on a 128-byte boundary: the bricks' sizes keep it
    static_assert(zbrick_elems<Tile>() * sizeof(double) % 128 == 0, "brick size breaks the 128-byte alignment");
    constexpr int kZBufs = sweep_zbufs<T>();
    double* wbr = stage + kZBufs * kZB;                                       // mixed z sweep: FP64 state bricks
    double* land = wbr + (sweep_state_bricks<T>() ? kZBufs * kZB : 0);        // [q][a][b][2]
    // mixed x, y sweeps: the FP64 landing area [q][a][b] of one slab (after the y sweep's staging)
    constexpr bool kMLand = sweep_mland<T, DIR>();
    double* mland = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(smem_raw + sweep_ring_bytes<T, Tile>() + (DIR == 1 ? 40 * kSweepThreads : 0)) + 127) &
        ~uintptr_t(127));
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(
        kZPairs ? land + zland_elems<Tile>() : (kMLand ? mland + 5 * kWC : stage + 5 * kSweepThreads));
    const FieldConst& fc = a.fc;
    const int n = fc.n, nt = fc.nt;
    const long long nt3 = fc.nt3;
    const Strides st = strides<DIR>(nt);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTB + tx;
    const int b0 = bx * kTB, a0 = by * kTA;
    const int f_begin = a.f0 + bz * a.seg_len;
    const int f_end = min(f_begin + a.seg_len, a.f1 > 0 ? a.f1 : n);
    const double dt = step_dt(a);
    // working units: dimensional for double, non-dimensional (dx = 1) for float
    const T dtw = kMixed ? T(dt * fc.u_s * fc.inv_dx) : T(dt);
    const T dxw = kMixed ? T(1) : T(fc.dx);
    const T inv_dxw = kMixed ? T(1) : T(fc.inv_dx);
    const Phys<T> ph{T(fc.gam), T(fc.gm1), kMixed ? T(1) : T(kR), fc.K};
    const float cv_mixed = float(1.0 / fc.gm1);   // R / (gamma - 1) in the non-dimensional units (R = 1)
    const T eps_r = kMixed ? T(fc.eps_rho) : T(kWenoEps);
    const T eps_m = kMixed ? T(fc.eps_m) : T(kWenoEps);
    const T eps_T = kMixed ? T(fc.eps_T) : T(kWenoEps);
    const double* __restrict__ W = a.W;
    const double suth_c = fc.mu0 * (fc.T0 + 110.4) * kR / ((kR * fc.T0) * sqrt(kR * fc.T0));
    // mixed form: tau' = tau us / dx = tc_a x^(3/2) / ((x + tc_b) p') (Sutherland) or tc_a x^0.76 / p'
    // (power law), x = T / T0, p' = p / p0
    const float tc_a = kMixed ? float(fc.visc == 1 ? fc.mu0 * fc.u_s * fc.inv_dx / fc.p0
                                                   : fc.mu0 * (fc.T0 + 110.4) * fc.u_s * fc.inv_dx / (fc.T0 * fc.p0))
                              : 0.f;
    const float tc_b = kMixed ? float(110.4 / fc.T0) : 0.f;

    if (DIR == 0 && bx == 0 && by == 0 && bz == 0 && tid == 0 && !a.skip_clock_init) {
        a.clock->wave[a.parity ^ 1] = 0ull;   // the z sweep of this step reduces into it
        a.clock->dt = dt;
    }
    if (f_begin >= f_end) return;

    // FP64 x and y sweeps with a tensor map: one thread moves each new slab (5 components of the
    // window, a box of the (k, i, j, q) tensor whose smem image is the slot's [q][a][b] layout)
    // with one bulk tensor copy completing on the mbarrier
    const bool maps = MM == kMapsOn || (MM == kMapsRuntime && a.tmap != nullptr);
    const bool use_tma = !kMixed && DIR != 2 && maps;
    const bool mtma = kMLand && maps;   // mixed x / y: slabs land in FP64 by tensor copy
    // failure-detection test hook: the first CTA's first copy is expected with kProbeExtraBytes more
    // than it delivers, so its first wait (kProbePolls polls) runs out and raises status bit 1; the
    // CTA then retires the extra bytes and waits for the copy itself, which lands normally
    const bool probe = use_tma && a.wait_probe && bx == 0 && by == 0 && bz == 0;
    const unsigned bar_u32 = smem_u32(bar);
    unsigned tma_phase = 0;
    if (use_tma || mtma) {
        if (tid == 0) mbar_init(bar_u32);
        __syncthreads();
    }

    auto slot = [&](int f) { return ring + ((f + 12) % kRing) * kSlot; };
    // one cell of a slab into its ring slot: the conserved values with the temperature, converted to
    // the non-dimensional single-precision units in the mixed form
    auto store_cell = [&](T* s, int c, double r, double m1, double m2, double m3, double E) {
        if constexpr (kMixed) {
            const double Tk = temperature<double>(r, m1, m2, m3, E, Phys<double>{fc.gam, fc.gm1, kR, fc.K});
            s[0 * kWC + c] = T(r * fc.inv_rho_s);
            s[1 * kWC + c] = T(m1 * fc.inv_m_s);
            s[2 * kWC + c] = T(m2 * fc.inv_m_s);
            s[3 * kWC + c] = T(m3 * fc.inv_m_s);
            s[4 * kWC + c] = T(E * fc.inv_E_s);
            s[5 * kWC + c] = T(Tk * fc.inv_T0);
        } else {
            s[0 * kWC + c] = r;
            s[1 * kWC + c] = m1;
            s[2 * kWC + c] = m2;
            s[3 * kWC + c] = m3;
            s[4 * kWC + c] = E;
            s[5 * kWC + c] = temperature<double>(r, m1, m2, m3, E, ph);
        }
    };
    auto load_slab = [&](int f) {
        T* s = slot(f);
        for (int c = tid; c < kWC; c += kSweepThreads) {
            const int aa = c / kWB, bb = c - aa * kWB;
            const int A = a0 + aa - 1, B = b0 + bb - 1;
            if (A > n || B > n) continue;
            const long long idx = (A + 3) * st.sA + (B + 3) * st.sB + (long long)(f + 3) * st.sn;
            store_cell(s, c, W[idx], W[nt3 + idx], W[2 * nt3 + idx], W[3 * nt3 + idx], W[4 * nt3 + idx]);
        }
    };

    // FP64: the slab of the next step travels global -> shared asynchronously during this step's
    // flux, straight into its ring slot (last read by this step's reconstruction); each thread
    // forms the temperature of the cells it copied once its copies have landed.  (Without tensor
    // maps the mixed form converts while loading.)
    auto issue_slab = [&](int f) {
        double* dst = reinterpret_cast<double*>(slot(f));
        for (int c = tid; c < kWC; c += kSweepThreads) {
            const int aa = c / kWB, bb = c - aa * kWB;
            const int A = a0 + aa - 1, B = b0 + bb - 1;
            if (A > n || B > n) continue;
            const long long idx = (A + 3) * st.sA + (B + 3) * st.sB + (long long)(f + 3) * st.sn;
#pragma unroll
            for (int q = 0; q < 5; q++) cp_async8(&dst[q * kWC + c], &W[q * nt3 + idx]);
        }
        cp_async_commit();
    };
    auto finish_slab = [&](int f) {
        T* s = slot(f);
        for (int c = tid; c < kWC; c += kSweepThreads) {
            const int aa = c / kWB, bb = c - aa * kWB;
            if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
            s[5 * kWC + c] = temperature<T>(s[c], s[kWC + c], s[2 * kWC + c], s[3 * kWC + c], s[4 * kWC + c], ph);
        }
    };

    // the segment's first six slabs arrive together (FP64 x / y sweeps with a tensor map: six bulk
    // tensor copies completing on one barrier phase), instead of six rounds of loads
    if (use_tma) {
        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar_u32),
                         "r"((unsigned)(6 * 5 * kWC * sizeof(double)))
                         : "memory");
            for (int f = f_begin - 3; f < f_begin + 3; f++)
                tma_box_load(smem_u32(slot(f)), a.tmap, b0 + 2, DIR == 0 ? f + 3 : a0 + 2, DIR == 0 ? a0 + 2 : f + 3,
                             bar_u32);
        }
        if (!mbar_wait_bounded(bar_u32, tma_phase)) atomicOr(&a.clock->status, 2);
        tma_phase ^= 1u;
        for (int f = f_begin - 3; f < f_begin + 3; f++) finish_slab(f);
    } else if (!kMixed) {
        // FP64 otherwise (the z sweep, odd nt): the first six slabs by cp.async, one wait for all
        for (int f = f_begin - 3; f < f_begin + 3; f++) issue_slab(f);
        cp_async_wait_all();
        for (int f = f_begin - 3; f < f_begin + 3; f++) finish_slab(f);
    } else {
        // mixed form: the first six slabs by one round of loads per cell (30 in flight), then converted
        for (int c = tid; c < kWC; c += kSweepThreads) {
            const int aa = c / kWB, bb = c - aa * kWB;
            const int A = a0 + aa - 1, B = b0 + bb - 1;
            if (A > n || B > n) continue;
            const long long idx0 = (A + 3) * st.sA + (B + 3) * st.sB;
            double v[6][5];
#pragma unroll
            for (int p = 0; p < 6; p++)
#pragma unroll
                for (int q = 0; q < 5; q++) v[p][q] = W[q * nt3 + idx0 + (long long)(f_begin + p) * st.sn];
#pragma unroll
            for (int p = 0; p < 6; p++) store_cell(slot(f_begin - 3 + p), c, v[p][0], v[p][1], v[p][2], v[p][3], v[p][4]);
        }
    }

    // FP64 z sweep.  Its normal k is the contiguous axis, so one value per window cell and plane is
    // 8 bytes of a different 128-byte line; the window's 1,620 lines per plane (16 x 16 windows)
    // do not stay in L1 for the four planes a 32-byte sector holds, and per-element loads fetch
    // each sector from L2 four times.  Planes k, k+1 with k + 3 even travel together instead.
    // Slabs (a.tmap): the two planes of the window and its halo land as one box in the landing area
    // and each thread moves its cells' values into the plane's ring slot as it forms their
    // temperature; the next box is requested once the landing area's second plane is in the ring,
    // one face before it is needed.  Accumulator (a.tmap_acc): cells k, k+1 form a pair, and the
    // pairs whose two cells both lie in this segment move as bricks: each brick is loaded while the
    // faces before it are computed (the load of a pair issued when the previous pair's second cell
    // starts), updated in shared memory by its two cells and stored once the second cell is
    // written.  A cell whose partner lies in another segment (at most the first and the last of
    // each) is read and written directly, so no two CTAs store the same brick.
    const bool zslab = kZPairs && (MM == kMapsOn || (MM == kMapsRuntime && a.tmap != nullptr));
    const bool zpair = kZPairs && (MM == kMapsOn || (MM == kMapsRuntime && a.tmap_acc != nullptr &&
                                                     (!sweep_state_bricks<T>() || a.tmap_wb != nullptr)));
    const unsigned zbar = smem_u32(bar), lbar = zbar + 16u;
    unsigned zph = 0;   // bit b: the phase of brick buffer b's barrier awaited next
    unsigned lph = 0;   // the phase of the landing area's barrier awaited next
    auto first_of_pair = [](int f) { return ((f + 3) & 1) == 0; };
    auto paired = [&](int f) {
        const int p = first_of_pair(f) ? f + 1 : f - 1;
        return p >= f_begin && p < f_end;
    };
    auto zbuf = [](int f) { return kZBufs == 2 ? ((f + 3) >> 1) & 1 : 0; };
    const int pf0 = first_of_pair(f_begin) ? f_begin : f_begin + 1;   // the segment's first pair
    auto zload = [&](int pf) {   // the brick of the pair whose first cell is pf (one thread)
        const int b = zbuf(pf);
        if constexpr (sweep_state_bricks<T>()) {   // the accumulator's and the FP64 state's bricks, one barrier phase
            tma_slab_load(smem_u32(stage + b * kZB), a.tmap_acc, pf + 3, b0 + 3, a0 + 3,
                          (unsigned)(2 * kZB * sizeof(double)), zbar + 8u * b);
            tma_box_load(smem_u32(wbr + b * kZB), a.tmap_wb, pf + 3, b0 + 3, a0 + 3, zbar + 8u * b);
        } else {
            tma_slab_load(smem_u32(stage + b * kZB), a.tmap_acc, pf + 3, b0 + 3, a0 + 3,
                          (unsigned)(kZB * sizeof(double)), zbar + 8u * b);
        }
    };
    auto zslab_load = [&](int p) {   // planes p, p+1 (p + 3 even) of the window and its halo (one thread)
        tma_slab_load(smem_u32(land), a.tmap, p + 3, b0 + 2, a0 + 2, (unsigned)(zland_elems<Tile>() * sizeof(double)), lbar);
    };
    // mixed x / y: plane f from the FP64 landing area [q][a][b] into its ring slot
    auto finish_slab_mland = [&](int f) {
        T* s = slot(f);
        for (int c = tid; c < kWC; c += kSweepThreads) {
            const int aa = c / kWB, bb = c - aa * kWB;
            if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
            store_cell(s, c, mland[c], mland[kWC + c], mland[2 * kWC + c], mland[3 * kWC + c], mland[4 * kWC + c]);
        }
    };
    // plane f from the landing area into its ring slot, with its temperature
    auto finish_slab_landed = [&](int f) {
        T* s = slot(f);
        const double* L = land + ((f + 3) & 1);
        for (int c = tid; c < kWC; c += kSweepThreads) {
            const int aa = c / kWB, bb = c - aa * kWB;
            if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
            store_cell(s, c, L[2 * c], L[2 * (kWC + c)], L[2 * (2 * kWC + c)], L[2 * (3 * kWC + c)], L[2 * (4 * kWC + c)]);
        }
    };
    if (zpair || zslab) {
        if (tid == 0) {
            mbar_init(zbar);
            mbar_init(zbar + 8u);
            mbar_init(lbar);
        }
        __syncthreads();
        if (tid == 0 && zpair && pf0 + 1 < f_end) zload(pf0);
        // the first plane not loaded directly, f_begin + 3, and its partner
        if (tid == 0 && zslab) zslab_load(first_of_pair(f_begin + 3) ? f_begin + 3 : f_begin + 2);
    }

    const bool active = (a0 + ty < n) && (b0 + tx < n);
    const int cc = (ty + 1) * kWB + (tx + 1);
    const long long cell0 = (a0 + ty + 3) * st.sA + (b0 + tx + 3) * st.sB;
    double Fprev[5] = {0, 0, 0, 0, 0};
    double wmax = 0.0;
    bool bad = false;

    for (int f = f_begin - 1; f < f_end; f++) {
        if (f == f_begin - 1) {
            // slab f + 3 came with the first six
        } else if (kMixed && !zslab && !mtma) {
            load_slab(f + 3);
        } else {
            if (use_tma) {
                if (probe && f == f_begin) {
                    if (!mbar_wait_bounded(bar_u32, tma_phase, kProbePolls)) atomicOr(&a.clock->status, 2);
                    if (tid == 0) mbar_complete_tx(bar_u32, kProbeExtraBytes);
                }
                if (!mbar_wait_bounded(bar_u32, tma_phase)) atomicOr(&a.clock->status, 2);
                tma_phase ^= 1u;
            } else if (mtma) {
                if (!mbar_wait_bounded(bar_u32, tma_phase)) atomicOr(&a.clock->status, 2);
                tma_phase ^= 1u;
            } else if (zslab) {
                // a box holds planes f+3 and f+4, or f+2 and f+3: wait for it where its first plane is taken
                if (first_of_pair(f + 3) || f == f_begin) {
                    if (!mbar_wait_bounded(lbar, lph)) atomicOr(&a.clock->status, 2);
                    lph ^= 1u;
                }
            } else {
                cp_async_wait_all();
            }
            if (zslab) finish_slab_landed(f + 3);
            else if (mtma) finish_slab_mland(f + 3);
            else finish_slab(f + 3);
        }
        __syncthreads();
        // the landing area's second plane is in the ring: the next two planes, wanted from the next face on
        if (zslab && tid == 0 && f >= f_begin && !first_of_pair(f + 3) && f + 1 < f_end) zslab_load(f + 4);
        if (zpair && tid == 0 && f > f_begin) {
            // the pair the previous cell completed goes out (its writes were fenced before the barrier)
            if (!first_of_pair(f - 1) && paired(f - 1))
                tma_box_store(a.tmap_acc, f + 1, b0 + 3, a0 + 3, smem_u32(stage + zbuf(f - 1) * kZB));
            if (kZBufs == 2) {   // the next pair comes in, into the buffer whose store left one cell ago
                if (!first_of_pair(f) && paired(f) && f + 2 < f_end) {
                    bulk_wait_read();
                    zload(f + 1);
                }
            } else if (first_of_pair(f) && f + 1 < f_end && f != pf0) {   // this cell's pair, once the store has read the buffer
                bulk_wait_read();
                zload(f);
            }
        }
        // reconstruct every face of the window once (the reference repeats this 5x per face)
        {
            const T* s0 = slot(f - 2);
            const T* s1 = slot(f - 1);
            const T* s2 = slot(f);
            const T* s3 = slot(f + 1);
            const T* s4 = slot(f + 2);
            const T* s5 = slot(f + 3);
            // FP64: one whole cell per thread, the window's remaining cells split into single WENO
            // scalars below (the remainder would otherwise take a full second round of a few
            // warps while the others wait at the barrier: 256^3 sweeps -1.7 %; no gain for FP32)
            constexpr bool kSplit = !kMixed && kWC > kSweepThreads;
            const int c_end = kSplit ? kSweepThreads : kWC;
            for (int c = tid; c < c_end; c += kSweepThreads) {
                const int aa = c / kWB, bb = c - aa * kWB;
                if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
                T l[5], r[5];
                if constexpr (kMixed) {
                    // rho with rho u, and rho v with rho w: two WENO scalars per packed instruction
#pragma unroll
                    for (int q = 0; q < 4; q += 2) {
                        const int oa = q * kWC + c, ob = oa + kWC;
                        F2 lq, rq;
                        weno_scalar<F2>(F2(s0[oa], s0[ob]), F2(s1[oa], s1[ob]), F2(s2[oa], s2[ob]), F2(s3[oa], s3[ob]),
                                        F2(s4[oa], s4[ob]), F2(s5[oa], s5[ob]), F2(q == 0 ? eps_r : eps_m, eps_m), lq,
                                        rq);
                        l[q] = lq.lo();
                        l[q + 1] = lq.hi();
                        r[q] = rq.lo();
                        r[q + 1] = rq.hi();
                    }
                    T Tl, Tr;
                    {
                        const int o = 5 * kWC + c;
                        weno_scalar<T>(s0[o], s1[o], s2[o], s3[o], s4[o], s5[o], eps_T, Tl, Tr);
                    }
                    // both face energies, src/update.cpp:673-674, one side per lane
                    const F2 rr(l[0], r[0]), mx(l[1], r[1]), my(l[2], r[2]), mz(l[3], r[3]);
                    const F2 ke = F2(0.5f) * (mx * mx + my * my + mz * mz) / rr;
                    const F2 e = F2(rr * F2(Tl, Tr)) * F2(cv_mixed) + ke;
                    l[4] = e.lo();
                    r[4] = e.hi();
                } else {
                    // FP64: the weighted averages of rho, rho u, rho v, rho w share one division among
                    // their eight denominators (each between 20 eps^3 and about IS^3, so the
                    // product stays far inside the double range for physical states); T and the
                    // two face energies share a second one (denominators of T, rho_l, rho_r)
                    T N[5][2], D[5][2];
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        const int o = (q < 4 ? q : 5) * kWC + c;
                        weno_nd<T>(s0[o], s1[o], s2[o], s3[o], s4[o], s5[o], q == 0 ? eps_r : (q < 4 ? eps_m : eps_T),
                                   N[q][0], D[q][0], N[q][1], D[q][1]);
                    }
                    {
                        T pq[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) pq[q] = D[q][0] * D[q][1];
                        const T p01 = pq[0] * pq[1], p23 = pq[2] * pq[3];
                        const T inv = T(1) / (p01 * p23);
                        const T i01 = p23 * inv, i23 = p01 * inv;   // 1 / p01, 1 / p23
                        const T iq[4] = {pq[1] * i01, pq[0] * i01, pq[3] * i23, pq[2] * i23};
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            l[q] = N[q][0] * (D[q][1] * iq[q]);
                            r[q] = N[q][1] * (D[q][0] * iq[q]);
                        }
                    }
                    const T pT = D[4][0] * D[4][1], plr = l[0] * r[0];
                    const T inv2 = T(1) / (pT * plr);
                    const T iT = plr * inv2, ilr = pT * inv2;   // 1 / pT, 1 / (rho_l rho_r)
                    const T Tl = N[4][0] * (D[4][1] * iT), Tr = N[4][1] * (D[4][0] * iT);
                    l[4] = face_energy_ir<T>(l[0], r[0] * ilr, l[1], l[2], l[3], Tl, ph);
                    r[4] = face_energy_ir<T>(r[0], l[0] * ilr, r[1], r[2], r[3], Tr, ph);
                }
#pragma unroll
                for (int q = 0; q < 5; q++) {
                    rec[q * kWC + c] = l[q];
                    rec[(5 + q) * kWC + c] = r[q];
                }
            }
            // the window's cells beyond one per thread: one WENO scalar per work item (5 per cell,
            // T into the energy slots), then their face energies
            if constexpr (kSplit) {
                constexpr int kRest = kWC - kSweepThreads;
                for (int it = tid; it < 5 * kRest; it += kSweepThreads) {
                    const int q = it / kRest, c = kSweepThreads + (it - q * kRest);
                    const int aa = c / kWB, bb = c - aa * kWB;
                    if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
                    const int o = (q < 4 ? q : 5) * kWC + c;
                    T fl, fr;
                    weno_scalar<T>(s0[o], s1[o], s2[o], s3[o], s4[o], s5[o], q == 0 ? eps_r : (q < 4 ? eps_m : eps_T),
                                   fl, fr);
                    rec[q * kWC + c] = fl;
                    rec[(5 + q) * kWC + c] = fr;
                }
                __syncthreads();
                for (int c = kSweepThreads + tid; c < kWC; c += kSweepThreads) {
                    const int aa = c / kWB, bb = c - aa * kWB;
                    if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
                    T* lc = rec + c;
                    T* rc = rec + 5 * kWC + c;
                    lc[4 * kWC] = face_energy<T>(lc[0], lc[kWC], lc[2 * kWC], lc[3 * kWC], lc[4 * kWC], ph);
                    rc[4 * kWC] = face_energy<T>(rc[0], rc[kWC], rc[2 * kWC], rc[3 * kWC], rc[4 * kWC], ph);
                }
            }
        }
        __syncthreads();
        if (f + 1 < f_end) {
            if (use_tma) {
                if (tid == 0) {
                    // box origin: window row a0-1, column b0-1 (ghost-layout +3), normal plane f+4
                    const int cb = b0 + 2, ca = a0 + 2, cn = f + 4 + 3;
                    tma_slab_load(smem_u32(slot(f + 4)), a.tmap, cb, DIR == 0 ? cn : ca, DIR == 0 ? ca : cn,
                                  (unsigned)(5 * kWC * sizeof(double)) +
                                      ((probe && f == f_begin - 1) ? kProbeExtraBytes : 0u),
                                  bar_u32);
                }
            } else if (mtma) {
                if (tid == 0) {   // the FP64 slab of plane f+4 into the landing area, converted next face
                    const int cb = b0 + 2, ca = a0 + 2, cn = f + 4 + 3;
                    tma_slab_load(smem_u32(mland), a.tmap, cb, DIR == 0 ? cn : ca, DIR == 0 ? ca : cn,
                                  (unsigned)(5 * kWC * sizeof(double)), bar_u32);
                }
            } else if (!kMixed && !zslab) {
                issue_slab(f + 4);
            }
        }
        if (active) {
            SmemFace<DIR, T, kWC> pv;
            pv.wf = slot(f);
            pv.wf1 = slot(f + 1);
            pv.rec = rec;
            pv.c = cc;
            pv.cN = cc + Neigh<DIR>::Na * kWB + Neigh<DIR>::Nb;
            pv.cS = cc - Neigh<DIR>::Na * kWB - Neigh<DIR>::Nb;
            pv.cF = cc + Neigh<DIR>::Fa * kWB + Neigh<DIR>::Fb;
            pv.cB = cc - Neigh<DIR>::Fa * kWB - Neigh<DIR>::Fb;
            pv.inv_dx = inv_dxw;
            // collision time of the left cell, mu(T)/p (src/update.cpp:276-278)
            const T* wl = slot(f);
            T tau0;
            if constexpr (kMixed) {
                // p' = p / p0 and T' = T / T0 in the working units; tau' = tau us / dx
                const float d = wl[cc], id = 1.0f / d;
                const float u = wl[kWC + cc] * id, v = wl[2 * kWC + cc] * id, w = wl[3 * kWC + cc] * id;
                const float p = (d * float(fc.gm1)) * (wl[4 * kWC + cc] * id - 0.5f * (u * u + v * v + w * w));
                const float x = p * id;   // T / T0
                // mu(T) / p in the working units, in single precision like the flux it enters
                tau0 = fc.visc == 1 ? tc_a * powf(x, 0.76f) / p : tc_a * (x * sqrtf(x)) / ((x + tc_b) * p);
            } else if (fc.visc == 1) {
                double d = wl[cc], id = 1.0 / d;
                double u = wl[kWC + cc] * id, v = wl[2 * kWC + cc] * id, w = wl[3 * kWC + cc] * id;
                double p = (d * fc.gm1) * (wl[4 * kWC + cc] * id - 0.5 * (u * u + v * v + w * w));
                tau0 = collision_time(fc, p * id * (1.0 / kR), p);
            } else {
                // Sutherland with pd = p rho = (gamma - 1)(E rho - |m|^2 / 2): T = pd / (R rho^2) and
                // mu(T) / p = C sqrt(pd) / (pd + 110.4 R rho^2), C = mu0 (T0 + 110.4) R / (R T0)^(3/2)
                const double d = wl[cc], m1 = wl[kWC + cc], m2 = wl[2 * kWC + cc], m3 = wl[3 * kWC + cc];
                const double pd = fc.gm1 * (wl[4 * kWC + cc] * d - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3));
                tau0 = suth_c * sqrt(pd) / (pd + (110.4 * kR) * (d * d));
            }
            const long long ci = cell0 + (long long)(f + 3) * st.sn;
            // the accumulator of this cell (y, z sweeps) travels to shared memory while the flux
            // is computed (the mixed z sweep, which also re-reads the state, loads it directly:
            // measured faster there)
            constexpr bool kFetchA = DIR == 1 || (DIR == 2 && !kMixed);
            const bool fetch_a = kFetchA && f >= f_begin && !zpair;
            if (fetch_a) {
#pragma unroll
                for (int q = 0; q < 5; q++) cp_async8(&stage[q * kSweepThreads + tid], &a.A[q * nt3 + ci]);
                cp_async_commit();
            }
            T Fr[5];
            gks_flux<T>(pv, tau0, dtw, dxw, ph, Fr);
            if (fetch_a) cp_async_wait_all();
            double F[5];
#pragma unroll
            for (int q = 0; q < 5; q++) {
                if constexpr (kMixed) F[perm<DIR>(q)] = (double)Fr[q] * fc.fscale[perm<DIR>(q)];
                else F[perm<DIR>(q)] = Fr[q];
            }
            if (f >= f_begin) {
                if (DIR == 0) {
#pragma unroll
                    for (int q = 0; q < 5; q++) a.A[q * nt3 + ci] = __dsub_rn(F[q], Fprev[q]);
                } else if (DIR == 1) {
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        double acc = stage[q * kSweepThreads + tid];
                        a.A[q * nt3 + ci] = __dsub_rn(__dadd_rn(acc, F[q]), Fprev[q]);
                    }
                } else {
                    double wn[5];
                    const bool zp = zpair && paired(f);
                    // the cell's accumulator in its pair's brick, laid out [q][a][b][k & 1]
                    double* zc = stage + zbuf(f) * kZB + (ty * kTB + tx) * 2 + ((f + 3) & 1);
                    if (zp && first_of_pair(f)) {
                        if (!mbar_wait_bounded(zbar + 8u * zbuf(f), (zph >> zbuf(f)) & 1u)) atomicOr(&a.clock->status, 2);
                    }
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        double acc = zp ? zc[q * 2 * kTA * kTB]
                                        : ((kFetchA && !zpair) ? stage[q * kSweepThreads + tid] : a.A[q * nt3 + ci]);
                        double s = __dsub_rn(__dadd_rn(acc, F[q]), Fprev[q]);
                        // the cell's FP64 state (the FP64 ring holds it; the mixed ring has FP32 copies, so
                        // the mixed form reads it from the pair's state brick, or directly)
                        const double wq = kMixed ? ((sweep_state_bricks<T>() && zp) ? zc[(wbr - stage) + q * 2 * kTA * kTB]
                                                                                    : W[q * nt3 + ci])
                                                 : (double)wl[q * kWC + cc];
                        wn[q] = __dsub_rn(wq, __dmul_rn(fc.inv_dx, s));
                        if (zp) zc[q * 2 * kTA * kTB] = wn[q];
                        else a.A[q * nt3 + ci] = wn[q];
                    }
                    if (zp && !first_of_pair(f)) fence_async_shared();   // the brick's copy out reads it
                    const double ws = wave_speed_recip(wn, fc.gam, fc.gm1);
                    if (!isfinite(ws) || !(wn[0] > 0.0)) bad = true;
                    else wmax = ws > wmax ? ws : wmax;
                }
            }
#pragma unroll
            for (int q = 0; q < 5; q++) Fprev[q] = F[q];
        }
        if (zpair && f >= f_begin && first_of_pair(f) && paired(f)) zph ^= 1u << zbuf(f);
    }
    if (zpair || zslab) {
        __syncthreads();   // the last pair's writes, fenced, before its copy out
        if (tid == 0) {
            const int fl = f_end - 1;
            if (zpair && !first_of_pair(fl) && paired(fl))
                tma_box_store(a.tmap_acc, fl + 2, b0 + 3, a0 + 3, smem_u32(stage + zbuf(fl) * kZB));
            bulk_wait_all();   // every brick stored before the shared memory is reused or released
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(zbar) : "memory");
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(zbar + 8u) : "memory");
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(lbar) : "memory");
        }
    }
    if (DIR == 2) {
        double m = block_max(wmax, reinterpret_cast<double*>(rec));
        if (tid == 0 && m > 0.0) atomicMax(&a.clock->wave[a.parity ^ 1], (unsigned long long)__double_as_longlong(m));
        if (bad) atomicOr(&a.clock->status, 1);
    }
    if (use_tma || mtma) {   // every wait on the barrier has returned: retire it (a persistent CTA re-initialises it)
        __syncthreads();
        if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar_u32) : "memory");
    }
}

template <int DIR, class T, class Tile, int MM = kMapsRuntime>
__global__ void __launch_bounds__(Tile::threads, Tile::ctas) sweep_kernel(SweepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    sweep_block<DIR, T, Tile, MM>(a, blockIdx.x, blockIdx.y + a.tile_a0, blockIdx.z, smem_raw);
}

// the kernel form for the maps a launch carries (the z sweep needs the accumulator's too, the mixed
// z sweep also the state's)
template <class T>
__host__ __device__ inline bool maps_present(int dir, const SweepArgs& a)
{
    if (dir != 2) return a.tmap != nullptr;
    return a.tmap != nullptr && a.tmap_acc != nullptr && (!sweep_detail::sweep_state_bricks<T>() || a.tmap_wb != nullptr);
}
template <int DIR, class T, class Tile>
void launch_form(const SweepArgs& a, dim3 grid, dim3 block, cudaStream_t s)
{
    const size_t smem = sweep_detail::sweep_smem_bytes<T, Tile, DIR>();
    if (maps_present<T>(DIR, a)) sweep_kernel<DIR, T, Tile, kMapsOn><<<grid, block, smem, s>>>(a);
    else sweep_kernel<DIR, T, Tile, kMapsOff><<<grid, block, smem, s>>>(a);
}
template <int DIR, class T, class Tile>
cudaError_t set_form_smem()
{
    const int bytes = (int)sweep_detail::sweep_smem_bytes<T, Tile, DIR>();
    cudaError_t e = cudaFuncSetAttribute(sweep_kernel<DIR, T, Tile, kMapsOn>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sweep_kernel<DIR, T, Tile, kMapsOff>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

// Work item `item` of an ensemble sweep of direction DIR: the member it belongs to (members in the
// order order[], items from off[]), its window (bx, by) and segment bz, and the member's sweep
// arguments.  Tensor maps: 4 per buffer and window variant (x slab, y slab, z brick, z slab box) of
// the buffer read and, for the z sweep, the buffer written; `variant` 1 = 16 x 16 windows (FP64),
// 0 = the 16 x 8 windows (FP64 variant 0 and the mixed form).
template <int DIR>
__device__ __forceinline__ void ensemble_item(const MemberDev* __restrict__ mem, const long long* __restrict__ off,
                                              const long long* __restrict__ order, int nm, int parity, long long item,
                                              int variant, SweepArgs& a, int& bx, int& by, int& bz)
{
    const int pos = find_member(off, nm, item);
    const MemberDev& md = mem[order[pos]];
    const long long local = item - off[pos];
    const int nseg = md.nseg[DIR];
    const int tb = md.tiles_b[DIR];
    bz = (int)(local % nseg);
    const long long t = local / nseg;
    bx = (int)(t % tb);
    by = (int)(t / tb);
    const bool maps = md.tmaps != nullptr;
    a.tmap = maps ? md.tmaps + 128 * ((parity * kSweepVariants64 + variant) * 4 + (DIR == 2 ? 3 : DIR)) : nullptr;
    a.tmap_acc = (maps && DIR == 2) ? md.tmaps + 128 * (((parity ^ 1) * kSweepVariants64 + variant) * 4 + 2) : nullptr;
    a.tmap_wb = (maps && DIR == 2) ? md.tmaps + 128 * ((parity * kSweepVariants64 + variant) * 4 + 2) : nullptr;
    a.tile_a0 = 0;
    a.f0 = 0;
    a.f1 = 0;
    a.skip_clock_init = 0;
    a.wait_probe = 0;
    a.W = md.buf[parity];
    a.A = md.buf[parity ^ 1];
    a.fc = md.fc;
    a.clock = md.clock;
    a.parity = parity;
    a.dt_fixed_mode = md.dt_fixed_mode;
    a.dt_fixed = md.dt_fixed;
    a.seg_len = md.seg_len[DIR];
}

// Persistent form for an ensemble: a fixed grid of CTAs takes the flattened
// (member, window, segment) work list of one sweep direction item by item from
// a global counter, so a CTA that finishes early takes the next item.  Member
// m uses segments of md.seg_len[DIR] faces; the list holds the members in the
// order order[] (longest items first), off[] their work-item offsets.
template <int DIR, class T, class Tile>
__global__ void __launch_bounds__(Tile::threads, Tile::ctas)
    ensemble_sweep_kernel(const MemberDev* __restrict__ mem, const long long* __restrict__ off,
                          const long long* __restrict__ order, int nm, int parity, unsigned long long* next)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long s_item;
    const long long total = off[nm];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (;;) {
        // the previous item ended with a barrier, so every thread has read s_item before it changes
        if (tid == 0) s_item = (long long)atomicAdd(next, 1ull);
        __syncthreads();
        const long long item = s_item;
        if (item >= total) break;
        SweepArgs a;
        int bx, by, bz;
        ensemble_item<DIR>(mem, off, order, nm, parity, item, (sizeof(T) == 8 && Tile::TA == 16) ? 1 : 0, a, bx, by, bz);
        sweep_block<DIR, T, Tile>(a, bx, by, bz, smem_raw);
        __syncthreads();   // the next item reuses the shared-memory ring
    }
}

template <class T, class Tile>
cudaError_t launch_sweep_rows_t(int dir, SweepArgs a, int j0, int j1, cudaStream_t s)
{
    const int n = a.fc.n;
    if (j0 < 0 || j1 > n || j0 >= j1) return cudaErrorInvalidValue;
    const int gb = (n + Tile::TB - 1) / Tile::TB;
    const dim3 block(Tile::TB, Tile::TA);
    if (dir == 1) {
        if (a.seg_len < 1) return cudaErrorInvalidValue;
        a.f0 = j0;
        a.f1 = j1;
        const dim3 grid(gb, (n + Tile::TA - 1) / Tile::TA, (j1 - j0 + a.seg_len - 1) / a.seg_len);
        launch_form<1, T, Tile>(a, grid, block, s);
        return cudaGetLastError();
    }
    if (j0 % Tile::TA) return cudaErrorInvalidValue;
    a.tile_a0 = j0 / Tile::TA;
    const dim3 grid(gb, (j1 + Tile::TA - 1) / Tile::TA - a.tile_a0, (n + a.seg_len - 1) / a.seg_len);
    if (dir == 0) launch_form<0, T, Tile>(a, grid, block, s);
    else launch_form<2, T, Tile>(a, grid, block, s);
    return cudaGetLastError();
}

template <class T, class Tile>
cudaError_t launch_ensemble_sweep_t(int dir, const MemberDev* mem, const long long* off, const long long* order, int nm,
                                    int parity, unsigned long long* next, cudaStream_t s)
{
    const dim3 block(Tile::TB, Tile::TA);
    const int grid = 148 * Tile::ctas;
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    if (dir == 0)
        ensemble_sweep_kernel<0, T, Tile>
            <<<grid, block, sweep_detail::sweep_smem_bytes<T, Tile, 0>(), s>>>(mem, off, order, nm, parity, next);
    else if (dir == 1)
        ensemble_sweep_kernel<1, T, Tile>
            <<<grid, block, sweep_detail::sweep_smem_bytes<T, Tile, 1>(), s>>>(mem, off, order, nm, parity, next);
    else
        ensemble_sweep_kernel<2, T, Tile>
            <<<grid, block, sweep_detail::sweep_smem_bytes<T, Tile, 2>(), s>>>(mem, off, order, nm, parity, next);
    return cudaGetLastError();
}

template <class T, class Tile>
cudaError_t set_ensemble_smem()
{
    using sweep_detail::sweep_smem_bytes;
    cudaError_t e = cudaFuncSetAttribute(ensemble_sweep_kernel<0, T, Tile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sweep_smem_bytes<T, Tile, 0>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(ensemble_sweep_kernel<1, T, Tile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sweep_smem_bytes<T, Tile, 1>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(ensemble_sweep_kernel<2, T, Tile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sweep_smem_bytes<T, Tile, 2>());
    return e;
}

}  // namespace gkm
