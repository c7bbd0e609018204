// Warp-specialized FP64 sweep (window variant 2: 16 x 16 faces, one CTA per SM).
//
// The plain sweep (sweep_impl.cuh) alternates, for every face plane, a
// reconstruction phase and a flux phase separated by barriers, so while its
// eight warps reconstruct no flux is computed and the FP64 pipe idles on the
// reconstructions' dependency chains.  Here one warpgroup (the producer) moves
// the slabs and reconstructs face f+1 while two warpgroups (the consumers, one
// face each per thread) compute the fluxes of face f:
//   producer, face f: slab f+3 landed (temperatures of its cells), wait until
//     the consumers released the reconstruction buffer of face f-2, reconstruct
//     face f into that buffer, arrive on its "full" barrier, then issue the copy
//     of slab f+4 into the ring slot of slab f-2 (read last by face f's
//     reconstructions and by the consumers' flux of face f-2);
//   consumers, face f: wait for the buffer's "full" barrier, flux of face f from
//     the buffer and slabs f, f+1, accumulate, arrive on the buffer's "empty"
//     barrier.
// The arithmetic of each face is the plain sweep's (the same reconstruction and
// flux code; every window cell takes the whole-cell reconstruction with shared
// divisions, where the plain 16 x 16 sweep splits its last cells into single
// WENO scalars, so the two differ by rounding only).  Registers: the CTA is
// launched with 384 threads at 168 registers; setmaxnreg moves the producer
// warpgroup to 104 and the consumer warpgroups to 200, which the launch's 64,512
// registers cover exactly, so the host launches this kernel only when it was
// compiled to 168 registers (ws_ready()).  Every wait is bounded; one that runs
// out raises bit 1 of the clock's status word.  Measured at 256^3: x and y
// sweeps 4.5 % and 3 % faster than the plain 16 x 16 sweep; the z sweep, whose
// producer moves each slab with per-element cp.async, 16 % slower (the
// autotuner keeps the plain kernel there).
#pragma once

#include "sweep_impl.cuh"

namespace gkm {
namespace sweep_ws_detail {

constexpr int kConsumers = 256;             // 16 x 16 faces, one per consumer thread
constexpr int kProducers = 128;             // one warpgroup
constexpr int kThreads = kConsumers + kProducers;
// 2 x 128 x 200 + 128 x 104 = 384 x 168.  Measured at 256^3 (x / y sweep, ms): 216 / 72 4.75 / 4.75,
// 208 / 88 4.57 / 4.67, 200 / 104 4.34 / 4.50, 192 / 120 5.75 / 6.20; the plain 16 x 16 sweep 4.55 / 4.65
constexpr int kConsumerRegs = 200, kProducerRegs = 104;
static_assert(2 * 128 * kConsumerRegs + 128 * kProducerRegs <= kThreads * 168, "register split above the launch's");

// named barriers (0 is __syncthreads)
__device__ __forceinline__ void producer_sync() { asm volatile("bar.sync 1, %0;\n" ::"n"(kProducers) : "memory"); }
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 2, %0;\n" ::"n"(kConsumers) : "memory"); }

__device__ __forceinline__ void mbar_init_count(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

template <class Tile>
__host__ __device__ constexpr size_t ws_smem_bytes()
{
    // the ring and one reconstruction buffer as the plain sweep lays them out, a second
    // reconstruction buffer, the consumers' accumulator staging, five mbarriers
    return sweep_detail::sweep_ring_bytes<double, Tile>() + sizeof(double) * 10 * (size_t)Tile::WC +
           sizeof(double) * 5 * (size_t)kConsumers + 5 * 8;
}

}  // namespace sweep_ws_detail

// the mbarriers of a warp-specialized CTA (after its ring, reconstruction buffers and staging):
// [0] slab copies, [1..2] "full", [3..4] "empty"
template <class Tile>
__device__ __forceinline__ unsigned ws_bars(unsigned char* smem_raw)
{
    using namespace sweep_detail;
    const double* stage = reinterpret_cast<const double*>(smem_raw + sweep_ring_bytes<double, Tile>() +
                                                          sizeof(double) * 10 * Tile::WC);
    return smem_u32(stage + 5 * sweep_ws_detail::kConsumers);
}
__device__ __forceinline__ void ws_init_bars(unsigned bar_tma)
{
    using namespace sweep_ws_detail;
    mbar_init_count(bar_tma, 1);
    for (int b = 0; b < 2; b++) {
        mbar_init_count(bar_tma + 8 + 8 * b, kProducers);
        mbar_init_count(bar_tma + 24 + 8 * b, kConsumers);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void ws_inval_bars(unsigned bar_tma)
{
    for (int b = 0; b < 5; b++) asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar_tma + 8 * b) : "memory");
}

// ROLE 0: the whole CTA (the single-cube kernel: barrier set-up, the register split, both warpgroup
// roles, barrier retirement).  ROLE 1 / 2: only the producer / consumer part of one work item, for a
// persistent kernel whose warpgroups have split their registers once and set up the barriers.
template <int DIR, class Tile, int MM, int ROLE = 0>
__device__ __forceinline__ void sweep_block_ws(const SweepArgs& a, int bx, int by, int bz, unsigned char* smem_raw)
{
    using namespace sweep_detail;
    using namespace sweep_ws_detail;
    static_assert(Tile::TB == 16 && Tile::TA == 16, "the warp-specialized sweep covers 16 x 16 windows");
    using T = double;
    constexpr int kTB = Tile::TB, kWB = Tile::WB, kWC = Tile::WC;
    constexpr int kSlot = slot_elems<T, Tile>();
    T* ring = reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    T* rec0 = ring + kRing * kSlot;   // two buffers [2][10][kWC]
    double* stage = reinterpret_cast<double*>(smem_raw + sweep_ring_bytes<T, Tile>() + sizeof(double) * 10 * kWC);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(stage + 5 * kConsumers);
    const unsigned bar_tma = smem_u32(bars);
    const unsigned bar_full0 = smem_u32(bars + 1), bar_empty0 = smem_u32(bars + 3);   // [2] each
    const FieldConst& fc = a.fc;
    const int n = fc.n, nt = fc.nt;
    const long long nt3 = fc.nt3;
    const Strides st = strides<DIR>(nt);
    const int tid = threadIdx.x;
    const int b0 = bx * kTB, a0 = by * Tile::TA;
    const int f_begin = a.f0 + bz * a.seg_len;
    const int f_end = min(f_begin + a.seg_len, a.f1 > 0 ? a.f1 : n);
    const double dt = step_dt(a);
    const Phys<T> ph{fc.gam, fc.gm1, kR, fc.K};
    const double* __restrict__ W = a.W;
    const double suth_c = fc.mu0 * (fc.T0 + 110.4) * kR / ((kR * fc.T0) * sqrt(kR * fc.T0));

    if (DIR == 0 && bx == 0 && by == 0 && bz == 0 && tid == 0 && !a.skip_clock_init) {
        a.clock->wave[a.parity ^ 1] = 0ull;   // the z sweep of this step reduces into it
        a.clock->dt = dt;
    }
    if (f_begin >= f_end) return;

    const bool use_tma = DIR != 2 && (MM == kMapsOn || (MM == kMapsRuntime && a.tmap != nullptr));
    if constexpr (ROLE == 0) {
        if (tid == 0) ws_init_bars(bar_tma);
        __syncthreads();
    }

    auto slot = [&](int f) { return ring + ((f + 12) % kRing) * kSlot; };
    auto recb = [&](int k) { return rec0 + (k & 1) * (10 * kWC); };   // face f_begin - 1 + k
    const int nf = f_end - f_begin + 1;                                   // faces f_begin-1 .. f_end-1
    bool timed_out = false;

    if (ROLE == 1 || (ROLE == 0 && tid >= kConsumers)) {
      if constexpr (ROLE != 2) {
        // ------------------------------------------------------------------ producer
        if constexpr (ROLE == 0) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kProducerRegs));
        const int ptid = tid - kConsumers;
        const bool probe = use_tma && a.wait_probe && bx == 0 && by == 0 && bz == 0;
        unsigned tma_phase = 0;
        auto issue_slab = [&](int f) {
            double* dst = slot(f);
            for (int c = ptid; c < kWC; c += kProducers) {
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
            for (int c = ptid; c < kWC; c += kProducers) {
                const int aa = c / kWB, bb = c - aa * kWB;
                if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
                s[5 * kWC + c] = temperature<T>(s[c], s[kWC + c], s[2 * kWC + c], s[3 * kWC + c], s[4 * kWC + c], ph);
            }
        };
        if (use_tma) {   // the segment's first six slabs as six bulk tensor copies on one barrier phase
            if (ptid == 0) {
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar_tma),
                             "r"((unsigned)(6 * 5 * kWC * sizeof(double)))
                             : "memory");
                for (int f = f_begin - 3; f < f_begin + 3; f++)
                    tma_box_load(smem_u32(slot(f)), a.tmap, b0 + 2, DIR == 0 ? f + 3 : a0 + 2, DIR == 0 ? a0 + 2 : f + 3,
                                 bar_tma);
            }
            if (!mbar_wait_bounded(bar_tma, tma_phase)) timed_out = true;
            tma_phase ^= 1u;
            for (int f = f_begin - 3; f < f_begin + 3; f++) finish_slab(f);
        } else {   // per-element cp.async, one wait for all six
            for (int f = f_begin - 3; f < f_begin + 3; f++) issue_slab(f);
            cp_async_wait_all();
            for (int f = f_begin - 3; f < f_begin + 3; f++) finish_slab(f);
        }
        for (int k = 0; k < nf; k++) {
            const int f = f_begin - 1 + k;
            if (k > 0) {   // slab f + 3, issued at the end of the previous face
                if (use_tma) {
                    if (probe && k == 1) {
                        if (!mbar_wait_bounded(bar_tma, tma_phase, kProbePolls)) timed_out = true;
                        if (ptid == 0) mbar_complete_tx(bar_tma, kProbeExtraBytes);
                    }
                    if (!mbar_wait_bounded(bar_tma, tma_phase)) timed_out = true;
                    tma_phase ^= 1u;
                } else {
                    cp_async_wait_all();
                }
                finish_slab(f + 3);
            }
            producer_sync();   // every cell of slab f + 3 complete for every producer thread
            if (k >= 2 && !mbar_wait_bounded(bar_empty0 + 8 * (k & 1), ((k >> 1) - 1) & 1u)) timed_out = true;
            // reconstruct face f once per window cell (five WENO scalars, one division shared by rho and the
            // momenta, one by T and the face energies), as the plain sweep's FP64 reconstruction
            {
                T* rec = recb(k);
                const T* s0 = slot(f - 2);
                const T* s1 = slot(f - 1);
                const T* s2 = slot(f);
                const T* s3 = slot(f + 1);
                const T* s4 = slot(f + 2);
                const T* s5 = slot(f + 3);
                for (int c = ptid; c < kWC; c += kProducers) {
                    const int aa = c / kWB, bb = c - aa * kWB;
                    if (a0 + aa - 1 > n || b0 + bb - 1 > n) continue;
                    T l[5], r[5];
                    T N[5][2], D[5][2];
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        const int o = (q < 4 ? q : 5) * kWC + c;
                        weno_nd<T>(s0[o], s1[o], s2[o], s3[o], s4[o], s5[o], kWenoEps, N[q][0], D[q][0], N[q][1],
                                   D[q][1]);
                    }
                    {
                        T pq[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) pq[q] = D[q][0] * D[q][1];
                        const T p01 = pq[0] * pq[1], p23 = pq[2] * pq[3];
                        const T inv = T(1) / (p01 * p23);
                        const T i01 = p23 * inv, i23 = p01 * inv;
                        const T iq[4] = {pq[1] * i01, pq[0] * i01, pq[3] * i23, pq[2] * i23};
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            l[q] = N[q][0] * (D[q][1] * iq[q]);
                            r[q] = N[q][1] * (D[q][0] * iq[q]);
                        }
                    }
                    const T pT = D[4][0] * D[4][1], plr = l[0] * r[0];
                    const T inv2 = T(1) / (pT * plr);
                    const T iT = plr * inv2, ilr = pT * inv2;
                    const T Tl = N[4][0] * (D[4][1] * iT), Tr = N[4][1] * (D[4][0] * iT);
                    l[4] = face_energy_ir<T>(l[0], r[0] * ilr, l[1], l[2], l[3], Tl, ph);
                    r[4] = face_energy_ir<T>(r[0], l[0] * ilr, r[1], r[2], r[3], Tr, ph);
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        rec[q * kWC + c] = l[q];
                        rec[(5 + q) * kWC + c] = r[q];
                    }
                }
            }
            mbar_arrive(bar_full0 + 8 * (k & 1));
            producer_sync();   // face f's reconstructions read slab f - 2 for the last time
            if (f + 1 < f_end) {
                if (use_tma) {
                    if (ptid == 0) {
                        const int cb = b0 + 2, ca = a0 + 2, cn = f + 4 + 3;
                        tma_slab_load(smem_u32(slot(f + 4)), a.tmap, cb, DIR == 0 ? cn : ca, DIR == 0 ? ca : cn,
                                      (unsigned)(5 * kWC * sizeof(double)) + ((probe && k == 0) ? kProbeExtraBytes : 0u),
                                      bar_tma);
                    }
                } else {
                    issue_slab(f + 4);
                }
            }
        }
        if (timed_out) atomicOr(&a.clock->status, 2);
      }
    } else {
      if constexpr (ROLE != 1) {
        // ------------------------------------------------------------------ consumers
        if constexpr (ROLE == 0) asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kConsumerRegs));
        const int tx = tid % kTB, ty = tid / kTB;
        const bool active = (a0 + ty < n) && (b0 + tx < n);
        const int cc = (ty + 1) * kWB + (tx + 1);
        const long long cell0 = (a0 + ty + 3) * st.sA + (b0 + tx + 3) * st.sB;
        double Fprev[5] = {0, 0, 0, 0, 0};
        double wmax = 0.0;
        bool bad = false;
        for (int k = 0; k < nf; k++) {
            const int f = f_begin - 1 + k;
            if (!mbar_wait_bounded(bar_full0 + 8 * (k & 1), (k >> 1) & 1u)) timed_out = true;
            if (active) {
                SmemFace<DIR, T, kWC> pv;
                pv.wf = slot(f);
                pv.wf1 = slot(f + 1);
                pv.rec = recb(k);
                pv.c = cc;
                pv.cN = cc + Neigh<DIR>::Na * kWB + Neigh<DIR>::Nb;
                pv.cS = cc - Neigh<DIR>::Na * kWB - Neigh<DIR>::Nb;
                pv.cF = cc + Neigh<DIR>::Fa * kWB + Neigh<DIR>::Fb;
                pv.cB = cc - Neigh<DIR>::Fa * kWB - Neigh<DIR>::Fb;
                pv.inv_dx = fc.inv_dx;
                const T* wl = slot(f);
                T tau0;
                if (fc.visc == 1) {
                    double d = wl[cc], id = 1.0 / d;
                    double u = wl[kWC + cc] * id, v = wl[2 * kWC + cc] * id, w = wl[3 * kWC + cc] * id;
                    double p = (d * fc.gm1) * (wl[4 * kWC + cc] * id - 0.5 * (u * u + v * v + w * w));
                    tau0 = collision_time(fc, p * id * (1.0 / kR), p);
                } else {
                    const double d = wl[cc], m1 = wl[kWC + cc], m2 = wl[2 * kWC + cc], m3 = wl[3 * kWC + cc];
                    const double pd = fc.gm1 * (wl[4 * kWC + cc] * d - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3));
                    tau0 = suth_c * sqrt(pd) / (pd + (110.4 * kR) * (d * d));
                }
                const long long ci = cell0 + (long long)(f + 3) * st.sn;
                constexpr bool kFetchA = DIR != 0;
                const bool fetch_a = kFetchA && f >= f_begin;
                if (fetch_a) {
#pragma unroll
                    for (int q = 0; q < 5; q++) cp_async8(&stage[q * kConsumers + tid], &a.A[q * nt3 + ci]);
                    cp_async_commit();
                }
                T F[5], Fr[5];
                gks_flux<T>(pv, tau0, T(dt), T(fc.dx), ph, Fr);
                if (fetch_a) cp_async_wait_all();
#pragma unroll
                for (int q = 0; q < 5; q++) F[perm<DIR>(q)] = Fr[q];
                if (f >= f_begin) {
                    if (DIR == 0) {
#pragma unroll
                        for (int q = 0; q < 5; q++) a.A[q * nt3 + ci] = __dsub_rn(F[q], Fprev[q]);
                    } else if (DIR == 1) {
#pragma unroll
                        for (int q = 0; q < 5; q++) {
                            const double acc = stage[q * kConsumers + tid];
                            a.A[q * nt3 + ci] = __dsub_rn(__dadd_rn(acc, F[q]), Fprev[q]);
                        }
                    } else {
                        double wn[5];
#pragma unroll
                        for (int q = 0; q < 5; q++) {
                            const double acc = stage[q * kConsumers + tid];
                            const double s = __dsub_rn(__dadd_rn(acc, F[q]), Fprev[q]);
                            wn[q] = __dsub_rn((double)wl[q * kWC + cc], __dmul_rn(fc.inv_dx, s));
                            a.A[q * nt3 + ci] = wn[q];
                        }
                        const double ws = wave_speed_recip(wn, fc.gam, fc.gm1);
                        if (!isfinite(ws) || !(wn[0] > 0.0)) bad = true;
                        else wmax = ws > wmax ? ws : wmax;
                    }
                }
#pragma unroll
                for (int q = 0; q < 5; q++) Fprev[q] = F[q];
            }
            mbar_arrive(bar_empty0 + 8 * (k & 1));
        }
        if (DIR == 2) {   // max |u| + c over the consumers: warp shuffles, then the warp maxima in order
            double v = wmax;
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            double* red = stage;   // every consumer has read its staged accumulator
            consumer_sync();
            if ((tid & 31) == 0) red[tid >> 5] = v;
            consumer_sync();
            if (tid == 0) {
                for (int w = 1; w < kConsumers / 32; w++) v = fmax(v, red[w]);
                if (v > 0.0) atomicMax(&a.clock->wave[a.parity ^ 1], (unsigned long long)__double_as_longlong(v));
            }
            if (bad) atomicOr(&a.clock->status, 1);
        }
        if (timed_out) atomicOr(&a.clock->status, 2);
      }
    }
    if constexpr (ROLE == 0) {
        __syncthreads();   // every wait has returned: retire the barriers
        if (tid == 0) ws_inval_bars(bar_tma);
    }
}

// MM: compiled for tensor copies of the slabs (x, y sweeps with maps) or per-element copies
template <int DIR, class Tile, int MM>
__global__ void __launch_bounds__(sweep_ws_detail::kThreads, 1) sweep_ws_kernel(SweepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    sweep_block_ws<DIR, Tile, MM>(a, blockIdx.x, blockIdx.y + a.tile_a0, blockIdx.z, smem_raw);
}

// Persistent warp-specialized form for an ensemble (x, y sweeps, 16 x 16 windows): one CTA per SM takes
// (member, window, segment) items from the work counter as ensemble_sweep_kernel does.  Each warpgroup
// splits its registers once and then runs its own loop over the items, so no code is shared between
// the two register budgets; per item, consumer thread 0 takes the item and sets up fresh barriers,
// a CTA barrier publishes both, and a second one closes the item.
template <int DIR, class Tile>
__global__ void __launch_bounds__(sweep_ws_detail::kThreads, 1)
    ensemble_ws_kernel(const MemberDev* __restrict__ mem, const long long* __restrict__ off,
                       const long long* __restrict__ order, int nm, int parity, unsigned long long* next)
{
    using namespace sweep_ws_detail;
    static_assert(DIR != 2, "the z sweep's persistent ensemble form is the plain kernel");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long s_item;
    const long long total = off[nm];
    const unsigned bars = ws_bars<Tile>(smem_raw);
    if (threadIdx.x >= kConsumers) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kProducerRegs));
        for (;;) {
            __syncthreads();   // the item and its barriers are set
            const long long item = s_item;
            if (item >= total) break;
            SweepArgs a;
            int bx, by, bz;
            ensemble_item<DIR>(mem, off, order, nm, parity, item, 1, a, bx, by, bz);
            sweep_block_ws<DIR, Tile, kMapsRuntime, 1>(a, bx, by, bz, smem_raw);
            __syncthreads();   // the item is done
        }
    } else {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kConsumerRegs));
        for (;;) {
            if (threadIdx.x == 0) {
                s_item = (long long)atomicAdd(next, 1ull);
                ws_init_bars(bars);
            }
            __syncthreads();
            const long long item = s_item;
            if (item >= total) break;
            SweepArgs a;
            int bx, by, bz;
            ensemble_item<DIR>(mem, off, order, nm, parity, item, 1, a, bx, by, bz);
            sweep_block_ws<DIR, Tile, kMapsRuntime, 2>(a, bx, by, bz, smem_raw);
            __syncthreads();
            if (threadIdx.x == 0) ws_inval_bars(bars);   // every wait of the item has returned
        }
        if (threadIdx.x == 0) ws_inval_bars(bars);
    }
}

}  // namespace gkm
