// Internal declarations shared by the kernel files and the C-ABI layer.
// Not part of the public interface (include/gkm.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gkm {

// Device-resident clock of one run: the reference keeps dt, t and iter as
// globals (src/update.cpp:6,10); here they live in device memory so that a
// step never waits for the host.
struct DevClock {
    double dt;                   // dt of the step being taken (written by the x sweep)
    double t;                    // simulated time in the reference's accounting: after each
                                 // step it adds the dt of the NEXT step (src/update.cpp:167-168,
                                 // timestep(W); t += dt)
    long long iter;              // completed steps
    unsigned long long wave[2];  // max(|u|+c) of the current/next state, as double bits
    int status;                  // bit 0: non-finite state detected
    int pad;
};

// Physical and grid constants of one field (reference globals of src/param.h:11-27).
struct FieldConst {
    int n;          // interior cells per side
    int nt;         // n + 6
    long long nt3;  // nt^3
    int K;
    int visc;       // 0 Sutherland, 1 power law 0.76
    double gam, gm1, dx, inv_dx, mu0, T0, cfl;
    // mixed-precision working units: rho / rho0, m / (rho0 us), E / p0, T / T0,
    // lengths in dx, us = sqrt(p0 / rho0); fscale turns a non-dimensional face flux
    // (time-integrated) back into the dimensional one, per component
    double p0, u_s, inv_rho_s, inv_m_s, inv_E_s, inv_T0;
    double eps_rho, eps_m, eps_T;   // the WENO epsilon 1e-10 expressed in those units
    double fscale[5];
};

// Sweep geometry: a CTA covers a TB x TA window of faces in the plane normal
// to the sweep and marches along the normal through seg_len faces.  Each
// compute type has a small set of windows (with the CTAs per SM their register
// budget targets); gkm_autotune picks the window and the segment length per
// sweep direction by timing them on the live state.
template <int TB_, int TA_, int CTAS_>
struct SweepTile {
    static constexpr int TB = TB_;           // window width along the first in-plane axis (threadIdx.x)
    static constexpr int TA = TA_;           // window height along the second in-plane axis (threadIdx.y)
    static constexpr int WB = TB + 2;        // window incl. one neighbour face each side
    static constexpr int WA = TA + 2;
    static constexpr int WC = WA * WB;       // cells in one slab of the window
    static constexpr int threads = TA * TB;
    static constexpr int ctas = CTAS_;
};
// FP64: 16 x 8 (255 registers, two 128-thread CTAs per SM) and 16 x 16 (one 256-thread CTA)
using SweepTile64a = SweepTile<16, 8, 2>;
using SweepTile64b = SweepTile<16, 16, 1>;
// FP32: 16 x 8 (168 registers, three CTAs per SM)
using SweepTile32a = SweepTile<16, 8, 3>;
// variant 2: 16 x 16 windows, warp-specialized (a producer warpgroup reconstructs face f+1 while
// two consumer warpgroups compute the fluxes of face f; sweep_ws.cuh); ensembles: its persistent
// form for x and y
constexpr int kSweepVariants64 = 3;
constexpr int kSweepVariants32 = 1;

struct SweepShape {
    int variant;   // window variant of the compute type
    int TB, TA;    // its window
    int ctas;      // CTAs per SM it targets
};
SweepShape sweep_shape(bool mixed, int variant);
constexpr int kRing = 6;            // slabs held: the 6-cell WENO stencil
constexpr int kSlabComps = 6;       // rho, rho u, rho v, rho w, rho E, T

struct SweepArgs {
    const double* __restrict__ W;   // current state, 5 components of nt^3 (reference layout)
    double* __restrict__ A;         // accumulator; the z sweep overwrites it with the new state
    FieldConst fc;
    DevClock* clock;
    int parity;                     // wave slot holding max(|u|+c) of W
    int dt_fixed_mode;              // 1: use dt_fixed instead of cfl dx / max(|u|+c)
    double dt_fixed;
    int seg_len;                    // faces per CTA along the normal
    int tile_a0;                    // first window row (x, z sweeps) of a launch over part of the j range
    int f0, f1;                     // y sweep over part of the j range: segments start at f0 and stop
                                    // at f1 (f0 = f1 = 0: the whole normal range)
    int skip_clock_init;            // 1: the clock's dt and next wave slot were set before the launch
    const void* tmap;               // FP64: tensor map of W for the slab copies (x, y: one slab; z: two)
    const void* tmap_acc;           // z sweep: tensor map of A for the accumulator bricks (else null)
    const void* tmap_wb;            // mixed z sweep: tensor map of W for the FP64 state bricks (else null)
    int wait_probe;                 // test hook: make CTA (0, 0, 0)'s first bounded copy wait run out
};

// kernel launchers (sweep.cu); sweep_prepare sets the sweep kernels' shared-memory limit once
cudaError_t sweep_prepare();
bool ws_ready();            // the warp-specialized FP64 sweep (variant 2) may run
bool ensemble_ws_ready();   // and its persistent ensemble form (x, y)
cudaError_t launch_sweep(int dir, int variant, const SweepArgs& a, int nseg, cudaStream_t s);
// The sweep of direction dir restricted to the interior y-planes [j0, j1): window rows (x, z
// sweeps; j0 must be a multiple of the window height) or normal segments from j0 to j1 (y sweep).
// The cells updated are exactly those of planes [j0, j1).
cudaError_t launch_sweep_rows(int dir, int variant, SweepArgs a, int j0, int j1, cudaStream_t s);
cudaError_t launch_sweep_mixed_rows(int dir, int variant, SweepArgs a, int j0, int j1, cudaStream_t s);
// Ghost cells of the ghost-layout y-planes [J0, J1) (0 <= J0 < J1 <= nt) from their periodic images
cudaError_t launch_halo_planes(double* W, const FieldConst& fc, int J0, int J1, cudaStream_t s);
// the clock update that closes a step with a given dt: t += dt, iter += 1
cudaError_t launch_clock_finish(DevClock* clock, double dt, cudaStream_t s);
// the same sweeps with the reconstruction and the flux in single precision (sweep_mixed.cu)
cudaError_t launch_sweep_mixed(int dir, int variant, const SweepArgs& a, int nseg, cudaStream_t s);
cudaError_t sweep_mixed_prepare();
// ghost wrap of W; with finish_step also the clock update that closes a step:
// iter += 1 and t += the dt of the next step (wave slot `slot`, or the fixed dt)
cudaError_t launch_halo(double* W, const FieldConst& fc, DevClock* clock, int finish_step, int slot,
                        int dt_fixed_mode, double dt_fixed, cudaStream_t s);

// dt = cfl*dx/max(|u|+c) from a wave-speed slot, or the fixed dt (src/update.cpp:1053)
__device__ __forceinline__ double cfl_dt(const FieldConst& fc, const DevClock* c, int slot, int dt_fixed_mode,
                                        double dt_fixed)
{
    if (dt_fixed_mode) return dt_fixed;
    const double mw = __longlong_as_double((long long)c->wave[slot]);
    return __ddiv_rn(__dmul_rn(fc.cfl, fc.dx), mw);
}
cudaError_t launch_wave_reduce(const double* W, const FieldConst& fc, DevClock* clock, int slot, cudaStream_t s);
cudaError_t launch_flux_faces(const double* in, long long nfaces, double gam, int K, double dt, double dx,
                              double* F, cudaStream_t s);
cudaError_t launch_weno_faces(const double* stencils, long long n, double gam, double* Wl, double* Wr,
                              cudaStream_t s);

// Lagrangian side (lagrangian.cu)
struct SplineGrid {
    int npts;        // data points per axis
    int pad;         // 2 natural, 3 periodic
    int periodic;
    double start, dinv;
};

struct SplineTables {
    const double* mt;    // Thomas multipliers, length npts+1
    const double* dp;    // Thomas pivots
    const double* z;     // periodic correction vector (periodic only)
    double denom;        // periodic Sherman-Morrison denominator
};

cudaError_t launch_spline_build(const double* W, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                double* coef_u, double* coef_v, double* coef_w, double* scratch, cudaStream_t s);
cudaError_t launch_spline_component(const double* W, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                    int component, double* coef, double* scratch, cudaStream_t s);
cudaError_t launch_particles_eval(const double* const coefs[3], const SplineGrid& g, long long np,
                                  const double* py, const double* px, const double* pz,
                                  double* Uu, double* Uv, double* Uw, cudaStream_t s);
// FP32 velocity splines: the three components' coefficients rounded to float after the same FP64
// line solves (buf: M^2 N doubles, the handle's spline scratch); evaluation reads them as floats
// and computes in FP64
cudaError_t launch_spline_build_f32(const double* W, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                    float* coef_u, float* coef_v, float* coef_w, double* buf, cudaStream_t s);
cudaError_t launch_particles_eval(const float* const coefs[3], const SplineGrid& g, long long np,
                                  const double* py, const double* px, const double* pz,
                                  double* Uu, double* Uv, double* Uw, cudaStream_t s);
struct ParticleArrays {   // y, x, z, u, v, w
    double* a[6];
};
cudaError_t launch_particles_heun(const double* const coefs[3], const SplineGrid& g, const DevClock* clock,
                                  long long np, const ParticleArrays& src, const ParticleArrays& dst,
                                  const long long* tag_src, long long* tag_dst, cudaStream_t s);
cudaError_t launch_particles_heun(const float* const coefs[3], const SplineGrid& g, const DevClock* clock,
                                  long long np, const ParticleArrays& src, const ParticleArrays& dst,
                                  const long long* tag_src, long long* tag_dst, cudaStream_t s);
// order the particles of src by blocks of 8^3 spline cells into dst (tags move with them);
// keys: np values, counts: ((npts + 7) / 8)^3, temp: scan_temp_size(counts) values
int scan_temp_size(long long n);
cudaError_t launch_particle_sort(const SplineGrid& g, long long np, const ParticleArrays& src, const ParticleArrays& dst,
                                 const long long* tag_src, long long* tag_dst, unsigned* keys, unsigned* counts,
                                 unsigned* temp, int* launches, cudaStream_t s);

struct StatsPartial {  // per-CTA partial sums of the PrintStats moments
    double v[16];
};

// particle properties (getParticleProp) and their statistics (GetParticleStats)
constexpr int kPropCount = 41;
constexpr int kSplineDensity = 0, kSplinePressure = 4, kSplinePlain = 5;   // launch_spline_source kinds (1..3 velocity)
cudaError_t launch_spline_source(const double* src, const FieldConst& fc, const SplineGrid& g, const SplineTables& tb,
                                 int kind, double* coef, double* scratch, cudaStream_t s);
cudaError_t launch_lap_nodes(const double* coef, const SplineGrid& g, const FieldConst& fc, double* out, cudaStream_t s);
cudaError_t launch_particle_props(const double* const coefs[8], const SplineGrid& g, long long np, const double* py,
                                  const double* px, const double* pz, double* props, cudaStream_t s);
cudaError_t launch_particle_stats(const double* props, long long np, StatsPartial* partials, int nblocks, double* out6,
                                  cudaStream_t s);
cudaError_t launch_stats(const double* W, const FieldConst& fc, const SplineGrid& g, const double* const coefs[3],
                         StatsPartial* partials, int nblocks, double* out16, cudaStream_t s);
cudaError_t launch_stats(const double* W, const FieldConst& fc, const SplineGrid& g, const float* const coefs[3],
                         StatsPartial* partials, int nblocks, double* out16, cudaStream_t s);

// ---------------------------------------------------------------- ensemble --
// Independent members (own grid size, parameters, state, splines, particles)
// advanced by shared launches: each launch walks a flattened work list whose
// per-member prefix offsets find the member of a work index.
struct MemberDev {
    double* buf[2];      // state buffers (current state = buf[parity])
    DevClock* clock;
    FieldConst fc;
    int dt_fixed_mode;
    double dt_fixed;
    int nseg[3];         // sweep segments along the normal, per direction
    int seg_len[3];      // faces per segment along the normal, per direction (chosen per member size)
    int tiles_b[3];      // windows along the first in-plane axis, per direction
    SplineGrid grid;
    SplineTables tb;
    double* coef[3];
    double* scratch[3];
    double* P[6];        // particles y, x, z, u, v, w
    long long np;
    // the member's tensor maps of its two state buffers for the FP64 x / y sweeps (the single
    // cube's table: index (buffer * kSweepVariants64 + variant) * 2 + direction), or null
    const unsigned char* tmaps;
};

struct EnsembleWork {           // prefix offsets, nm + 1 entries each, in device memory
    const long long* item[3];   // sweep work items per direction
    const long long* ghost;     // ghost cells
    const long long* line0;     // spline pass-0 lines of the 3 components
    const long long* line1;     // spline pass-1 lines of the 3 components
    const long long* warp2;     // spline pass-2 groups of 32 lines, 3 components
    const long long* part;      // particles
};

// largest m with off[m] <= idx (off[0] = 0, off[nm] = total)
__device__ __forceinline__ int find_member(const long long* __restrict__ off, int nm, long long idx)
{
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= idx) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// One sweep direction over all members: off[] are the prefix offsets of the members' work items in
// the order order[] (position -> member); CTAs fetch items from *next (zero before the launch), so
// the list is taken in order, its longest items first when order[] sorts them so.
cudaError_t launch_ensemble_sweep64(int dir, int variant, const MemberDev* mem, const long long* off,
                                    const long long* order, int nm, int parity, unsigned long long* next,
                                    cudaStream_t s);
cudaError_t launch_ensemble_sweep32(int dir, int variant, const MemberDev* mem, const long long* off,
                                    const long long* order, int nm, int parity, unsigned long long* next,
                                    cudaStream_t s);
cudaError_t launch_ensemble_halo(const MemberDev* mem, const long long* off, int nm, long long total, int buf,
                                 int finish_step, cudaStream_t s);
cudaError_t launch_ensemble_splines(const MemberDev* mem, const EnsembleWork& w, const long long totals[3], int nm,
                                    int buf, cudaStream_t s);
cudaError_t launch_ensemble_heun(const MemberDev* mem, const long long* off, int nm, long long total, cudaStream_t s);

// Thomas tables of the spline line solves (gkm_capi.cu)
void spline_line_tables(int N, int periodic, double* mt, double* dp, double* z, double* denom);

// FMA throughput probe (probe.cu)
cudaError_t probe_fma_peak(double* fp64_tflops, double* fp32_tflops);

}  // namespace gkm
