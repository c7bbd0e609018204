/*
 * gkm.h — C ABI of the B200-native DNS_GKM_LPT step (libgkm_b200.so).
 *
 * Drop-in boundary for the reference's hot path: the compressible
 * decaying-isotropic-turbulence step (WENO-SYMOO reconstruction, gas-kinetic
 * flux, conservative update, dt / TKE / dissipation reductions) and the
 * Lagrangian-particle step (velocity splines, tricubic evaluation, Heun
 * advection) of nishantp9/DNS_GKM_LPT.  Plain pointers and sizes only.
 *
 * Data layout at this boundary is the reference's own (src/param.h:26,40-41):
 * five FP64 arrays W[q], q = rho, rho u, rho v, rho w, rho E, each of
 * nt^3 = (n+6)^3 values, index (j*nt + i)*nt + k with j = y, i = x, k = z
 * (z fastest), three ghost layers on each side.  Particle positions are
 * (y, x, z) and velocities (u, v, w) per particle, as in class Particle
 * (src/ParticleTrack.h:14-36).
 *
 * Every call returns gkm_status; GKM_OK is 0.  Nothing calls exit().  A handle
 * owns all its device memory and one CUDA stream; host arrays stay owned by
 * the caller and are touched only inside the call that receives them.  A
 * handle is not thread-safe; independent handles are.
 */
#ifndef GKM_B200_H
#define GKM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GKM_ABI_VERSION 1

typedef enum gkm_status {
    GKM_OK = 0,
    GKM_ERR_ARG = 1,        /* a null pointer, a size out of range, an unknown enum */
    GKM_ERR_CONFIG = 2,     /* the configuration is not supported */
    GKM_ERR_CUDA = 3,       /* a CUDA call failed; gkm_last_error() has the text */
    GKM_ERR_NONFINITE = 4,  /* the state holds NaN/Inf or non-positive density */
    GKM_ERR_STATE = 5,      /* call out of order (e.g. step before upload) */
    GKM_ERR_NOMEM = 6       /* device allocation failed */
} gkm_status;

typedef enum gkm_visc_law {
    GKM_VISC_SUTHERLAND = 0, /* mu0 (T/T0)^1.5 (T0+110.4)/(T+110.4), src/update.cpp:277 */
    GKM_VISC_POWER076 = 1    /* mu0 (T/T0)^0.76 */
} gkm_visc_law;

typedef enum gkm_spline_mode {
    GKM_SPLINE_NATURAL_GHOST3 = 0, /* the reference's grid: nt points, natural ends (src/Interpolation.cpp:3-31) */
    GKM_SPLINE_PERIODIC = 1        /* n interior cell centres, periodic */
} gkm_spline_mode;

typedef enum gkm_spline_precision {
    GKM_SPLINE_COEF_FP64 = 0, /* velocity-spline coefficients stored in FP64 (the reference's double) */
    GKM_SPLINE_COEF_FP32 = 1  /* the same FP64 line solves, coefficients stored rounded to FP32 and
                                 read as floats by the tricubic evaluation (FP64 arithmetic): half the
                                 coefficient memory and gather traffic; no counterpart in the reference */
} gkm_spline_precision;

typedef enum gkm_precision {
    GKM_PREC_FP64 = 0, /* FP64 everywhere (the reference's ptype = double) */
    GKM_PREC_MIXED = 1 /* WENO + gas-kinetic flux in FP32 on non-dimensional values; BGK time
                          coefficients, flux differences, the update, dt and all reductions in FP64 */
} gkm_precision;

/* Contents of InitialConditions/params, read by GetParams (src/FlowField.cpp:9-58). */
typedef struct gkm_params {
    int32_t n;      /* cells per side (nc) */
    int32_t pad_;
    double gam;     /* ratio of specific heats */
    double den0;    /* reference density */
    double Mt;      /* turbulent Mach number */
    double Re;      /* Taylor Reynolds number */
    double mu0;     /* reference viscosity */
    double p0;      /* reference pressure */
    double t0;      /* eddy turnover time */
} gkm_params;

typedef struct gkm_config {
    gkm_params params;
    double cfl;              /* the reference fixes 0.10 at compile time (src/param.h:20) */
    int32_t visc_law;        /* gkm_visc_law */
    int32_t spline_mode;     /* gkm_spline_mode */
    int32_t precision;       /* gkm_precision */
    int32_t device;          /* CUDA device ordinal */
    int64_t max_particles;   /* capacity of the particle arrays */
    int32_t use_graphs;      /* 1: replay each step as a captured CUDA graph */
    int32_t spline_build;    /* velocity splines: 0 auto, 1 one component per launch, 2 each pass
                                for all three components in one launch (two more scratch
                                arrays; auto picks it for grids up to about 440^3); same bits */
    int32_t test_wait_probe; /* failure-detection test hook (no reference counterpart), 0 = off.
                                1: in every FP64 x / y sweep launch that lands its slabs by bulk
                                tensor copy, the first CTA arms its first copy's barrier with 16
                                bytes more than the copy delivers and polls it 256 times, so that
                                bounded wait runs out and raises the status the host reports as
                                GKM_ERR_CUDA; the CTA then retires the extra bytes and waits for
                                the copy, so results are unchanged and nothing stays in flight */
    int32_t spline_precision; /* gkm_spline_precision.  With FP32 coefficients the splines are built
                                 one component at a time in one FP64 buffer of (N+P)^2 N values
                                 (besides the 3 (N+P)^3 floats); particle properties (gkm_particle_props
                                 and what uses them) need FP64 coefficients and return GKM_ERR_CONFIG */
    int32_t reserved[4];
} gkm_config;

/* One PrintStats line (src/update.cpp:835-840), field part. */
typedef struct gkm_stats {
    double t_over_t0, TKE, Diss, SijSij;
    double SKEWu, SKEWv, SKEWw, KURTu, KURTv, KURTw;
    double Prms, Trms, Vrms;
} gkm_stats;

typedef struct gkm_handle gkm_handle;

/* ---------------------------------------------------------------- life cycle */

/* Defaults: cfl 0.10, Sutherland, natural_ghost3, FP64, device 0, graphs on. */
void gkm_config_default(gkm_config* cfg);

/* Replaces GetParams + segment + MAKE5s + DevAlloc::DevAlloc
 * (src/FlowField.cpp:9-58,275-284; src/Main.cpp:36; src/GPUAlloc.cu:3-68)
 * for a single-GPU run with the whole periodic cube on one device. */
gkm_status gkm_create(const gkm_config* cfg, gkm_handle** out);
/* Releases everything the handle owns (DevAlloc::~DevAlloc, src/GPUAlloc.cu:70-132). */
gkm_status gkm_destroy(gkm_handle* h);
/* Text of the last error on this handle (never NULL). */
const char* gkm_last_error(const gkm_handle* h);
int gkm_abi_version(void);
/* Cells per side including ghosts (nt = n + 6), the extent of every W array. */
int gkm_nt(const gkm_handle* h);

/* ------------------------------------------------------------- field state */

/* Host -> device copy of the conserved state in the reference layout, then
 * the periodic ghost wrap and the dt reduction.  Replaces the H2D half of
 * evolve() (src/GPUupdate.cu:89-93) and Initialize_DHIT's result
 * (src/FlowField.cpp:60-114).  Ghost values in W may be stale.  The W[q]
 * may also be device pointers (unified addressing picks the copy direction),
 * e.g. an initial field generated on the GPU. */
gkm_status gkm_upload_state(gkm_handle* h, const double* const W[5]);
/* Device -> host copy (ghosts included, already wrapped); D2H half of evolve()
 * (src/GPUupdate.cu:209-213).  Device destination pointers work as well. */
gkm_status gkm_download_state(gkm_handle* h, double* const W[5]);

/* timestep(W) (src/update.cpp:1031-1054): dt = cfl*dx / max(|u| + c) of the
 * current state; also makes that dt the one the next step uses. */
gkm_status gkm_timestep(gkm_handle* h, double* dt_out);
/* Fix dt for the following steps (dt > 0) or return to the CFL rule (dt == 0). */
gkm_status gkm_set_dt(gkm_handle* h, double dt);

/* nsteps x { evolveEulerian; HaloTransfer; timestep }
 * (src/update.cpp:147,154,167; derivsX/Y/Z + update, :206-516).  Asynchronous
 * on the handle's stream. */
gkm_status gkm_evolve_eulerian(gkm_handle* h, int32_t nsteps);

/* The reference's GPU plug point, void evolve(ptype *W[5], DevAlloc *dev,
 * ptype dt) (src/GPUupdate.h:33, src/GPUupdate.cu:79-219): copy W in, take
 * one Eulerian step with the given dt, copy W out.  Synchronous.  The output
 * ghosts are already wrapped.  With pinned (cudaHostAlloc / cudaHostRegister)
 * or device W the step runs as a pipeline over chunks of y-planes, so the
 * copies in and out overlap the sweeps; pageable W takes one copy in, the
 * step, one copy out.  Both give the same result. */
gkm_status gkm_evolve(gkm_handle* h, double* const W[5], double dt);
/* Shape of that pipeline (no reference counterpart): y-planes per chunk (a
 * multiple of 16; 0 picks about n/8) and compute streams (1..4, default 2). */
gkm_status gkm_set_pipeline(gkm_handle* h, int32_t chunk_planes, int32_t compute_streams);

/* nsteps of the body of Evolve's loop (src/update.cpp:124-170): Eulerian
 * step, velocity splines of the new state (generateSplines, :1235-1247),
 * particle advection (evolveParticles / Particle::track, :1056-1086 and
 * src/ParticleTrack.cpp:42-73), dt of the next step.  Asynchronous. */
gkm_status gkm_step(gkm_handle* h, int32_t nsteps);

/* The Lagrangian half of Evolve's loop body on its own: velocity splines of
 * the current state, then Heun advection of every particle with the dt of the
 * last Eulerian step (generateSplines + evolveParticles, src/update.cpp:158-159).
 * gkm_step(h, n) equals n x { gkm_evolve_eulerian(h, 1); gkm_evolve_particles(h); }. */
gkm_status gkm_evolve_particles(gkm_handle* h);

/* nsteps full steps (with_particles != 0) or Eulerian steps, with CUDA events
 * around each phase on the handle's stream; synchronises.  ms[0..6] receive
 * the summed milliseconds of: x sweep, y sweep, z sweep (incl. the dt
 * reduction), halo wrap, spline build, particle advection, whole steps. */
gkm_status gkm_step_timed(gkm_handle* h, int32_t nsteps, int32_t with_particles, double ms[7]);

/* Sweep autotuner (no counterpart in the reference, whose loops have one
 * fixed shape): for each sweep direction, times every window variant of the
 * handle's precision with segment lengths from n down to 8 faces along the
 * sweep normal, `reps` launches each (CUDA events on the handle's stream), and
 * keeps the fastest.  The state is not changed; captured graphs are rebuilt. */
gkm_status gkm_autotune(gkm_handle* h, int32_t reps);
/* The sweep shapes in use: for x, y, z in turn: window variant, window width,
 * window height, segment length (faces per CTA along the normal).  FP64 window
 * variants: 0 = 16 x 8 (two CTAs per SM), 1 = 16 x 16, 2 = 16 x 16
 * warp-specialized (a producer warpgroup reconstructs the next face plane while
 * two consumer warpgroups compute fluxes; ensembles run its persistent form for
 * x and y; the plug-point pipeline of gkm_evolve runs it as variant 1).
 * FP32: 0 = 16 x 8. */
gkm_status gkm_sweep_config(const gkm_handle* h, int32_t out[12]);
/* Set the sweep shapes (no reference counterpart): for x, y, z in turn the
 * window variant and the segment length (in[2d], in[2d+1]).  GKM_ERR_CONFIG for
 * a variant this precision or this GPU does not have. */
gkm_status gkm_set_sweep_config(gkm_handle* h, const int32_t in[6]);

/* Kernels this handle has launched so far (graph replays count their kernels). */
gkm_status gkm_launch_count(const gkm_handle* h, int64_t* count);

/* Device FMA throughput probe on `device` (independent FMA chains, CUDA-event
 * timed): FP64 and FP32 in TFLOP/s, an FMA counted as 2 flops. */
gkm_status gkm_probe_fma_peak(int32_t device, double* fp64_tflops, double* fp32_tflops);

/* t, dt of the last step and completed steps (the globals t, dt, iter of
 * src/update.cpp:6,10).  Synchronises; GKM_ERR_NONFINITE if the state broke. */
gkm_status gkm_get_clock(gkm_handle* h, double* t, double* dt, int64_t* iter);
gkm_status gkm_synchronize(gkm_handle* h);

/* -------------------------------------------------------------- particles */

/* Load particles (Particle::initializeParticle / locateParticles,
 * src/ParticleTrack.cpp:11-17, src/update.cpp:1286-1322); pos is np x (y, x, z).
 * U (np x (u, v, w)) may be NULL: then U is evaluated from the velocity spline
 * of the current state (getParticleProp, src/ParticleTrack.cpp:99-107). */
gkm_status gkm_particles_upload(gkm_handle* h, int64_t np, const double* pos, const double* U);
gkm_status gkm_particles_download(gkm_handle* h, double* pos, double* U);

/* ---------------------------------------------------------- splines, stats */

/* Build the u, v, w splines of the current state (generateSplines 3-field
 * form, src/update.cpp:1235-1247, via get_bsplinep, src/Interpolation.cpp:3-31). */
gkm_status gkm_generate_splines(gkm_handle* h);
/* Coefficients of velocity component c (0 u, 1 v, 2 w): (N+P)^3 values,
 * N = nt (natural_ghost3, P = 2) or n (periodic, P = 3); axis 0 slowest. */
gkm_status gkm_spline_coefs(gkm_handle* h, int32_t c, double* out, int64_t capacity);
/* PrintStats field moments (src/update.cpp:688-842) of the current state. */
gkm_status gkm_stats_compute(gkm_handle* h, gkm_stats* out);

/* Velocity spline of one component built without allocating any device
 * memory.  No counterpart in the reference (whose einspline build allocates on
 * the host); it serves callers that cannot call cudaMalloc: programs whose
 * device memory already belongs to their own pool allocator, and programs
 * that must not let an allocation synchronise the device.
 *   W          device pointer to the state, 5 x (n+6)^3 doubles in the
 *              reference layout with valid ghosts (gkm_device_state gives one)
 *   component  1 = u, 2 = v, 3 = w (rho u / rho, ...)
 *   coefs      device pointer to (N+P)^3 doubles (as gkm_spline_coefs)
 *   stream     cudaStream_t as void*, NULL for the legacy stream
 * The intermediate results live in one static device array of 32 MiB (plus
 * 24 KiB of solver tables) that every GPU loading the library holds until
 * exit; grids needing more (natural_ghost3: about n > 150) return
 * GKM_ERR_CONFIG with a message on stderr.  The first call on a device looks
 * up that array's device address (kept until exit, so do not call it after
 * cudaDeviceReset), so make it before any stream capture.  The solver tables
 * are filled on the device: a call launches kernels and copies nothing.
 * Calls share the array and the tables: calls that overlap on the GPU race,
 * on one stream or several, so order them on one stream or serialise them.
 * Nothing in the array needs clearing; every element is written before it is
 * read.  Results equal gkm_generate_splines + gkm_spline_coefs bit for bit. */
gkm_status gkm_spline_build_noalloc(const double* W, int32_t n, int32_t spline_mode, int32_t component,
                                    double* coefs, void* stream);

/* ----------------------------------------------------- particle properties
 *
 * getParticleProp (src/ParticleTrack.cpp:99-113) for every particle at its
 * current position: the reference's eight splines of the current state
 * (generateSplines, src/update.cpp:1200-1233: rho, u, v, w, p, and the
 * Laplacians of u, v, w evaluated at every spline node and splined again),
 * then value + gradient of each (value + gradient + Hessian for p).  props
 * receives np x GKM_PROP_COUNT doubles, particle-major, in upload order:
 *   0 rho            1..3 grad rho           4..6 u, v, w
 *   7..9 grad u      10..12 grad v           13..15 grad w
 *   16 p             17..19 grad p           20..28 Hessian of p (row-major)
 *   29..31 lap u, lap v, lap w               32..40 grad lap u, v, w
 * Every gradient is (d/dy, d/dx, d/dz), the spline axis order (members DEN,
 * gradD, U, gradU, ..., hessP, lapU, ..., gradLapW of class Particle,
 * src/ParticleTrack.h:20-21).  The five extra splines (5 x (N+P)^3 doubles)
 * and an nt^3 node array are allocated on first use. */
#define GKM_PROP_COUNT 41
gkm_status gkm_particle_props(gkm_handle* h, double* props);

/* GetParticleStats (src/update.cpp:1111-1162) from the properties above:
 * particle-averaged |U|^2, S_ij S_ij, and the skewness of du/dx and dw/dz. */
typedef struct gkm_particle_stats {
    double TKE, SijSij, SKEWu, SKEWw;
    int64_t count;
} gkm_particle_stats;
gkm_status gkm_particle_stats_compute(gkm_handle* h, gkm_particle_stats* out);

/* ------------------------------------------------------------ output files
 *
 * The reference's output formats written from the current device state, so
 * its post-processing and restart readers take them unchanged.  The caller
 * picks the path; the reference's own names are Results/Field/Field_<rank>_
 * <iter>, Results/Particles/P_<rank>_<iter>, Results/Time/T_<iter> and
 * InitialCondition/Init<py><px><pz> (000 for the single cube). */

/* writeField (src/update.cpp:1324-1339): per interior cell, y-major then x
 * then z, "%d %d %d %.15e x5" with the x, y, z indices and rho, u, v, w, p. */
gkm_status gkm_write_field(gkm_handle* h, const char* path);
/* writeParticleData (src/update.cpp:1341-1368), one line per particle in
 * upload order (tag = upload index): position, rho, U, p and the gradients and
 * Hessian of gkm_particle_props in the reference's column order. */
gkm_status gkm_write_particles(gkm_handle* h, const char* path);
/* The time file of writeParticleData (src/update.cpp:1370-1378): t, the dt of
 * the coming step, t0 as "%.15e %.15e %.15e". */
gkm_status gkm_write_time(gkm_handle* h, const char* path);
/* WriteReInit (src/update.cpp:1381-1422): u, v, w, rho, p of the interior
 * cells, each n^3 doubles in MATLAB (column-major) order, the initial-field
 * format that Initialize_DHIT reads (src/FlowField.cpp:60-114). */
gkm_status gkm_write_reinit(gkm_handle* h, const char* path);

/* ---------------------------------------------------- single-call numerics */

/* flux() of src/GKMflux.cpp:11-229 on nfaces independent faces, host
 * buffers.  in: nfaces x 51 doubles = WL[5] WR[5] Wl[5] Wr[5] DWxl DWxr DWyl
 * DWyr DWzl DWzr [6x5] tau; F: nfaces x 5.  K = int((5-3gam)/(gam-1)). */
gkm_status gkm_flux_faces(const double* in, int64_t nfaces, double gam, double dt, double dx, double* F);
/* ApplyWENO of src/update.cpp:556-680 on n stencils of 6 cells x 5
 * components (host buffers); Wl, Wr: n x 5. */
gkm_status gkm_weno_faces(const double* stencils, int64_t n, double gam, double* Wl, double* Wr);

/* ---------------------------------------------------------------- interop */

/* Run on a caller's stream (cudaStream_t passed as void*); NULL restores the
 * handle's own stream.  Captured step graphs are rebuilt on the next step. */
gkm_status gkm_set_stream(gkm_handle* h, void* stream);
/* Device pointer of the current state (5 x nt^3 doubles, component-major);
 * valid until the next step. */
gkm_status gkm_device_state(gkm_handle* h, double** W);

/* ---------------------------------------------------------------- ensemble
 *
 * Many independent periodic cubes (grid size, Mt, Re, seed, particles may all
 * differ) stepped together on one GPU.  No reference counterpart: the
 * reference runs one cube per job (src/Main.cpp:10-49), and a parameter
 * sweep there is one job per case.  Each stage of a step is ONE launch over a
 * flattened work list of every member: the x, y, z sweeps (persistent CTAs
 * walking (member, window, segment) items), the ghost wrap, the three spline
 * passes and the Heun advection.  A step is captured as one CUDA graph per
 * buffer parity.  Every member evolves exactly as the same cube stepped alone
 * through gkm_step (bit for bit with the same sweep segment length).
 *
 * All members share the device, the precision and the ensemble's stream.
 * gkm_ensemble_member returns a member's handle for the single-cube calls
 * (gkm_upload_state, gkm_download_state, gkm_particles_upload/download,
 * gkm_stats_compute, gkm_get_clock, gkm_set_dt, ...); those calls run on the
 * ensemble's stream.  gkm_destroy and gkm_set_stream refuse member handles.
 * gkm_ensemble_step needs every member's state uploaded and all members at
 * the same buffer parity (true when they were uploaded and then stepped only
 * by the ensemble). */
typedef struct gkm_ensemble gkm_ensemble;

gkm_status gkm_ensemble_create(const gkm_config* members, int32_t n_members, gkm_ensemble** out);
gkm_status gkm_ensemble_destroy(gkm_ensemble* e);
const char* gkm_ensemble_last_error(const gkm_ensemble* e);
int32_t gkm_ensemble_size(const gkm_ensemble* e);
gkm_handle* gkm_ensemble_member(gkm_ensemble* e, int32_t m);
/* nsteps full steps (Eulerian + ghost wrap, and with with_particles the
 * splines of the new state and Heun advection of every member's particles). */
gkm_status gkm_ensemble_step(gkm_ensemble* e, int32_t nsteps, int32_t with_particles);
/* As gkm_ensemble_step without graphs, with CUDA-event times summed over the
 * steps: ms[0..2] x/y/z sweeps, ms[3] ghost wrap, ms[4] splines,
 * ms[5] particles, ms[6] whole steps. */
gkm_status gkm_ensemble_step_timed(gkm_ensemble* e, int32_t nsteps, int32_t with_particles, double ms[7]);
/* Per sweep direction, times over the whole ensemble (reps launches each):
 * every window variant with one segment length for all members, then, for
 * each grid size in turn (largest first), every segment length for the
 * members of that size; keeps the fastest.  The state is untouched and every
 * member's clock is restored.  A sweep launch takes the members with the
 * longest segments first. */
gkm_status gkm_ensemble_autotune(gkm_ensemble* e, int32_t reps);
/* out[4d..4d+3] = window variant, window width, window height, and the
 * segment length the variant was chosen with (before the per-size lengths) */
gkm_status gkm_ensemble_sweep_config(const gkm_ensemble* e, int32_t out[12]);
/* Segment length of every member per direction: out[d * n_members + m]
 * (capacity >= 3 x n_members).  No reference counterpart. */
gkm_status gkm_ensemble_segments(const gkm_ensemble* e, int32_t* out, int64_t capacity);
/* Set the ensemble's sweep shapes by hand (no reference counterpart): for x, y, z in turn the window
 * variant and one segment length for every member (in[2d], in[2d+1]); lengths above a member's n
 * mean one segment.  FP64 variant 2 (16 x 16, warp-specialized) runs the persistent
 * warp-specialized kernel for x and y and the 16 x 16 kernel for z.  GKM_ERR_CONFIG for a variant
 * this precision or this GPU does not have. */
gkm_status gkm_ensemble_set_sweep_config(gkm_ensemble* e, const int32_t in[6]);
gkm_status gkm_ensemble_launch_count(const gkm_ensemble* e, int64_t* count);
gkm_status gkm_ensemble_synchronize(gkm_ensemble* e);
/* The ensemble's stream (cudaStream_t as void*), for events or interop. */
gkm_status gkm_ensemble_stream(const gkm_ensemble* e, void** stream);

#ifdef __cplusplus
}
#endif

#endif
