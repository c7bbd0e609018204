/*
 * CPU oracle for the DNS_GKM_LPT hot path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU algorithm for the compressible
 * decaying-isotropic-turbulence step and the Lagrangian-particle step.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it,
 * and only as the checker; the shipped library never links or calls it.
 *
 * Every function cites the reference file:line it restates.  The restatement
 * keeps the reference's floating-point evaluation order (left-to-right sums,
 * the same divisions), so with -O2 -ffp-contract=off it reproduces the
 * reference CPU build bit for bit; tests/test_oracle_pin.py checks that
 * against golden vectors produced by the reference itself (oracle/_ref).
 *
 * Layout (reference src/param.h:26,40-41): 5 separate FP64 arrays W[q],
 * q = rho, rho*u, rho*v, rho*w, rho*E; index (j,i,k) -> (j*nt + i)*nt + k with
 * j = y (slowest), i = x, k = z (fastest); nt = n + 6 (3 ghost layers a side).
 *
 * The spline part (orc_spline_*) has no reference source to restate: the
 * reference calls einspline, which is not vendored.  It is the project's own
 * uniform cubic B-spline and is pinned by known-answer tests, not by the
 * reference ("parity unpinned" for splines/particles against real einspline).
 */
#ifndef GKM_ORACLE_H
#define GKM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
	int n;		 /* interior cells per side (reference nc / nc_seg*) */
	int nt;		 /* n + 6 */
	int K;		 /* internal degrees of freedom, int((5-3g)/(g-1)) */
	int visc_law; /* 0 = Sutherland (reference), 1 = mu0 (T/T0)^0.76 */
	double gam, den0, p0, Mt, Re, mu0, t0;
	double dx, T0, cfl;
} orc_params;

/* reference src/FlowField.cpp:36-50 (GetParams) with procDim = 1x1x1 */
void orc_params_init(orc_params *p, int n, double gam, double den0, double Mt, double Re,
					 double mu0, double p0, double t0, double cfl);

/* ---- numerics (reference src/GKMflux.cpp, src/update.cpp) ---- */
void orc_c2p(const double W[5], double gam, double *den, double U[3], double *P);
void orc_slopesolver(const double b[5], const double U[3], double lam, int K, double a[5]);
void orc_mcal(double M[5], const double I[7], const double Y[7], const double Z[7],
			  double Ie2, double Ie4, int k, int l, int m, const double ax[5]);
void orc_mcal0(double M[5], const double I[7], const double Y[7], const double Z[7],
			   double Ie2, int k, int l, int m);
void orc_flux(const double WL[5], const double WR[5], const double Wl[5], const double Wr[5],
			  const double DWxl[5], const double DWxr[5], const double DWyl[5], const double DWyr[5],
			  const double DWzl[5], const double DWzr[5], double tau, double dt, double dx,
			  double gam, int K, double F[5]);
void orc_weno(const double WLLL[5], const double WLL[5], const double WL[5], const double WR[5],
			  const double WRR[5], const double WRRR[5], double gam, double Wl[5], double Wr[5]);
double orc_viscosity(const orc_params *p, double T);

/* one face-normal sweep: dir 0 = x (derivsX), 1 = y (derivsY), 2 = z (derivsZ).
 * Writes F[q] at every face the reference loop visits. */
void orc_sweep(const orc_params *p, int dir, double *const W[5], double *F[5], double dt);
void orc_update(const orc_params *p, double *W[5], double *const Fx[5], double *const Fy[5], double *const Fz[5]);
void orc_halo(const orc_params *p, double *W[5]);
double orc_max_wave_speed(const orc_params *p, double *const W[5]);
double orc_timestep(const orc_params *p, double *const W[5]);
/* evolveEulerian + HaloTransfer; F* are caller scratch of nt^3 each (15 arrays) */
void orc_step(const orc_params *p, double *W[5], double *Fx[5], double *Fy[5], double *Fz[5], double dt);

/* ---- splines (project B-spline behind einspline's role) ---- */
typedef struct
{
	double *coefs;
	int n[3];		 /* data points per axis, axis 0 slowest */
	int periodic;	 /* 0 natural ends, 1 periodic */
	double start[3]; /* position of data point 0 */
	double dinv[3];	 /* 1 / spacing */
} orc_spline;

int orc_spline_pad(int periodic);
void orc_spline1d(const double *f, long fs, int N, int periodic, double *c, long cs);
void orc_spline3d_build(const double *data, const int n[3], int periodic, double *coefs, double *scratch);
/* what: 0 value, 1 value+grad, 2 value+grad+laplacian, 3 value+grad+hessian */
void orc_spline3d_eval(const orc_spline *s, double a, double b, double c, int what,
					   double *val, double grad[3], double *lapl, double hess[9]);

/* natural_ghost3 grid of the reference (src/Interpolation.cpp:3-31) */
void orc_grid_natural_ghost3(const orc_params *p, double *start, double *dinv);
/* periodic grid over the n interior cell centres */
void orc_grid_periodic(const orc_params *p, double *start, double *dinv);

/* ---- particles (reference src/ParticleTrack.cpp:48-73) ---- */
void orc_heun(double pos[3], const double U[3], const orc_spline *su, const orc_spline *sv,
			  const orc_spline *sw, double dt);

/* ---- stats (reference src/update.cpp:688-842) ---- */
typedef struct
{
	double TKE, Diss, SijSij, SKEWu, SKEWv, SKEWw, KURTu, KURTv, KURTw, Prms, Trms, Vrms;
} orc_stats;
void orc_print_stats(const orc_params *p, double *const W[5], const orc_spline *sden,
					 const orc_spline *su, const orc_spline *sv, const orc_spline *sw, orc_stats *out);

/* ---- particle properties (src/ParticleTrack.cpp:99-113 with the eight splines
 * of src/update.cpp:1200-1233) and their statistics (src/update.cpp:1111-1162).
 * W: 5 arrays nt^3 with valid ghosts; pos: np*3 (y,x,z); out: np*41 (the
 * property table of include/gkm.h); stats: TKE, SijSij, SKEWu, SKEWw. */
void orc_particle_props(const orc_params *p, double *const W[5], int spline_mode, long np, const double *pos,
						double *out);
void orc_particle_stats(const double *props, long np, double out[4]);

/* ---- whole-run driver mirroring Evolve's loop body (src/update.cpp:124-170) ----
 * mode bits: spline_mode 0 natural_ghost3 / 1 periodic.
 * W: 5 arrays nt^3 (interior filled; ghosts are refreshed here).
 * pos: np*3 (y,x,z) per particle, U: np*3 (u,v,w).  dt_hist: nsteps entries.
 * stats: filled every 10 steps (nsteps/10+1 entries) when not NULL. */
int orc_run(const orc_params *p, double *W[5], int nsteps, int spline_mode, long np,
			double *pos, double *U, double *dt_hist, orc_stats *stats);

#ifdef __cplusplus
}
#endif

#endif
