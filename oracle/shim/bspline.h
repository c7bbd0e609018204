/*
 * Stand-in for einspline's <bspline.h>, used ONLY to compile the reference CPU
 * sources as the test oracle (oracle/Makefile -> oracle/_ref/).  Test
 * infrastructure, never part of the shipped library.
 *
 * einspline 0.9.2 (fork github.com/nishantp9/einspline-0.9.2, named in the
 * reference README.md:14-25) is neither vendored nor installed, so this header
 * declares the einspline entry points the reference calls
 * (src/Interpolation.cpp:28,58; src/ParticleTrack.cpp:54-56,104-112;
 * src/update.cpp:162,165,731-738,1225-1227,1439-1441) and implements them with
 * the project's own uniform cubic B-spline (oracle/gkm_oracle.c,
 * orc_spline_*), written from the B-spline mathematics.  Spline parity against
 * real einspline is therefore unpinned; the project spline is pinned by
 * known-answer tests instead (cubic reproduction, node interpolation, natural
 * end conditions, O(h^4) convergence).
 */
#ifndef GKM_ORACLE_BSPLINE_SHIM_H
#define GKM_ORACLE_BSPLINE_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { PERIODIC, DERIV1, DERIV2, FLAT, NATURAL, ANTIPERIODIC } bc_code;

typedef struct
{
	bc_code lCode, rCode;
	double lVal, rVal;
} BCtype_d;

typedef struct
{
	double start, end;
	int num;
	double delta, delta_inv;
} Ugrid;

/* coefficient block of (num+2) per axis for NATURAL (c_{-1}..c_{num}),
 * (num+3) per axis for PERIODIC (wrapped copies, see orc_spline_*). */
typedef struct
{
	double *coefs;
	int n0, n1, n2;		   /* data points per axis (first argument = slowest) */
	int periodic;		   /* 0: natural ends, 1: periodic */
	double start[3], dinv[3];
} UBspline_3d_d;

UBspline_3d_d *create_UBspline_3d_d(Ugrid g0, Ugrid g1, Ugrid g2, BCtype_d bc0, BCtype_d bc1, BCtype_d bc2, double *data);
void destroy_Bspline(void *spline);
void eval_UBspline_3d_d(UBspline_3d_d *s, double a, double b, double c, double *val);
void eval_UBspline_3d_d_vg(UBspline_3d_d *s, double a, double b, double c, double *val, double *grad);
void eval_UBspline_3d_d_vgl(UBspline_3d_d *s, double a, double b, double c, double *val, double *grad, double *lapl);
void eval_UBspline_3d_d_vgh(UBspline_3d_d *s, double a, double b, double c, double *val, double *grad, double *hess);

#ifdef __cplusplus
}
#endif

#endif
