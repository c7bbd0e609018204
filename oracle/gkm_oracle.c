/*
 * CPU oracle for the DNS_GKM_LPT hot path — TEST INFRASTRUCTURE ONLY.
 * See gkm_oracle.h for the contract.  Built by oracle/Makefile with
 * -O2 -ffp-contract=off so that the evaluation order written here is the one
 * executed; the reference CPU build (makefileCPU_local:4,13: -O3 -std=c++11 on
 * x86-64, no FMA) executes the same order.
 */
#include "gkm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* reference src/param.h:17-21 */
#define ORC_PI atan(1.0) * 4.0
#define ORC_EPS pow(10.0, -10.0)
#define ORC_PRN 0.70
#define ORC_R 287.0

#define IDX(p, j, i, k) ((((long)(j)) * (p)->nt + (i)) * (p)->nt + (k))

/* reference src/FlowField.cpp:19-50 */
void orc_params_init(orc_params *p, int n, double gam, double den0, double Mt, double Re,
					 double mu0, double p0, double t0, double cfl)
{
	memset(p, 0, sizeof(*p));
	p->n = n;
	p->nt = n + 6;
	p->gam = gam;
	p->K = (int)((5.0 - 3.0 * gam) / (gam - 1.0));
	p->den0 = den0;
	p->p0 = p0;
	p->t0 = t0;
	p->dx = 2.0 * ORC_PI / n;
	p->T0 = p0 / (ORC_R * den0);
	p->Mt = Mt;
	p->mu0 = mu0;
	p->Re = Re;
	p->cfl = cfl;
	p->visc_law = 0;
}

/* reference src/GKMflux.cpp:302-309 */
void orc_c2p(const double W[5], double gam, double *den, double U[3], double *P)
{
	double d = W[0];
	*den = d;
	U[0] = W[1] / d;
	U[1] = W[2] / d;
	U[2] = W[3] / d;
	*P = (d * (gam - 1)) * (W[4] / d - 0.5 * (U[0] * U[0] + U[1] * U[1] + U[2] * U[2]));
}

/* reference src/GKMflux.cpp:283-297 (Prandtl correction on the energy slope) */
void orc_slopesolver(const double b[5], const double U[3], double lam, int K, double a[5])
{
	double usq = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
	double r2 = b[1] - U[0] * b[0];
	double r3 = b[2] - U[1] * b[0];
	double r4 = b[3] - U[2] * b[0];
	double r5 = 2 * b[4] - b[0] * (usq + (K + 3) / (2 * lam));

	a[4] = (1 / ORC_PRN) * (r5 - 2 * U[0] * r2 - 2 * U[1] * r3 - 2 * U[2] * r4) * (4 * lam * lam) / (K + 3);
	a[3] = 2 * lam * r4 - U[2] * a[4];
	a[2] = 2 * lam * r3 - U[1] * a[4];
	a[1] = 2 * lam * r2 - U[0] * a[4];
	a[0] = b[0] - a[1] * U[0] - a[2] * U[1] - a[3] * U[2] - .5 * a[4] * (usq + (K + 3) / (2 * lam));
}

/*
 * Moments of psi = (1, u, v, w, (u^2+v^2+w^2+xi^2)/2) against
 * u^k v^l w^m (a0 + a1 u + a2 v + a3 w + a4 psi_4) over a Maxwellian whose
 * normal-direction table is I (full or half space) and whose tangential tables
 * are Y, Z.  reference src/GKMflux.cpp:238-267.  tm(a,b,c) is the triple
 * product I[k+a] Y[l+b] Z[m+c], multiplied left to right as the reference does.
 */
#define tm(a, b, c) (I[k + (a)] * Y[l + (b)] * Z[m + (c)])
void orc_mcal(double M[5], const double I[7], const double Y[7], const double Z[7],
			  double Ie2, double Ie4, int k, int l, int m, const double ax[5])
{
	double v0 = 0.5 * (tm(2, 0, 0) + tm(0, 2, 0) + tm(0, 0, 2) + tm(0, 0, 0) * Ie2);
	M[0] = ax[0] * tm(0, 0, 0) + ax[1] * tm(1, 0, 0) + ax[2] * tm(0, 1, 0) + ax[3] * tm(0, 0, 1) + ax[4] * v0;
	double v1 = 0.5 * (tm(3, 0, 0) + tm(1, 2, 0) + tm(1, 0, 2) + tm(1, 0, 0) * Ie2);
	M[1] = ax[0] * tm(1, 0, 0) + ax[1] * tm(2, 0, 0) + ax[2] * tm(1, 1, 0) + ax[3] * tm(1, 0, 1) + ax[4] * v1;
	double v2 = 0.5 * (tm(2, 1, 0) + tm(0, 3, 0) + tm(0, 1, 2) + tm(0, 1, 0) * Ie2);
	M[2] = ax[0] * tm(0, 1, 0) + ax[1] * tm(1, 1, 0) + ax[2] * tm(0, 2, 0) + ax[3] * tm(0, 1, 1) + ax[4] * v2;
	double v3 = 0.5 * (tm(2, 0, 1) + tm(0, 2, 1) + tm(0, 0, 3) + tm(0, 0, 1) * Ie2);
	M[3] = ax[0] * tm(0, 0, 1) + ax[1] * tm(1, 0, 1) + ax[2] * tm(0, 1, 1) + ax[3] * tm(0, 0, 2) + ax[4] * v3;
	M[4] = 0.25 * ax[4] * (tm(4, 0, 0) + tm(0, 4, 0) + tm(0, 0, 4) + tm(0, 0, 0) * Ie4 + 2 * tm(2, 2, 0) + 2 * tm(2, 0, 2) + 2 * tm(2, 0, 0) * Ie2 + 2 * tm(0, 2, 2) + 2 * tm(0, 2, 0) * Ie2 + 2 * tm(0, 0, 2) * Ie2) +
		   ax[0] * v0 + ax[1] * v1 + ax[2] * v2 + ax[3] * v3;
}

/* the same moments with unit weight, reference src/GKMflux.cpp:269-278 */
void orc_mcal0(double M[5], const double I[7], const double Y[7], const double Z[7],
			   double Ie2, int k, int l, int m)
{
	M[0] = tm(0, 0, 0);
	M[1] = tm(1, 0, 0);
	M[2] = tm(0, 1, 0);
	M[3] = tm(0, 0, 1);
	M[4] = 0.5 * (tm(2, 0, 0) + tm(0, 2, 0) + tm(0, 0, 2) + tm(0, 0, 0) * Ie2);
}
#undef tm

/* Maxwellian moment tables of one state: x half-space (sign +1 for u>0,
 * -1 for u<0), and the full-space tables of all three directions.
 * reference src/GKMflux.cpp:45-68 and :85-103 */
typedef struct
{
	double lam, Ie2, Ie4;
	double H[7];	/* half-space table in x (Ip or In) */
	double H2[7];	/* second half table (state e only: In) */
	double F[3][7]; /* full-space tables x, y, z */
} orc_tables;

static void orc_build_tables(orc_tables *t, const double U[3], double lam, int K, int halves)
{
	/* halves: +1 -> H = positive half; -1 -> H = negative half; 2 -> H positive, H2 negative */
	t->lam = lam;
	t->Ie2 = K / (2 * lam);
	t->Ie4 = 3 * K / (4 * lam * lam) + K * (K - 1) / (4 * lam * lam);
	for (int j = 0; j < 3; j++)
	{
		t->F[j][0] = 1.0;
		t->F[j][1] = U[j];
	}
	double ex = exp(-lam * U[0] * U[0]);
	if (halves == 1 || halves == 2)
	{
		t->H[0] = 0.5 * (erfc(-sqrt(lam) * U[0]));
		t->H[1] = U[0] * t->H[0] + 0.5 * ex / sqrt(lam * ORC_PI);
	}
	else
	{
		t->H[0] = 0.5 * (erfc(sqrt(lam) * U[0]));
		t->H[1] = U[0] * t->H[0] - 0.5 * ex / sqrt(lam * ORC_PI);
	}
	if (halves == 2)
	{
		t->H2[0] = 0.5 * (erfc(sqrt(lam) * U[0]));
		t->H2[1] = U[0] * t->H2[0] - 0.5 * ex / sqrt(lam * ORC_PI);
	}
	for (int i = 2; i < 7; i++)
	{
		t->H[i] = U[0] * t->H[i - 1] + t->H[i - 2] * (i - 1) / (2 * lam);
		for (int j = 0; j < 3; j++)
			t->F[j][i] = U[j] * t->F[j][i - 1] + t->F[j][i - 2] * (i - 1) / (2 * lam);
		if (halves == 2)
			t->H2[i] = U[0] * t->H2[i - 1] + t->H2[i - 2] * (i - 1) / (2 * lam);
	}
}

/*
 * Gas-kinetic (BGK) flux across one face, integrated over [0, dt].
 * reference src/GKMflux.cpp:11-229.  Inputs: left/right cell averages WL/WR,
 * reconstructed face states Wl/Wr, normal (x) and tangential (y, z) slopes of
 * each side, the collision time tau (mu/p of the left cell), dt, dx.
 */
void orc_flux(const double WL[5], const double WR[5], const double Wl[5], const double Wr[5],
			  const double DWxl[5], const double DWxr[5], const double DWyl[5], const double DWyr[5],
			  const double DWzl[5], const double DWzr[5], double tau, double dt, double dx,
			  double gam, int K, double F[5])
{
	double denl, Ul[3], Pl, denr, Ur[3], Pr, dene, Ue[3], Pe;
	orc_tables L, R, E;

	orc_c2p(Wl, gam, &denl, Ul, &Pl);
	orc_c2p(Wr, gam, &denr, Ur, &Pr);
	double laml = 0.5 * denl / Pl;
	double lamr = 0.5 * denr / Pr;
	orc_build_tables(&L, Ul, laml, K, 1);
	orc_build_tables(&R, Ur, lamr, K, -1);

	/* equilibrium state at the face, :73-80 */
	double Mpgl000[5], Mngr000[5], We[5];
	orc_mcal0(Mpgl000, L.H, L.F[1], L.F[2], L.Ie2, 0, 0, 0);
	orc_mcal0(Mngr000, R.H, R.F[1], R.F[2], R.Ie2, 0, 0, 0);
	for (int q = 0; q < 5; q++)
		We[q] = denl * Mpgl000[q] + denr * Mngr000[q];
	orc_c2p(We, gam, &dene, Ue, &Pe);
	double lame = 0.5 * dene / Pe;
	orc_build_tables(&E, Ue, lame, K, 2);

	/* slopes, phase I, :107-125 */
	double bxl[5], bxr[5], byl[5], byr[5], bzl[5], bzr[5], bx_l[5], bx_r[5];
	double axl[5], axr[5], ayl[5], ayr[5], azl[5], azr[5], ax_l[5], ax_r[5];
	for (int i = 0; i < 5; i++)
	{
		bxl[i] = DWxl[i] / denl;
		bxr[i] = DWxr[i] / denr;
		byl[i] = DWyl[i] / denl;
		byr[i] = DWyr[i] / denr;
		bzl[i] = DWzl[i] / denl;
		bzr[i] = DWzr[i] / denr;
		bx_l[i] = 2 * (We[i] - WL[i]) / (dene * dx);
		bx_r[i] = 2 * (WR[i] - We[i]) / (dene * dx);
	}
	orc_slopesolver(bxl, Ul, laml, K, axl);
	orc_slopesolver(bxr, Ur, lamr, K, axr);
	orc_slopesolver(byl, Ul, laml, K, ayl);
	orc_slopesolver(byr, Ur, lamr, K, ayr);
	orc_slopesolver(bzl, Ul, laml, K, azl);
	orc_slopesolver(bzr, Ur, lamr, K, azr);
	orc_slopesolver(bx_l, Ue, lame, K, ax_l);
	orc_slopesolver(bx_r, Ue, lame, K, ax_r);

	/* slopes, phase II, :130-151 */
	double m1[5], m2[5], m3[5], m4[5], m5[5], m6[5], m7[5], m8[5], m9[5], m10[5];
	orc_mcal(m1, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 0, 0, 0, ayl);
	orc_mcal(m2, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 0, 0, 0, ayr);
	orc_mcal(m3, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 0, 0, 0, azl);
	orc_mcal(m4, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 0, 0, 0, azr);
	orc_mcal(m5, L.F[0], L.F[1], L.F[2], L.Ie2, L.Ie4, 1, 0, 0, axl);
	orc_mcal(m6, R.F[0], R.F[1], R.F[2], R.Ie2, R.Ie4, 1, 0, 0, axr);
	orc_mcal(m7, L.F[0], L.F[1], L.F[2], L.Ie2, L.Ie4, 0, 1, 0, ayl);
	orc_mcal(m8, R.F[0], R.F[1], R.F[2], R.Ie2, R.Ie4, 0, 1, 0, ayr);
	orc_mcal(m9, L.F[0], L.F[1], L.F[2], L.Ie2, L.Ie4, 0, 0, 1, azl);
	orc_mcal(m10, R.F[0], R.F[1], R.F[2], R.Ie2, R.Ie4, 0, 0, 1, azr);

	double by_[5], bz_[5], Bl[5], Br[5], ay_[5], az_[5], Al[5], Ar[5];
	for (int i = 0; i < 5; i++)
	{
		by_[i] = m1[i] + m2[i];
		bz_[i] = m3[i] + m4[i];
		Bl[i] = -m5[i] - m7[i] - m9[i];
		Br[i] = -m6[i] - m8[i] - m10[i];
	}
	orc_slopesolver(by_, Ue, lame, K, ay_);
	orc_slopesolver(bz_, Ue, lame, K, az_);
	orc_slopesolver(Bl, Ul, laml, K, Al);
	orc_slopesolver(Br, Ur, lamr, K, Ar);

	/* collision time, :156-157 */
	double w = fabs(denl / laml - denr / lamr) / (fabs(denl / laml + denr / lamr));
	tau = tau + dt * w;

	/* time-derivative slope A_, :162-191 */
	double gm0 = dt - tau * (1 - exp(-dt / tau));
	double gm1 = -(1 - exp(-dt / tau)) / gm0;
	double gm2 = (-dt + 2 * tau * (1 - exp(-dt / tau)) - dt * exp(-dt / tau)) / gm0;
	double gm3 = -gm1;
	double gm4 = (dt * exp(-dt / tau) - tau * (1 - exp(-dt / tau))) / gm0;
	double gm5 = tau * gm3;

	double e000[5], e100_axl_[5], e100_axr_[5], e010_ay[5], e001_az[5];
	double l100[5], r100[5], l010[5], r010[5], l001[5], r001[5], l000A[5], r000A[5];
	orc_mcal0(e000, E.F[0], E.F[1], E.F[2], E.Ie2, 0, 0, 0);
	orc_mcal(e100_axl_, E.H, E.F[1], E.F[2], E.Ie2, E.Ie4, 1, 0, 0, ax_l);
	orc_mcal(e100_axr_, E.H2, E.F[1], E.F[2], E.Ie2, E.Ie4, 1, 0, 0, ax_r);
	orc_mcal(e010_ay, E.F[0], E.F[1], E.F[2], E.Ie2, E.Ie4, 0, 1, 0, ay_);
	orc_mcal(e001_az, E.F[0], E.F[1], E.F[2], E.Ie2, E.Ie4, 0, 0, 1, az_);
	orc_mcal(l100, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 1, 0, 0, axl);
	orc_mcal(r100, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 1, 0, 0, axr);
	orc_mcal(l010, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 0, 1, 0, ayl);
	orc_mcal(r010, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 0, 1, 0, ayr);
	orc_mcal(l001, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 0, 0, 1, azl);
	orc_mcal(r001, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 0, 0, 1, azr);
	orc_mcal(l000A, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 0, 0, 0, Al);
	orc_mcal(r000A, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 0, 0, 0, Ar);

	double B_[5], A_[5];
	for (int i = 0; i < 5; i++)
	{
		B_[i] = gm1 * dene * e000[i] + gm2 * dene * (e100_axl_[i] + e100_axr_[i] + e010_ay[i] + e001_az[i]) + gm3 * (denl * Mpgl000[i] + denr * Mngr000[i]) +
				(gm4 + gm5) * (denl * (l100[i] + l010[i] + l001[i]) + denr * (r100[i] + r010[i] + r001[i])) +
				gm5 * (denl * l000A[i] + denr * r000A[i]);
		B_[i] = B_[i] / dene;
	}
	orc_slopesolver(B_, Ue, lame, K, A_);

	/* time-integrated flux, :197-228 */
	double P = -tau * (exp(-dt / tau) - 1);
	double Q = -tau * dt * exp(-dt / tau) - tau * tau * (exp(-dt / tau) - 1);
	double p0 = (dt - P);
	double p1 = 0.5 * dt * dt - tau * (p0);
	double p2 = -tau * (p0) + Q;
	double p3 = P;
	double p4 = -Q - tau * P;
	double p5 = -tau * P;

	double f_l100[5], f_r100[5], f_e100[5], f_e100A[5], f_e200l[5], f_e200r[5], f_e110[5], f_e101[5];
	double f_l200[5], f_r200[5], f_l110[5], f_r110[5], f_l101[5], f_r101[5], f_l100A[5], f_r100A[5];
	orc_mcal0(f_l100, L.H, L.F[1], L.F[2], L.Ie2, 1, 0, 0);
	orc_mcal0(f_r100, R.H, R.F[1], R.F[2], R.Ie2, 1, 0, 0);
	orc_mcal0(f_e100, E.F[0], E.F[1], E.F[2], E.Ie2, 1, 0, 0);
	orc_mcal(f_e100A, E.F[0], E.F[1], E.F[2], E.Ie2, E.Ie4, 1, 0, 0, A_);
	orc_mcal(f_e200l, E.H, E.F[1], E.F[2], E.Ie2, E.Ie4, 2, 0, 0, ax_l);
	orc_mcal(f_e200r, E.H2, E.F[1], E.F[2], E.Ie2, E.Ie4, 2, 0, 0, ax_r);
	orc_mcal(f_e110, E.F[0], E.F[1], E.F[2], E.Ie2, E.Ie4, 1, 1, 0, ay_);
	orc_mcal(f_e101, E.F[0], E.F[1], E.F[2], E.Ie2, E.Ie4, 1, 0, 1, az_);
	orc_mcal(f_l200, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 2, 0, 0, axl);
	orc_mcal(f_r200, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 2, 0, 0, axr);
	orc_mcal(f_l110, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 1, 1, 0, ayl);
	orc_mcal(f_r110, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 1, 1, 0, ayr);
	orc_mcal(f_l101, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 1, 0, 1, azl);
	orc_mcal(f_r101, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 1, 0, 1, azr);
	orc_mcal(f_l100A, L.H, L.F[1], L.F[2], L.Ie2, L.Ie4, 1, 0, 0, Al);
	orc_mcal(f_r100A, R.H, R.F[1], R.F[2], R.Ie2, R.Ie4, 1, 0, 0, Ar);

	for (int i = 0; i < 5; i++)
	{
		F[i] = p0 * dene * f_e100[i] + p1 * dene * f_e100A[i] + p2 * dene * (f_e200l[i] + f_e200r[i] + f_e110[i] + f_e101[i]) +
			   p3 * (denl * f_l100[i] + denr * f_r100[i]) + p4 * (denl * (f_l200[i] + f_l110[i] + f_l101[i]) + denr * (f_r200[i] + f_r110[i] + f_r101[i])) +
			   p5 * (denl * f_l100A[i] + denr * f_r100A[i]);
	}
}

/*
 * WENO-SYMOO reconstruction of one face from a 6-cell stencil.
 * reference src/update.cpp:556-680: 4 candidate stencils with linear weights
 * 1/20, 9/20, 9/20, 1/20, the 4th smoothness indicator replaced by the
 * largest of the four, alpha_k = gamma_k / (eps + IS_k).  Applied to rho,
 * rho u, rho v, rho w and to temperature; the face energy is rebuilt from the
 * reconstructed density, momentum and temperature.
 */
static void orc_weno_scalar(double a3, double a2, double a1, double b1, double b2, double b3,
							double *fl, double *fr)
{
	/* a3..a1 = LLL, LL, L; b1..b3 = R, RR, RRR */
	const double g0 = 1.0 / 20.0, g1 = 9.0 / 20.0, g2 = 9.0 / 20.0, g3 = 1.0 / 20.0;
	double P0p = a3 / 3 - 7 * a2 / 6 + 11 * a1 / 6;
	double P0n = b3 / 3 - 7 * b2 / 6 + 11 * b1 / 6;
	double P1p = -a2 / 6 + 5 * a1 / 6 + b1 / 3;
	double P1n = -b2 / 6 + 5 * b1 / 6 + a1 / 3;
	double P2p = a1 / 3 + 5 * b1 / 6 - b2 / 6;
	double P2n = b1 / 3 + 5 * a1 / 6 - a2 / 6;
	double P3p = 11 * b1 / 6 - 7 * b2 / 6 + b3 / 3;
	double P3n = 11 * a1 / 6 - 7 * a2 / 6 + a3 / 3;

	double IS0p = 13 * pow((a3 - 2 * a2 + a1), 2) / 12 + pow((a3 - 4 * a2 + 3 * a1), 2) / 4;
	double IS0n = 13 * pow((b3 - 2 * b2 + b1), 2) / 12 + pow((b3 - 4 * b2 + 3 * b1), 2) / 4;
	double IS1p = 13 * pow((a2 - 2 * a1 + b1), 2) / 12 + pow((-a2 + b1), 2) / 4;
	double IS1n = 13 * pow((b2 - 2 * b1 + a1), 2) / 12 + pow((-b2 + a1), 2) / 4;
	double IS2p = 13 * pow((a1 - 2 * b1 + b2), 2) / 12 + pow((-3 * a1 + 4 * b1 - b2), 2) / 4;
	double IS2n = 13 * pow((b1 - 2 * a1 + a2), 2) / 12 + pow((-3 * b1 + 4 * a1 - a2), 2) / 4;
	double IS3p = 13 * pow((b1 - 2 * b2 + b3), 2) / 12 + pow((-5 * b1 + 8 * b2 - 3 * b3), 2) / 4;
	double IS3n = 13 * pow((a1 - 2 * a2 + a3), 2) / 12 + pow((-5 * a1 + 8 * a2 - 3 * a3), 2) / 4;

	double mp = (IS0p < IS1p) ? IS1p : IS0p; /* std::max(a,b) returns a unless a < b */
	mp = (mp < IS2p) ? IS2p : mp;
	mp = (mp < IS3p) ? IS3p : mp;
	double mn = (IS0n < IS1n) ? IS1n : IS0n;
	mn = (mn < IS2n) ? IS2n : mn;
	mn = (mn < IS3n) ? IS3n : mn;
	IS3p = mp;
	IS3n = mn;

	double A0p = g0 * (1 / (ORC_EPS + IS0p)), A0n = g0 * (1 / (ORC_EPS + IS0n));
	double A1p = g1 * (1 / (ORC_EPS + IS1p)), A1n = g1 * (1 / (ORC_EPS + IS1n));
	double A2p = g2 * (1 / (ORC_EPS + IS2p)), A2n = g2 * (1 / (ORC_EPS + IS2n));
	double A3p = g3 * (1 / (ORC_EPS + IS3p)), A3n = g3 * (1 / (ORC_EPS + IS3n));
	double Sp = A0p + A1p + A2p + A3p;
	double Sn = A0n + A1n + A2n + A3n;
	*fl = ((A0p / Sp) * P0p + (A1p / Sp) * P1p + (A2p / Sp) * P2p + (A3p / Sp) * P3p);
	*fr = ((A0n / Sn) * P0n + (A1n / Sn) * P1n + (A2n / Sn) * P2n + (A3n / Sn) * P3n);
}

static double orc_temperature(const double W[5], double gam)
{
	/* reference src/update.cpp:615-620 */
	return (gam - 1) * (W[4] / W[0] - 0.5 * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) / (W[0] * W[0])) / ORC_R;
}

void orc_weno(const double WLLL[5], const double WLL[5], const double WL[5], const double WR[5],
			  const double WRR[5], const double WRRR[5], double gam, double Wl[5], double Wr[5])
{
	for (int i = 0; i < 4; i++)
		orc_weno_scalar(WLLL[i], WLL[i], WL[i], WR[i], WRR[i], WRRR[i], &Wl[i], &Wr[i]);
	double Tl, Tr;
	orc_weno_scalar(orc_temperature(WLLL, gam), orc_temperature(WLL, gam), orc_temperature(WL, gam),
					orc_temperature(WR, gam), orc_temperature(WRR, gam), orc_temperature(WRRR, gam), &Tl, &Tr);
	/* reference src/update.cpp:673-674 */
	Wl[4] = Wl[0] * ORC_R * Tl / (gam - 1.0) + 0.5 * (Wl[1] * Wl[1] + Wl[2] * Wl[2] + Wl[3] * Wl[3]) / Wl[0];
	Wr[4] = Wr[0] * ORC_R * Tr / (gam - 1.0) + 0.5 * (Wr[1] * Wr[1] + Wr[2] * Wr[2] + Wr[3] * Wr[3]) / Wr[0];
}

/* reference src/update.cpp:277 (Sutherland, 110.4 K); the power law is the
 * configuration option named in the workload description */
double orc_viscosity(const orc_params *p, double T)
{
	if (p->visc_law == 1)
		return p->mu0 * pow((T / p->T0), 0.76);
	return p->mu0 * pow((T / p->T0), 1.5) * (p->T0 + 110.4) / (T + 110.4);
}

static void orc_load(double *const W[5], long c, double out[5])
{
	for (int q = 0; q < 5; q++)
		out[q] = W[q][c];
}

static void orc_stencil_weno(const orc_params *p, double *const W[5], long c, long sn, double Wl[5], double Wr[5])
{
	double s[6][5];
	for (int o = 0; o < 6; o++)
		orc_load(W, c + (o - 2) * sn, s[o]);
	orc_weno(s[0], s[1], s[2], s[3], s[4], s[5], p->gam, Wl, Wr);
}

static void swap_comp(double v[5], int a, int b)
{
	double t = v[a];
	v[a] = v[b];
	v[b] = t;
}

/*
 * derivsX / derivsY / derivsZ, reference src/update.cpp:214-503.
 * Faces are stored at the index of their left cell.  Tangential neighbour
 * faces ("N/S" feed the y-slot slope, "F/B" the z-slot slope):
 *   x: N = j+1, S = j-1, F = k+1, B = k-1, components unchanged;
 *   y: N = i-1, S = i+1 (slope scaled by -0.5), F = k+1, B = k-1, swap 1<->2;
 *   z: N = i+1, S = i-1, F = j+1, B = j-1, swap 1<->3.
 * (In the z sweep the y-slot slope is d/dx and the z-slot slope d/dy while the
 * velocity slots hold v and u; the restatement keeps that pairing.)
 */
void orc_sweep(const orc_params *p, int dir, double *const W[5], double *F[5], double dt)
{
	const int nt = p->nt;
	const long sk = 1, si = nt, sj = (long)nt * nt;
	long sn, sN, sS, sF, sB;
	double yscale;
	int swap_with;
	int jlo = 3, ilo = 3, klo = 3;
	if (dir == 0)
	{
		sn = si; sN = sj; sS = -sj; sF = sk; sB = -sk; yscale = 0.5; swap_with = 0; ilo = 2;
	}
	else if (dir == 1)
	{
		sn = sj; sN = -si; sS = si; sF = sk; sB = -sk; yscale = -0.5; swap_with = 2; jlo = 2;
	}
	else
	{
		sn = sk; sN = si; sS = -si; sF = sj; sB = -sj; yscale = 0.5; swap_with = 3; klo = 2;
	}
	const double dx = p->dx;
	for (int j = jlo; j < nt - 3; j++)
		for (int i = ilo; i < nt - 3; i++)
			for (int k = klo; k < nt - 3; k++)
			{
				long c = ((long)j * nt + i) * nt + k;
				double WL[5], WR[5], Wl[5], Wr[5], WlN[5], WrN[5], WlS[5], WrS[5], WlF[5], WrF[5], WlB[5], WrB[5];
				double DWxl[5], DWxr[5], DWyl[5], DWyr[5], DWzl[5], DWzr[5], Fo[5];
				orc_load(W, c, WL);
				orc_load(W, c + sn, WR);
				orc_stencil_weno(p, W, c, sn, Wl, Wr);
				orc_stencil_weno(p, W, c + sN, sn, WlN, WrN);
				orc_stencil_weno(p, W, c + sS, sn, WlS, WrS);
				orc_stencil_weno(p, W, c + sF, sn, WlF, WrF);
				orc_stencil_weno(p, W, c + sB, sn, WlB, WrB);
				for (int q = 0; q < 5; q++)
				{
					DWxl[q] = 2 * (Wl[q] - WL[q]) / dx;
					DWxr[q] = 2 * (WR[q] - Wr[q]) / dx;
					DWyl[q] = yscale * (WlN[q] - WlS[q]) / dx;
					DWyr[q] = yscale * (WrN[q] - WrS[q]) / dx;
					DWzl[q] = 0.5 * (WlF[q] - WlB[q]) / dx;
					DWzr[q] = 0.5 * (WrF[q] - WrB[q]) / dx;
				}
				/* c2p() of the left cell, reference src/update.cpp:844-853 */
				double deni = WL[0];
				double ui = WL[1] / deni, vi = WL[2] / deni, wi = WL[3] / deni;
				double Vsqr = (ui * ui + vi * vi + wi * wi);
				double Pi = (deni * (p->gam - 1)) * (WL[4] / deni - 0.5 * Vsqr);
				double Ti = Pi / (ORC_R * deni);
				double tau = orc_viscosity(p, Ti) / Pi;
				if (swap_with)
				{
					double *vs[10] = {WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr};
					for (int v = 0; v < 10; v++)
						swap_comp(vs[v], 1, swap_with);
				}
				orc_flux(WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr, tau, dt, dx, p->gam, p->K, Fo);
				if (swap_with)
					swap_comp(Fo, 1, swap_with);
				for (int q = 0; q < 5; q++)
					F[q][c] = Fo[q];
			}
}

/* reference src/update.cpp:505-516 */
void orc_update(const orc_params *p, double *W[5], double *const Fx[5], double *const Fy[5], double *const Fz[5])
{
	const int nt = p->nt;
	const long si = nt, sj = (long)nt * nt;
	const double dx = p->dx;
	for (int j = 3; j < nt - 3; j++)
		for (int i = 3; i < nt - 3; i++)
			for (int k = 3; k < nt - 3; k++)
			{
				long c = ((long)j * nt + i) * nt + k;
				for (int q = 0; q < 5; q++)
					W[q][c] -= (1 / dx) * (Fx[q][c] - Fx[q][c - si] + Fy[q][c] - Fy[q][c - sj] + Fz[q][c] - Fz[q][c - 1]);
			}
}

/* HaloTransfer on a 1x1x1 periodic topology, reference src/update.cpp:855-1029:
 * every ghost cell ends up holding the interior cell at the wrapped index. */
static int wrap3(int a, int n)
{
	if (a < 3)
		return a + n;
	if (a >= n + 3)
		return a - n;
	return a;
}

void orc_halo(const orc_params *p, double *W[5])
{
	const int nt = p->nt, n = p->n;
	for (int j = 0; j < nt; j++)
		for (int i = 0; i < nt; i++)
			for (int k = 0; k < nt; k++)
			{
				int jj = wrap3(j, n), ii = wrap3(i, n), kk = wrap3(k, n);
				if (jj == j && ii == i && kk == k)
					continue;
				long c = ((long)j * nt + i) * nt + k, s = ((long)jj * nt + ii) * nt + kk;
				for (int q = 0; q < 5; q++)
					W[q][c] = W[q][s];
			}
}

/* reference src/update.cpp:1031-1054 */
double orc_max_wave_speed(const orc_params *p, double *const W[5])
{
	const int nt = p->nt;
	double mx = 0.0;
	for (int j = 3; j < nt - 3; j++)
		for (int i = 3; i < nt - 3; i++)
			for (int k = 3; k < nt - 3; k++)
			{
				long c = ((long)j * nt + i) * nt + k;
				double deni = W[0][c];
				double ui = W[1][c] / deni, vi = W[2][c] / deni, wi = W[3][c] / deni;
				double Vsqr = (ui * ui + vi * vi + wi * wi);
				double Pi = (deni * (p->gam - 1)) * (W[4][c] / deni - 0.5 * Vsqr);
				double val = sqrt(Vsqr) + sqrt(p->gam * Pi / deni);
				if (mx < val)
					mx = val;
			}
	return mx;
}

double orc_timestep(const orc_params *p, double *const W[5])
{
	return p->cfl * p->dx / orc_max_wave_speed(p, W);
}

void orc_step(const orc_params *p, double *W[5], double *Fx[5], double *Fy[5], double *Fz[5], double dt)
{
	orc_sweep(p, 0, W, Fx, dt);
	orc_sweep(p, 1, W, Fy, dt);
	orc_sweep(p, 2, W, Fz, dt);
	orc_update(p, W, Fx, Fy, Fz);
	orc_halo(p, W);
}

/* ------------------------------------------------------------------------
 * Uniform cubic B-spline (project formulation; no reference source exists).
 * Natural ends: c_0 = f_0, c_{N-1} = f_{N-1} (these follow from f'' = 0 and
 * the interpolation rows), interior rows c_{i-1} + 4 c_i + c_{i+1} = 6 f_i
 * solved by Thomas elimination, then c_{-1} = 2c_0 - c_1, c_N = 2c_{N-1} -
 * c_{N-2}.  Stored as N+2 values (c_{-1}..c_N).
 * Periodic: cyclic rows solved by Sherman-Morrison on the Thomas solver,
 * stored as N+3 values s[m] = c_{(m-1) mod N}.
 * ---------------------------------------------------------------------- */
int orc_spline_pad(int periodic) { return periodic ? 3 : 2; }

void orc_spline1d(const double *f, long fs, int N, int periodic, double *c, long cs)
{
	double *dp = (double *)malloc(sizeof(double) * (size_t)(N + 1));
	double *mt = (double *)malloc(sizeof(double) * (size_t)(N + 1));
	double *x = (double *)malloc(sizeof(double) * (size_t)(N + 1));
	if (!periodic)
	{
		double c0 = f[0], cl = f[(long)(N - 1) * fs];
		dp[1] = 4.0;
		for (int i = 2; i <= N - 2; i++)
		{
			mt[i] = 1.0 / dp[i - 1];
			dp[i] = 4.0 - mt[i];
		}
		double rp = 0.0;
		for (int i = 1; i <= N - 2; i++)
		{
			double r = 6.0 * f[(long)i * fs];
			if (i == 1)
				r = r - c0;
			if (i == N - 2)
				r = r - cl;
			rp = (i == 1) ? r : r - mt[i] * rp;
			x[i] = rp;
		}
		x[N - 2] = x[N - 2] / dp[N - 2];
		for (int i = N - 3; i >= 1; i--)
			x[i] = (x[i] - x[i + 1]) / dp[i];
		x[0] = c0;
		x[N - 1] = cl;
		c[0] = 2.0 * x[0] - x[1];
		for (int i = 0; i < N; i++)
			c[(long)(i + 1) * cs] = x[i];
		c[(long)(N + 1) * cs] = 2.0 * x[N - 1] - x[N - 2];
	}
	else
	{
		/* A = B + u v^T with gamma = -4: B diag (8, 4, ..., 4, 4.25),
		 * u = (-4, 0.., 1), v = (1, 0.., -0.25) */
		double *z = (double *)malloc(sizeof(double) * (size_t)N);
		dp[0] = 8.0;
		for (int i = 1; i < N; i++)
		{
			mt[i] = 1.0 / dp[i - 1];
			dp[i] = ((i == N - 1) ? 4.25 : 4.0) - mt[i];
		}
		/* z = B^-1 u */
		double rp = -4.0;
		z[0] = rp;
		for (int i = 1; i < N; i++)
		{
			double r = (i == N - 1) ? 1.0 : 0.0;
			rp = r - mt[i] * rp;
			z[i] = rp;
		}
		z[N - 1] = z[N - 1] / dp[N - 1];
		for (int i = N - 2; i >= 0; i--)
			z[i] = (z[i] - z[i + 1]) / dp[i];
		double denom = 1.0 + (z[0] + (-0.25) * z[N - 1]);
		/* y = B^-1 (6 f) */
		rp = 6.0 * f[0];
		x[0] = rp;
		for (int i = 1; i < N; i++)
		{
			rp = 6.0 * f[(long)i * fs] - mt[i] * rp;
			x[i] = rp;
		}
		x[N - 1] = x[N - 1] / dp[N - 1];
		for (int i = N - 2; i >= 0; i--)
			x[i] = (x[i] - x[i + 1]) / dp[i];
		double fac = (x[0] + (-0.25) * x[N - 1]) / denom;
		for (int i = 0; i < N; i++)
			x[i] = x[i] - fac * z[i];
		for (int m = 0; m < N + 3; m++)
			c[(long)m * cs] = x[(m - 1 + N) % N];
		free(z);
	}
	free(dp);
	free(mt);
	free(x);
}

/* tensor-product build: axis 0 (slowest) first, then axis 1, then axis 2 */
void orc_spline3d_build(const double *data, const int n[3], int periodic, double *coefs, double *scratch)
{
	(void)scratch;
	const int P = orc_spline_pad(periodic);
	const long n0 = n[0], n1 = n[1], n2 = n[2];
	const long m0 = n0 + P, m1 = n1 + P, m2 = n2 + P;
	double *A = (double *)malloc(sizeof(double) * (size_t)(m0 * n1 * n2));
	double *B = (double *)malloc(sizeof(double) * (size_t)(m0 * m1 * n2));
	for (long i1 = 0; i1 < n1; i1++)
		for (long i2 = 0; i2 < n2; i2++)
			orc_spline1d(data + i1 * n2 + i2, n1 * n2, (int)n0, periodic, A + i1 * n2 + i2, n1 * n2);
	for (long a = 0; a < m0; a++)
		for (long i2 = 0; i2 < n2; i2++)
			orc_spline1d(A + a * n1 * n2 + i2, n2, (int)n1, periodic, B + a * m1 * n2 + i2, n2);
	for (long a = 0; a < m0; a++)
		for (long b = 0; b < m1; b++)
			orc_spline1d(B + (a * m1 + b) * n2, 1, (int)n2, periodic, coefs + (a * m1 + b) * m2, 1);
	free(A);
	free(B);
}

static void orc_basis(double t, double w[4], double d[4], double h[4], double dinv)
{
	double t2 = t * t, t3 = t2 * t, s = 1.0 - t;
	w[0] = (1.0 / 6.0) * (s * s * s);
	w[1] = (1.0 / 6.0) * (3.0 * t3 - 6.0 * t2 + 4.0);
	w[2] = (1.0 / 6.0) * (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0);
	w[3] = (1.0 / 6.0) * t3;
	d[0] = (-0.5 * (s * s)) * dinv;
	d[1] = (0.5 * (3.0 * t2 - 4.0 * t)) * dinv;
	d[2] = (0.5 * (-3.0 * t2 + 2.0 * t + 1.0)) * dinv;
	d[3] = (0.5 * t2) * dinv;
	double d2 = dinv * dinv;
	h[0] = s * d2;
	h[1] = (3.0 * t - 2.0) * d2;
	h[2] = (-3.0 * t + 1.0) * d2;
	h[3] = t * d2;
}

static int orc_locate(const orc_spline *s, int ax, double x, double *t)
{
	double u = (x - s->start[ax]) * s->dinv[ax];
	double fl = floor(u);
	int i = (int)fl;
	int N = s->n[ax];
	if (s->periodic)
	{
		*t = u - fl;
		i %= N;
		if (i < 0)
			i += N;
		return i;
	}
	if (i < 0)
		i = 0;
	if (i > N - 2)
		i = N - 2;
	*t = u - (double)i;
	return i;
}

void orc_spline3d_eval(const orc_spline *s, double a, double b, double c, int what,
					   double *val, double grad[3], double *lapl, double hess[9])
{
	const int P = orc_spline_pad(s->periodic);
	const long m1 = s->n[1] + P, m2 = s->n[2] + P;
	double ta, tb, tc;
	int ia = orc_locate(s, 0, a, &ta), ib = orc_locate(s, 1, b, &tb), ic = orc_locate(s, 2, c, &tc);
	double wa[4], da[4], ha[4], wb[4], db[4], hb[4], wc[4], dc[4], hc[4];
	orc_basis(ta, wa, da, ha, s->dinv[0]);
	orc_basis(tb, wb, db, hb, s->dinv[1]);
	orc_basis(tc, wc, dc, hc, s->dinv[2]);
	/* contract axis 2 first: C_w[a][b], C_d[a][b], C_h[a][b] */
	double cw[4][4], cd[4][4], ch[4][4];
	for (int x = 0; x < 4; x++)
		for (int y = 0; y < 4; y++)
		{
			const double *row = s->coefs + ((long)(ia + x) * m1 + (ib + y)) * m2 + ic;
			cw[x][y] = wc[0] * row[0] + wc[1] * row[1] + wc[2] * row[2] + wc[3] * row[3];
			cd[x][y] = dc[0] * row[0] + dc[1] * row[1] + dc[2] * row[2] + dc[3] * row[3];
			ch[x][y] = hc[0] * row[0] + hc[1] * row[1] + hc[2] * row[2] + hc[3] * row[3];
		}
	/* then axis 1, then axis 0 */
	double v = 0, g0 = 0, g1 = 0, g2 = 0, h00 = 0, h01 = 0, h02 = 0, h11 = 0, h12 = 0, h22 = 0;
	for (int x = 0; x < 4; x++)
	{
		double bw = wb[0] * cw[x][0] + wb[1] * cw[x][1] + wb[2] * cw[x][2] + wb[3] * cw[x][3];
		double bd = db[0] * cw[x][0] + db[1] * cw[x][1] + db[2] * cw[x][2] + db[3] * cw[x][3];
		double bh = hb[0] * cw[x][0] + hb[1] * cw[x][1] + hb[2] * cw[x][2] + hb[3] * cw[x][3];
		double bwd = wb[0] * cd[x][0] + wb[1] * cd[x][1] + wb[2] * cd[x][2] + wb[3] * cd[x][3];
		double bdd = db[0] * cd[x][0] + db[1] * cd[x][1] + db[2] * cd[x][2] + db[3] * cd[x][3];
		double bwh = wb[0] * ch[x][0] + wb[1] * ch[x][1] + wb[2] * ch[x][2] + wb[3] * ch[x][3];
		v += wa[x] * bw;
		g0 += da[x] * bw;
		g1 += wa[x] * bd;
		g2 += wa[x] * bwd;
		h00 += ha[x] * bw;
		h01 += da[x] * bd;
		h02 += da[x] * bwd;
		h11 += wa[x] * bh;
		h12 += wa[x] * bdd;
		h22 += wa[x] * bwh;
	}
	*val = v;
	if (what >= 1)
	{
		grad[0] = g0;
		grad[1] = g1;
		grad[2] = g2;
	}
	if (what == 2)
		*lapl = h00 + h11 + h22;
	if (what == 3)
	{
		hess[0] = h00; hess[1] = h01; hess[2] = h02;
		hess[3] = h01; hess[4] = h11; hess[5] = h12;
		hess[6] = h02; hess[7] = h12; hess[8] = h22;
	}
}

/* grid of the reference's splines, src/Interpolation.cpp:11-26 with sta = 0:
 * nt points starting at -3 dx + dx/2; spacing as einspline derives it from
 * (end - start) / (num - 1) */
void orc_grid_natural_ghost3(const orc_params *p, double *start, double *dinv)
{
	double s = (0 - 3) * p->dx + 0.5 * p->dx;
	double e = s + (p->nt - 1) * p->dx;
	double delta = (e - s) / (double)(p->nt - 1);
	*start = s;
	*dinv = 1.0 / delta;
}

void orc_grid_periodic(const orc_params *p, double *start, double *dinv)
{
	*start = 0.5 * p->dx;
	*dinv = 1.0 / p->dx;
}

/* reference src/ParticleTrack.cpp:48-73; pos = (y, x, z), U = (u, v, w) */
void orc_heun(double pos[3], const double U[3], const orc_spline *su, const orc_spline *sv,
			  const orc_spline *sw, double dt)
{
	double U2[3], g[3], l, h[9];
	double a = pos[0] + U[1] * dt, b = pos[1] + U[0] * dt, c = pos[2] + U[2] * dt;
	orc_spline3d_eval(su, a, b, c, 0, &U2[0], g, &l, h);
	orc_spline3d_eval(sv, a, b, c, 0, &U2[1], g, &l, h);
	orc_spline3d_eval(sw, a, b, c, 0, &U2[2], g, &l, h);
	pos[0] += 0.5 * (U[1] + U2[1]) * dt;
	pos[1] += 0.5 * (U[0] + U2[0]) * dt;
	pos[2] += 0.5 * (U[2] + U2[2]) * dt;
	for (int q = 0; q < 3; q++)
	{
		if (pos[q] > 2 * ORC_PI)
			pos[q] = fmod(pos[q], 2 * ORC_PI);
		if (pos[q] < 0)
			pos[q] = 2 * ORC_PI - fmod(-pos[q], 2 * ORC_PI);
	}
}

/* reference src/update.cpp:688-842 (PrintStats), single rank */
void orc_print_stats(const orc_params *p, double *const W[5], const orc_spline *sden,
					 const orc_spline *su, const orc_spline *sv, const orc_spline *sw, orc_stats *out)
{
	const int nt = p->nt;
	const double dx = p->dx, gam = p->gam;
	const double Nc = (double)p->n * p->n * p->n;
	double sTKE = 0, sDiss = 0, sS = 0, u2 = 0, u3 = 0, u4 = 0, v2 = 0, v3 = 0, v4 = 0, w2 = 0, w3 = 0, w4 = 0;
	double Pm = 0, Tm = 0, Vm = 0;
	double gU[3], gV[3], gW[3], l, h[9], g[3];
	for (int j = 3; j < nt - 3; j++)
		for (int i = 3; i < nt - 3; i++)
			for (int k = 3; k < nt - 3; k++)
			{
				long c = ((long)j * nt + i) * nt + k;
				double deni = W[0][c];
				double ui = W[1][c] / deni, vi = W[2][c] / deni, wi = W[3][c] / deni;
				double Vsqr = (ui * ui + vi * vi + wi * wi);
				double Pi = (deni * (gam - 1)) * (W[4][c] / deni - 0.5 * Vsqr);
				double Ti = Pi / (ORC_R * deni);
				Pm += Pi;
				Tm += Ti;
				Vm += 1 / deni;
				double y = (0 + j - 3) * dx + 0.5 * dx;
				double x = (0 + i - 3) * dx + 0.5 * dx;
				double z = (0 + k - 3) * dx + 0.5 * dx;
				orc_spline3d_eval(sden, y, x, z, 0, &deni, g, &l, h);
				orc_spline3d_eval(su, y, x, z, 1, &ui, gU, &l, h);
				orc_spline3d_eval(sv, y, x, z, 1, &vi, gV, &l, h);
				orc_spline3d_eval(sw, y, x, z, 1, &wi, gW, &l, h);
				double dudx = gU[1], dudy = gU[0], dudz = gU[2];
				double dvdx = gV[1], dvdy = gV[0], dvdz = gV[2];
				double dwdx = gW[1], dwdy = gW[0], dwdz = gW[2];
				double mu = orc_viscosity(p, Ti);
				sDiss += mu * (dudx * dudx + dudy * dudy + dudz * dudz + dvdx * dvdx + dvdy * dvdy + dvdz * dvdz + dwdx * dwdx + dwdy * dwdy + dwdz * dwdz);
				sTKE += deni * (ui * ui + vi * vi + wi * wi);
				sS += (dudx * dudx + 0.5 * pow(dudy + dvdx, 2) + 0.5 * pow(dudz + dwdx, 2) + 0.5 * pow(dwdy + dvdz, 2) + dvdy * dvdy + dwdz * dwdz);
				u2 += dudx * dudx;
				u3 += dudx * dudx * dudx;
				u4 += dudx * dudx * dudx * dudx;
				v2 += dvdy * dvdy;
				v3 += dvdy * dvdy * dvdy;
				v4 += dvdy * dvdy * dvdy * dvdy;
				w2 += dwdz * dwdz;
				w3 += dwdz * dwdz * dwdz;
				w4 += dwdz * dwdz * dwdz * dwdz;
			}
	out->TKE = sTKE / Nc;
	out->Diss = sDiss / Nc;
	out->SijSij = sS / Nc;
	u2 /= Nc; u3 /= Nc; u4 /= Nc;
	v2 /= Nc; v3 /= Nc; v4 /= Nc;
	w2 /= Nc; w3 /= Nc; w4 /= Nc;
	out->SKEWu = u3 / pow(u2, 1.5);
	out->SKEWv = v3 / pow(v2, 1.5);
	out->SKEWw = w3 / pow(w2, 1.5);
	out->KURTu = u4 / pow(u2, 2);
	out->KURTv = v4 / pow(v2, 2);
	out->KURTw = w4 / pow(w2, 2);
	Pm /= Nc;
	Tm /= Nc;
	Vm /= Nc;
	double Pr = 0, Tr = 0, Vr = 0;
	for (int j = 3; j < nt - 3; j++)
		for (int i = 3; i < nt - 3; i++)
			for (int k = 3; k < nt - 3; k++)
			{
				long c = ((long)j * nt + i) * nt + k;
				double deni = W[0][c];
				double ui = W[1][c] / deni, vi = W[2][c] / deni, wi = W[3][c] / deni;
				double Vsqr = (ui * ui + vi * vi + wi * wi);
				double Pi = (deni * (gam - 1)) * (W[4][c] / deni - 0.5 * Vsqr);
				double Ti = Pi / (ORC_R * deni);
				Pr += pow((Pm - Pi), 2);
				Tr += pow((Tm - Ti), 2);
				Vr += pow((Vm - 1 / deni), 2);
			}
	Pr = sqrt(Pr / Nc);
	Tr = sqrt(Tr / Nc);
	Vr = sqrt(Vr / Nc);
	out->Prms = Pr / (gam * p->p0 * p->Mt * p->Mt);
	out->Trms = Tr / ((gam - 1) * p->T0 * p->Mt * p->Mt);
	out->Vrms = Vr / (p->Mt * p->Mt / p->den0);
}

/* build the velocity (and optionally density) splines of the current field */
static void orc_build_field_splines(const orc_params *p, double *const W[5], int spline_mode,
									orc_spline s[4], int with_density)
{
	const int nt = p->nt, n = p->n;
	const long Nt = (long)nt * nt * nt;
	int periodic = spline_mode == 1;
	int npts = periodic ? n : nt;
	int P = orc_spline_pad(periodic);
	long M = (long)(npts + P) * (npts + P) * (npts + P);
	double start, dinv;
	if (periodic)
		orc_grid_periodic(p, &start, &dinv);
	else
		orc_grid_natural_ghost3(p, &start, &dinv);
	double *f = (double *)malloc(sizeof(double) * (size_t)Nt);
	for (int q = with_density ? 0 : 1; q < 4; q++)
	{
		/* reference src/update.cpp:1202-1207 (den, u = rho u / den, ...) */
		long m = 0;
		for (int j = 0; j < nt; j++)
			for (int i = 0; i < nt; i++)
				for (int k = 0; k < nt; k++)
				{
					if (periodic && (j < 3 || j >= n + 3 || i < 3 || i >= n + 3 || k < 3 || k >= n + 3))
						continue;
					long c = ((long)j * nt + i) * nt + k;
					f[m++] = (q == 0) ? W[0][c] : W[q][c] / W[0][c];
				}
		s[q].coefs = (double *)malloc(sizeof(double) * (size_t)M);
		s[q].periodic = periodic;
		for (int a = 0; a < 3; a++)
		{
			s[q].n[a] = npts;
			s[q].start[a] = start;
			s[q].dinv[a] = dinv;
		}
		orc_spline3d_build(f, s[q].n, periodic, s[q].coefs, NULL);
	}
	free(f);
}

/* one more spline of the field from an nt^3 (ghost-layout) array; nodes as orc_build_field_splines */
static void orc_build_array_spline(const orc_params *p, const double *a, int spline_mode, orc_spline *s)
{
	const int nt = p->nt, n = p->n;
	const int periodic = spline_mode == 1;
	const int npts = periodic ? n : nt;
	const int P = orc_spline_pad(periodic);
	const long M = (long)(npts + P) * (npts + P) * (npts + P);
	double start, dinv;
	if (periodic)
		orc_grid_periodic(p, &start, &dinv);
	else
		orc_grid_natural_ghost3(p, &start, &dinv);
	double *f = (double *)malloc(sizeof(double) * (size_t)npts * npts * npts);
	long m = 0;
	for (int j = 0; j < nt; j++)
		for (int i = 0; i < nt; i++)
			for (int k = 0; k < nt; k++)
			{
				if (periodic && (j < 3 || j >= n + 3 || i < 3 || i >= n + 3 || k < 3 || k >= n + 3))
					continue;
				f[m++] = a[((long)j * nt + i) * nt + k];
			}
	s->coefs = (double *)malloc(sizeof(double) * (size_t)M);
	s->periodic = periodic;
	for (int ax = 0; ax < 3; ax++)
	{
		s->n[ax] = npts;
		s->start[ax] = start;
		s->dinv[ax] = dinv;
	}
	orc_spline3d_build(f, s->n, periodic, s->coefs, NULL);
	free(f);
}

/* reference src/update.cpp:1200-1233 (the eight splines) and
 * src/ParticleTrack.cpp:99-113 (getParticleProp); out: np x 41, the
 * property table of include/gkm.h */
void orc_particle_props(const orc_params *p, double *const W[5], int spline_mode, long np, const double *pos,
						double *out)
{
	const int nt = p->nt, n = p->n;
	const long Nt = (long)nt * nt * nt;
	const int periodic = spline_mode == 1;
	orc_spline s[8];
	memset(s, 0, sizeof(s));
	orc_build_field_splines(p, W, spline_mode, s, 1);   /* rho, u, v, w */
	double *a = (double *)malloc(sizeof(double) * (size_t)Nt);
	/* p = (den (gam - 1)) (W4 / den - 0.5 Vsqr), src/update.cpp:1202-1209 */
	for (long c = 0; c < Nt; c++)
	{
		double den = W[0][c];
		double u = W[1][c] / den, v = W[2][c] / den, w = W[3][c] / den;
		double Vsqr = u * u + v * v + w * w;
		a[c] = (den * (p->gam - 1)) * (W[4][c] / den - 0.5 * Vsqr);
	}
	orc_build_array_spline(p, a, spline_mode, &s[4]);
	/* Laplacians at the nodes, src/update.cpp:1217-1228: the reference's For
	 * loops visit the interior nodes only; the ghost nodes of its (freshly
	 * allocated) arrays stay zero and enter the natural_ghost3 splines as such */
	for (int f = 0; f < 3; f++)
	{
		for (int j = 0; j < nt; j++)
			for (int i = 0; i < nt; i++)
				for (int k = 0; k < nt; k++)
				{
					long c = ((long)j * nt + i) * nt + k;
					if (j < 3 || j >= n + 3 || i < 3 || i >= n + 3 || k < 3 || k >= n + 3)
					{
						a[c] = 0.0;
						continue;
					}
					double y = (j - 3) * p->dx + 0.5 * p->dx;
					double x = (i - 3) * p->dx + 0.5 * p->dx;
					double z = (k - 3) * p->dx + 0.5 * p->dx;
					double v, g[3], h[9];
					orc_spline3d_eval(&s[1 + f], y, x, z, 2, &v, g, &a[c], h);
				}
		orc_build_array_spline(p, a, spline_mode, &s[5 + f]);
	}
	free(a);
	for (long q = 0; q < np; q++)
	{
		const double y = pos[3 * q], x = pos[3 * q + 1], z = pos[3 * q + 2];
		double *o = out + 41 * q;
		double l, h[9];
		orc_spline3d_eval(&s[0], y, x, z, 1, &o[0], &o[1], &l, h);
		for (int f = 0; f < 3; f++)
			orc_spline3d_eval(&s[1 + f], y, x, z, 1, &o[4 + f], &o[7 + 3 * f], &l, h);
		orc_spline3d_eval(&s[4], y, x, z, 3, &o[16], &o[17], &l, &o[20]);
		for (int f = 0; f < 3; f++)
			orc_spline3d_eval(&s[5 + f], y, x, z, 1, &o[29 + f], &o[32 + 3 * f], &l, h);
	}
	for (int q = 0; q < 8; q++)
		free(s[q].coefs);
}

/* reference src/update.cpp:1111-1162 on a property table */
void orc_particle_stats(const double *props, long np, double out[4])
{
	double tke = 0, sij = 0, ux2 = 0, ux3 = 0, wz2 = 0, wz3 = 0;
	for (long q = 0; q < np; q++)
	{
		const double *o = props + 41 * q;
		tke += (o[4] * o[4] + o[5] * o[5] + o[6] * o[6]);
		double dudx = o[8], dvdx = o[11], dwdx = o[14];
		double dudy = o[7], dvdy = o[10], dwdy = o[13];
		double dudz = o[9], dvdz = o[12], dwdz = o[15];
		sij += (dudx * dudx + 0.5 * pow(dudy + dvdx, 2) + 0.5 * pow(dudz + dwdx, 2) + 0.5 * pow(dwdy + dvdz, 2) +
				dvdy * dvdy + dwdz * dwdz);
		ux2 += dudx * dudx;
		ux3 += dudx * dudx * dudx;
		wz2 += dwdz * dwdz;
		wz3 += dwdz * dwdz * dwdz;
	}
	tke /= np;
	sij /= np;
	ux2 /= np;
	ux3 /= np;
	wz2 /= np;
	wz3 /= np;
	out[0] = tke;
	out[1] = sij;
	out[2] = ux3 / pow(ux2, 1.5);
	out[3] = wz3 / pow(wz2, 1.5);
}

static void orc_free_splines(orc_spline s[4])
{
	for (int q = 0; q < 4; q++)
	{
		free(s[q].coefs);
		s[q].coefs = NULL;
	}
}

int orc_run(const orc_params *p, double *W[5], int nsteps, int spline_mode, long np,
			double *pos, double *U, double *dt_hist, orc_stats *stats)
{
	const long Nt = (long)p->nt * p->nt * p->nt;
	double *Fx[5], *Fy[5], *Fz[5];
	for (int q = 0; q < 5; q++)
	{
		Fx[q] = (double *)calloc((size_t)Nt, sizeof(double));
		Fy[q] = (double *)calloc((size_t)Nt, sizeof(double));
		Fz[q] = (double *)calloc((size_t)Nt, sizeof(double));
	}
	orc_spline s[4];
	memset(s, 0, sizeof(s));
	double g[3], l, h[9];

	orc_halo(p, W);
	double dt = orc_timestep(p, W);
	orc_build_field_splines(p, W, spline_mode, s, stats != NULL);
	for (long q = 0; q < np; q++)
		for (int c = 0; c < 3; c++)
			orc_spline3d_eval(&s[1 + c], pos[3 * q], pos[3 * q + 1], pos[3 * q + 2], 0, &U[3 * q + c], g, &l, h);
	int ns = 0;
	for (int it = 0; it < nsteps; it++)
	{
		if (stats && it % 10 == 0)
			orc_print_stats(p, W, &s[0], &s[1], &s[2], &s[3], &stats[ns++]);
		orc_free_splines(s);
		orc_step(p, W, Fx, Fy, Fz, dt);
		orc_build_field_splines(p, W, spline_mode, s, stats != NULL);
		for (long q = 0; q < np; q++)
		{
			orc_heun(&pos[3 * q], &U[3 * q], &s[1], &s[2], &s[3], dt);
			for (int c = 0; c < 3; c++)
				orc_spline3d_eval(&s[1 + c], pos[3 * q], pos[3 * q + 1], pos[3 * q + 2], 0, &U[3 * q + c], g, &l, h);
		}
		if (dt_hist)
			dt_hist[it] = dt;
		dt = orc_timestep(p, W);
	}
	if (stats && nsteps % 10 == 0)
		orc_print_stats(p, W, &s[0], &s[1], &s[2], &s[3], &stats[ns++]);
	orc_free_splines(s);
	for (int q = 0; q < 5; q++)
	{
		free(Fx[q]);
		free(Fy[q]);
		free(Fz[q]);
	}
	return ns;
}
