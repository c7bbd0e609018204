/*
 * einspline entry points (names from the reference's call sites) implemented
 * on the project spline of oracle/gkm_oracle.c.  TEST INFRASTRUCTURE ONLY:
 * linked into oracle/_ref/ so the reference's own update.cpp,
 * ParticleTrack.cpp and Interpolation.cpp compile and run unchanged.
 */
#include "bspline.h"
#include "../gkm_oracle.h"

#include <stdlib.h>

static void to_orc(const UBspline_3d_d *s, orc_spline *o)
{
	o->coefs = s->coefs;
	o->n[0] = s->n0;
	o->n[1] = s->n1;
	o->n[2] = s->n2;
	o->periodic = s->periodic;
	for (int a = 0; a < 3; a++)
	{
		o->start[a] = s->start[a];
		o->dinv[a] = s->dinv[a];
	}
}

UBspline_3d_d *create_UBspline_3d_d(Ugrid g0, Ugrid g1, Ugrid g2, BCtype_d bc0, BCtype_d bc1, BCtype_d bc2, double *data)
{
	(void)bc1;
	(void)bc2;
	UBspline_3d_d *s = (UBspline_3d_d *)calloc(1, sizeof(UBspline_3d_d));
	Ugrid *g[3] = {&g0, &g1, &g2};
	s->periodic = bc0.lCode == PERIODIC;
	s->n0 = g0.num;
	s->n1 = g1.num;
	s->n2 = g2.num;
	for (int a = 0; a < 3; a++)
	{
		/* spacing as einspline derives it: (end-start)/(num-1), or /num if periodic */
		double delta = (g[a]->end - g[a]->start) / (double)(s->periodic ? g[a]->num : g[a]->num - 1);
		s->start[a] = g[a]->start;
		s->dinv[a] = 1.0 / delta;
	}
	int P = orc_spline_pad(s->periodic);
	size_t m = (size_t)(s->n0 + P) * (size_t)(s->n1 + P) * (size_t)(s->n2 + P);
	s->coefs = (double *)malloc(sizeof(double) * m);
	int n[3] = {s->n0, s->n1, s->n2};
	orc_spline3d_build(data, n, s->periodic, s->coefs, NULL);
	return s;
}

void destroy_Bspline(void *spline)
{
	UBspline_3d_d *s = (UBspline_3d_d *)spline;
	if (!s)
		return;
	free(s->coefs);
	free(s);
}

void eval_UBspline_3d_d(UBspline_3d_d *s, double a, double b, double c, double *val)
{
	orc_spline o;
	double g[3], l, h[9];
	to_orc(s, &o);
	orc_spline3d_eval(&o, a, b, c, 0, val, g, &l, h);
}

void eval_UBspline_3d_d_vg(UBspline_3d_d *s, double a, double b, double c, double *val, double *grad)
{
	orc_spline o;
	double l, h[9];
	to_orc(s, &o);
	orc_spline3d_eval(&o, a, b, c, 1, val, grad, &l, h);
}

void eval_UBspline_3d_d_vgl(UBspline_3d_d *s, double a, double b, double c, double *val, double *grad, double *lapl)
{
	orc_spline o;
	double h[9];
	to_orc(s, &o);
	orc_spline3d_eval(&o, a, b, c, 2, val, grad, lapl, h);
}

void eval_UBspline_3d_d_vgh(UBspline_3d_d *s, double a, double b, double c, double *val, double *grad, double *hess)
{
	orc_spline o;
	double l;
	to_orc(s, &o);
	orc_spline3d_eval(&o, a, b, c, 3, val, grad, &l, hess);
}
