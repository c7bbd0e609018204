/*
 * Driver around the UNMODIFIED reference CPU sources — TEST INFRASTRUCTURE ONLY.
 *
 * oracle/Makefile compiles src/{update,GKMflux,FlowField,param,ParticleTrack,
 * Interpolation}.cpp where they lie in the reference tree (flags of
 * makefileCPU_local:4,13 plus -D UseCPU), with oracle/shim/mpi.h (one rank)
 * and oracle/shim/bspline.h (project spline behind einspline's names), and
 * links this file into oracle/_ref/libgkm_ref.so.
 *
 * Main.cpp is replaced by gkmref_setup() (src/Main.cpp:15-41 with procDim
 * 1x1x1), and the body of Evolve's loop (src/update.cpp:124-170) by
 * gkmref_run(), which calls the reference's own functions in the same order
 * and skips only the file output (writeField, WriteReInit,
 * writeParticleData).  The CFL number is a compile-time macro of the reference
 * (src/param.h:20, 0.10); gkmref_set_cfl() recomputes dt = cfl*dx/maxVAL from
 * the maxVAL that the reference's timestep() leaves behind, the same formula
 * as src/update.cpp:1053 with another cfl.
 */
#include <chrono>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <unistd.h>

#include "param.h"
#include "update.h"
#include "FlowField.h"

extern ptype dt, t, maxVAL, TKE, Diss, SijSij, SKEWu, SKEWv, SKEWw, KURTu, KURTv, KURTw;
extern ptype part_TKE, part_SijSij, part_SKEWu, part_SKEWw;
extern int count, iter, sendSz;

namespace
{
struct RefState
{
	bool ready = false;
	double cflnum = 0.10;
	ptype *W[5] = {};
	ptype *Fx[5] = {}, *Fy[5] = {}, *Fz[5] = {};
	ptype *halo[12] = {};
	ptype *den = nullptr, *u = nullptr, *v = nullptr, *w = nullptr, *p = nullptr;
	ptype *lapU = nullptr, *lapV = nullptr, *lapW = nullptr;
	Particle *particles = nullptr;
	ptype *sendP[27] = {}, *recvP[27] = {};
	double stats_line[16] = {};
};
RefState S;

void halo() { HaloTransfer(S.W, S.halo[0], S.halo[1], S.halo[2], S.halo[3], S.halo[4], S.halo[5],
						   S.halo[6], S.halo[7], S.halo[8], S.halo[9], S.halo[10], S.halo[11]); }

void apply_cfl()
{
	timestep(S.W);
	dt = S.cflnum * dx / maxVAL;
}

void print_stats(UBspline_3d_d *sp[8])
{
	std::ostringstream os;
	std::streambuf *old = std::cout.rdbuf(os.rdbuf());
	PrintStats(S.W, sp);
	std::cout.rdbuf(old);
	std::istringstream is(os.str());
	for (int q = 0; q < 16; q++)
		if (!(is >> S.stats_line[q]))
			S.stats_line[q] = 0;
	/* full-precision copies of the values PrintStats keeps in globals */
	S.stats_line[1] = TKE;
	S.stats_line[2] = Diss;
	S.stats_line[3] = SijSij;
	S.stats_line[4] = SKEWu;
	S.stats_line[5] = SKEWv;
	S.stats_line[6] = SKEWw;
	S.stats_line[7] = KURTu;
	S.stats_line[8] = KURTv;
	S.stats_line[9] = KURTw;
}
} // namespace

extern "C"
{

/* src/Main.cpp:15-41 on one rank; icdir holds InitialConditions/{params,Init000,unirand,particleCount} */
int gkmref_setup(const char *icdir, double cflnum, int with_particles)
{
	char old[4096];
	if (!getcwd(old, sizeof(old)) || chdir(icdir) != 0)
		return -1;
	nprocs = 1;
	myrank_3d = 0;
	for (int d = 0; d < 3; d++)
	{
		procDim[d] = 1;
		procId[d] = 0;
	}
	GetParams();
	segment();
	for (int q = 0; q < 5; q++)
	{
		S.W[q] = new ptype[Nt_seg];
		S.Fx[q] = new ptype[Nt_seg]();
		S.Fy[q] = new ptype[Nt_seg]();
		S.Fz[q] = new ptype[Nt_seg]();
	}
	Initialize_DHIT(S.W);
	int hs = 5 * 3 * nt_segx * nt_segz;
	for (int b = 0; b < 12; b++)
		S.halo[b] = new ptype[hs];
	/* src/update.cpp:69-72 allocates these uninitialised; generateSplines writes
	 * lapU/V/W only at interior nodes (src/update.cpp:1217-1228), so the ghost
	 * nodes of the Laplacian splines keep the allocation's contents: zero pages
	 * at the reference's sizes (fresh mmap'd blocks).  Zero them here. */
	S.den = new ptype[Nt_seg]();
	S.u = new ptype[Nt_seg]();
	S.v = new ptype[Nt_seg]();
	S.w = new ptype[Nt_seg]();
	S.p = new ptype[Nt_seg]();
	S.lapU = new ptype[Nt_seg]();
	S.lapV = new ptype[Nt_seg]();
	S.lapW = new ptype[Nt_seg]();
	S.cflnum = cflnum;

	/* src/update.cpp:94-120 */
	halo();
	UBspline_3d_d *sp[8];
	generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
	apply_cfl();
	t = 0;
	::count = 0;
	iter = 0;
	if (with_particles)
	{
		sendSz = 8 * int(numparticles / (nc_segx * nprocs));
		int bufsz = sendSz < 9 ? 9 : sendSz; /* the reference writes slot 0 even when sendSz is 0 */
		for (int b = 0; b < 27; b++)
		{
			S.sendP[b] = new ptype[bufsz]();
			S.recvP[b] = new ptype[bufsz]();
		}
		S.particles = new Particle[int(1.5 * numparticles / nprocs) + 1];
		locateParticles(S.particles, sp);
	}
	for (int q = 0; q < 8; q++)
		destroy_Bspline(sp[q]);
	S.ready = true;
	return chdir(old) == 0 ? 0 : -2;
}

int gkmref_nt() { return nt_segx; }
double gkmref_dt() { return dt; }
double gkmref_dx() { return dx; }
double gkmref_time() { return t; }
int gkmref_count() { return ::count; }
void gkmref_set_cfl(double cflnum)
{
	S.cflnum = cflnum;
	apply_cfl();
}
void gkmref_set_dt(double v) { dt = v; }

void gkmref_get_W(double *out)
{
	for (int q = 0; q < 5; q++)
		std::memcpy(out + (size_t)q * Nt_seg, S.W[q], sizeof(double) * Nt_seg);
}
void gkmref_set_W(const double *in)
{
	for (int q = 0; q < 5; q++)
		std::memcpy(S.W[q], in + (size_t)q * Nt_seg, sizeof(double) * Nt_seg);
}
void gkmref_get_flux(int dir, double *out)
{
	ptype **F = dir == 0 ? S.Fx : dir == 1 ? S.Fy : S.Fz;
	for (int q = 0; q < 5; q++)
		std::memcpy(out + (size_t)q * Nt_seg, F[q], sizeof(double) * Nt_seg);
}

/* particles in the reference's order: pos (y,x,z), U (u,v,w), tag */
int gkmref_get_particles(double *pos, double *U, int *tags)
{
	for (int q = 0; q < ::count; q++)
	{
		for (int c = 0; c < 3; c++)
		{
			pos[3 * q + c] = S.particles[q].pos[c];
			U[3 * q + c] = S.particles[q].U[c];
		}
		tags[q] = S.particles[q].tagId;
	}
	return ::count;
}

/* one Eulerian step + halo + dt, src/update.cpp:147,154,167 */
void gkmref_eulerian_step()
{
	evolveEulerian(S.W, S.Fx, S.Fy, S.Fz);
	halo();
	apply_cfl();
	t += dt;
	iter++;
}

/* loop body of Evolve, src/update.cpp:127-169, without file output.
 * dt_hist[nsteps] receives the dt of each step; stats[16*k] the PrintStats
 * line of every step with iter % 10 == 0.  Returns the number of stats lines. */
int gkmref_run(int nsteps, double *dt_hist, double *stats, int max_stats)
{
	int ns = 0;
	for (int s = 0; s < nsteps; s++)
	{
		UBspline_3d_d *sp[8], *spn[3];
		generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
		for (int q = 0; q < ::count; q++)
			S.particles[q].getParticleProp(sp);
		if (S.particles)
			GetParticleStats(S.particles, sp);
		if (iter % 10 == 0)
		{
			print_stats(sp);
			if (stats && ns < max_stats)
				std::memcpy(stats + 16 * ns, S.stats_line, sizeof(S.stats_line));
			ns++;
		}
		if (dt_hist)
			dt_hist[s] = dt;
		evolveEulerian(S.W, S.Fx, S.Fy, S.Fz);
		halo();
		generateSplines(S.W, spn, S.u, S.v, S.w);
		if (S.particles)
			evolveParticles(S.particles, sp, spn, S.sendP, S.recvP);
		for (int q = 0; q < 8; q++)
			destroy_Bspline(sp[q]);
		for (int q = 0; q < 3; q++)
			destroy_Bspline(spn[q]);
		apply_cfl();
		t += dt;
		iter++;
	}
	return ns;
}

/* getParticleProp at the current positions, i.e. the start of the next loop
 * iteration (src/update.cpp:127,135-136): refreshes each particle's U */
void gkmref_particle_props()
{
	UBspline_3d_d *sp[8];
	generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
	for (int q = 0; q < ::count; q++)
		S.particles[q].getParticleProp(sp);
	for (int q = 0; q < 8; q++)
		destroy_Bspline(sp[q]);
}

/* PrintStats of the current field alone (the line the next loop iteration would print) */
void gkmref_stats(double *out16)
{
	UBspline_3d_d *sp[8];
	generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
	print_stats(sp);
	std::memcpy(out16, S.stats_line, sizeof(S.stats_line));
	for (int q = 0; q < 8; q++)
		destroy_Bspline(sp[q]);
}

/* Timing of the reference CPU path on this process's core:
 *  eulerian: evolveEulerian + HaloTransfer + timestep   (per step)
 *  particle: velocity splines (generateSplines, 3-field form) + evolveParticles
 *            + the velocity part of getParticleProp at the new positions. */
void gkmref_particle_props();

void gkmref_time_steps(int nsteps, double *sec_eulerian, double *sec_particles)
{
	using clk = std::chrono::steady_clock;
	double te = 0, tp = 0;
	/* the reference sets U by getParticleProp before any advection (src/update.cpp:135-136);
	 * class Particle leaves it uninitialised */
	if (S.particles && iter == 0)
		gkmref_particle_props();
	for (int s = 0; s < nsteps; s++)
	{
		UBspline_3d_d *spn[3];
		auto a = clk::now();
		evolveEulerian(S.W, S.Fx, S.Fy, S.Fz);
		halo();
		auto b = clk::now();
		if (S.particles)
		{
			generateSplines(S.W, spn, S.u, S.v, S.w);
			UBspline_3d_d *sp[8] = {spn[0], spn[0], spn[1], spn[2], spn[0], spn[0], spn[0], spn[0]};
			evolveParticles(S.particles, sp, spn, S.sendP, S.recvP);
			for (int q = 0; q < ::count; q++)
			{
				Particle &P = S.particles[q];
				eval_UBspline_3d_d_vg(spn[0], P.pos[0], P.pos[1], P.pos[2], &P.U[0], P.gradU);
				eval_UBspline_3d_d_vg(spn[1], P.pos[0], P.pos[1], P.pos[2], &P.U[1], P.gradV);
				eval_UBspline_3d_d_vg(spn[2], P.pos[0], P.pos[1], P.pos[2], &P.U[2], P.gradW);
			}
			for (int q = 0; q < 3; q++)
				destroy_Bspline(spn[q]);
		}
		auto c = clk::now();
		apply_cfl();
		auto d = clk::now();
		t += dt;
		iter++;
		te += std::chrono::duration<double>(b - a).count() + std::chrono::duration<double>(d - c).count();
		tp += std::chrono::duration<double>(c - b).count();
	}
	*sec_eulerian = te;
	*sec_particles = tp;
}

/* getParticleProp of every particle at its current position (the start of the
 * next loop iteration) as the property table of include/gkm.h: per particle
 * 41 values (DEN, gradD, U, gradU, gradV, gradW, P, gradP, hessP, lapU, lapV,
 * lapW, gradLapU, gradLapV, gradLapW; gradients in (y, x, z) order); tags
 * receives tagId.  Returns the particle count. */

int gkmref_particle_table(double *out, int *tags)
{
	gkmref_particle_props();
	for (int q = 0; q < ::count; q++)
	{
		const Particle &P = S.particles[q];
		double *o = out + 41 * (size_t)q;
		int m = 0;
		o[m++] = P.DEN;
		for (int a = 0; a < 3; a++) o[m++] = P.gradD[a];
		for (int a = 0; a < 3; a++) o[m++] = P.U[a];
		for (int a = 0; a < 3; a++) o[m++] = P.gradU[a];
		for (int a = 0; a < 3; a++) o[m++] = P.gradV[a];
		for (int a = 0; a < 3; a++) o[m++] = P.gradW[a];
		o[m++] = P.P;
		for (int a = 0; a < 3; a++) o[m++] = P.gradP[a];
		for (int a = 0; a < 9; a++) o[m++] = P.hessP[a];
		o[m++] = P.lapU;
		o[m++] = P.lapV;
		o[m++] = P.lapW;
		for (int a = 0; a < 3; a++) o[m++] = P.gradLapU[a];
		for (int a = 0; a < 3; a++) o[m++] = P.gradLapV[a];
		for (int a = 0; a < 3; a++) o[m++] = P.gradLapW[a];
		tags[q] = P.tagId;
	}
	return ::count;
}

/* GetParticleStats (src/update.cpp:1111-1162) after gkmref_particle_table */
void gkmref_particle_stats(double *out4)
{
	GetParticleStats(S.particles, nullptr);
	out4[0] = part_TKE;
	out4[1] = part_SijSij;
	out4[2] = part_SKEWu;
	out4[3] = part_SKEWw;
}

/* The reference's own writers (writeField, WriteReInit, writeParticleData;
 * src/update.cpp:1324-1422) on the current state, as at the top of a loop
 * iteration, into <dir>/Results/{Field,Particles,Time} and
 * <dir>/InitialCondition.  Returns 0 on success. */
int gkmref_write_outputs(const char *dir)
{
	char old[4096];
	if (!getcwd(old, sizeof(old)) || chdir(dir) != 0)
		return -1;
	UBspline_3d_d *sp[8];
	generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
	writeField(S.den, S.u, S.v, S.w, S.p);
	WriteReInit(S.W);
	if (S.particles)
	{
		for (int q = 0; q < ::count; q++)
			S.particles[q].getParticleProp(sp);
		writeParticleData(S.particles);
	}
	for (int q = 0; q < 8; q++)
		destroy_Bspline(sp[q]);
	return chdir(old) == 0 ? 0 : -2;
}

/* direct calls into the reference numerics, for single-face checks */
void gkmref_flux(const double *WL, const double *WR, const double *Wl, const double *Wr,
				 const double *DWxl, const double *DWxr, const double *DWyl, const double *DWyr,
				 const double *DWzl, const double *DWzr, double tau, double dt_, double dx_,
				 double gam_, double *F)
{
	::gam = gam_;
	::K = int((5.0 - 3.0 * gam_) / (gam_ - 1.0));
	ptype a[10][5];
	const double *src[10] = {WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr};
	for (int v = 0; v < 10; v++)
		for (int q = 0; q < 5; q++)
			a[v][q] = src[v][q];
	flux(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], tau, dt_, dx_, F);
}

void gkmref_weno(const double *s6x5, double gam_, double *Wl, double *Wr)
{
	::gam = gam_;
	ptype a[6][5];
	for (int o = 0; o < 6; o++)
		for (int q = 0; q < 5; q++)
			a[o][q] = s6x5[5 * o + q];
	ApplyWENO(a[0], a[1], a[2], a[3], a[4], a[5], Wl, Wr);
}

} // extern "C"
