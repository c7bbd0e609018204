/*
 * Driver around the reference's -D UseGPU build with the libgkm_b200 plug
 * point — TEST INFRASTRUCTURE ONLY.
 *
 * oracle/Makefile (target refgpu) compiles src/{update,FlowField,param,
 * ParticleTrack,Interpolation}.cpp where they lie in the reference tree,
 * update.cpp with -D UseGPU as makefileGPU does, together with
 * dns_gkm_lpt_b200/plug/GPUupdate_b200.cpp (in place of src/GPUupdate.cu and
 * src/GPUAlloc.cu) and this file (in place of src/Main.cpp), into
 * oracle/_ref/libgkm_ref_gpu.so linked against libgkm_b200.so.  So the
 * reference's own loop body runs, with its Eulerian step going
 * evolveEulerian(W, dev) -> evolve(W, dev, dt) -> gkm_evolve on the GPU.
 *
 * gkmrefgpu_setup(): src/Main.cpp:15-41 on one rank plus Evolve's set-up
 * (src/update.cpp:55-57 new DevAlloc, :94-120 halo, splines, dt, particles).
 * gkmrefgpu_run(): the body of Evolve's loop (src/update.cpp:124-170) without
 * the file output.  The CFL number is the reference's compile-time 0.10
 * (src/param.h:20); as in ref_driver.cpp, dt = cfl * dx / maxVAL is recomputed
 * with the test's cfl from the maxVAL the reference's timestep() leaves.
 */
#include <cstring>
#include <unistd.h>

#include "param.h"
#include "update.h"
#include "FlowField.h"

extern ptype dt, t, maxVAL;
extern int count, iter, sendSz;

namespace
{
struct RefState
{
	double cflnum = 0.10;
	ptype *W[5] = {};
	ptype *halo[12] = {};
	ptype *den = nullptr, *u = nullptr, *v = nullptr, *w = nullptr, *p = nullptr;
	ptype *lapU = nullptr, *lapV = nullptr, *lapW = nullptr;
	Particle *particles = nullptr;
	ptype *sendP[27] = {}, *recvP[27] = {};
	DevAlloc *dev = nullptr;
};
RefState S;

void halo() { HaloTransfer(S.W, S.halo[0], S.halo[1], S.halo[2], S.halo[3], S.halo[4], S.halo[5],
						   S.halo[6], S.halo[7], S.halo[8], S.halo[9], S.halo[10], S.halo[11]); }

void apply_cfl()
{
	timestep(S.W);
	dt = S.cflnum * dx / maxVAL;
}
} // namespace

extern "C"
{

int gkmrefgpu_setup(const char *icdir, double cflnum)
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
		S.W[q] = new ptype[Nt_seg];
	Initialize_DHIT(S.W);
	S.dev = new DevAlloc(); /* src/update.cpp:55-57 */
	int hs = 5 * 3 * nt_segx * nt_segz;
	for (int b = 0; b < 12; b++)
		S.halo[b] = new ptype[hs];
	S.den = new ptype[Nt_seg]();
	S.u = new ptype[Nt_seg]();
	S.v = new ptype[Nt_seg]();
	S.w = new ptype[Nt_seg]();
	S.p = new ptype[Nt_seg]();
	S.lapU = new ptype[Nt_seg]();
	S.lapV = new ptype[Nt_seg]();
	S.lapW = new ptype[Nt_seg]();
	S.cflnum = cflnum;

	halo();
	UBspline_3d_d *sp[8];
	generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
	apply_cfl();
	t = 0;
	::count = 0;
	iter = 0;
	sendSz = 8 * int(numparticles / (nc_segx * nprocs));
	int bufsz = sendSz < 9 ? 9 : sendSz;
	for (int b = 0; b < 27; b++)
	{
		S.sendP[b] = new ptype[bufsz]();
		S.recvP[b] = new ptype[bufsz]();
	}
	S.particles = new Particle[int(1.5 * numparticles / nprocs) + 1];
	locateParticles(S.particles, sp);
	for (int q = 0; q < 8; q++)
		destroy_Bspline(sp[q]);
	return chdir(old) == 0 ? 0 : -2;
}

/* the body of Evolve's loop, src/update.cpp:127-169, without file output;
 * dt_hist[nsteps] receives the dt of each step */
void gkmrefgpu_run(int nsteps, double *dt_hist)
{
	for (int s = 0; s < nsteps; s++)
	{
		UBspline_3d_d *sp[8], *spn[3];
		generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
		for (int q = 0; q < ::count; q++)
			S.particles[q].getParticleProp(sp);
		GetParticleStats(S.particles, sp);
		if (dt_hist)
			dt_hist[s] = dt;
		evolveEulerian(S.W, S.dev); /* src/update.cpp:150-152 -> evolve(W, dev, dt) */
		halo();
		generateSplines(S.W, spn, S.u, S.v, S.w);
		evolveParticles(S.particles, sp, spn, S.sendP, S.recvP);
		for (int q = 0; q < 8; q++)
			destroy_Bspline(sp[q]);
		for (int q = 0; q < 3; q++)
			destroy_Bspline(spn[q]);
		apply_cfl();
		t += dt;
		iter++;
	}
}

int gkmrefgpu_nt() { return nt_segx; }
double gkmrefgpu_dt() { return dt; }

void gkmrefgpu_get_W(double *out)
{
	for (int q = 0; q < 5; q++)
		std::memcpy(out + (size_t)q * Nt_seg, S.W[q], sizeof(double) * Nt_seg);
}

/* getParticleProp at the current positions (the next iteration's U), then the
 * particles in the reference's order: pos (y,x,z), U (u,v,w), tag */
int gkmrefgpu_get_particles(double *pos, double *U, int *tags)
{
	UBspline_3d_d *sp[8];
	generateSplines(S.W, sp, S.den, S.u, S.v, S.w, S.p, S.lapU, S.lapV, S.lapW);
	for (int q = 0; q < ::count; q++)
		S.particles[q].getParticleProp(sp);
	for (int q = 0; q < 8; q++)
		destroy_Bspline(sp[q]);
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

/* delete dev at the end of Evolve: DevAlloc::~DevAlloc releases the GPU handle */
void gkmrefgpu_finish()
{
	delete S.dev;
	S.dev = nullptr;
}

} // extern "C"
