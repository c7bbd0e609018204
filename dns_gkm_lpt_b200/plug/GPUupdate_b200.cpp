// GPUupdate_b200.cpp — the reference's GPU plug point implemented on libgkm_b200.so.
//
// In the reference's -D UseGPU build (makefileGPU) this one C++ file replaces
// src/GPUupdate.cu and src/GPUAlloc.cu.  It defines what the rest of that build
// calls:
//   DevAlloc::DevAlloc() / DevAlloc::~DevAlloc()       (src/GPUAlloc.h:8-26)
//   void evolve(ptype *W[5], DevAlloc *dev, ptype dt)   (src/GPUupdate.h:33)
// evolve() is reached from evolveEulerian(W, dev) (src/update.cpp:193-198) once
// per step of Evolve's loop; every other function of that build (HaloTransfer,
// generateSplines, evolveParticles, timestep, PrintStats, the writers) stays
// the reference's own.  It compiles against the reference's headers (they need
// no CUDA header) with -I<reference>/src -I<repo>/include and links with
// -L<repo>/dns_gkm_lpt_b200/lib -lgkm_b200.
//
// One GPU holds the whole periodic cube: the build must run with one rank
// (procDim 1 x 1 x 1), where the reference's halo exchange is the periodic wrap
// that gkm_evolve already applies to the ghosts it returns.
// gkm.h comes first: the reference's param.h defines cfl, R, pi and eps as object-like macros,
// and gkm_config has a member named cfl
#include "gkm.h"

#include "GPUupdate.h"   // void evolve(ptype *W[5], DevAlloc *dev, ptype dt); param.h globals
#include "GPUAlloc.h"    // class DevAlloc

#include <cstdio>
#include <cstdlib>

static const double kReferenceCfl = cfl;   // src/param.h:20
#undef cfl

namespace
{
gkm_handle *g_gkm = nullptr;   // the reference keeps one DevAlloc per rank; one handle here

void gkm_check(gkm_status s, const char *what)
{
	if (s != GKM_OK)
	{
		std::fprintf(stderr, "%s failed (status %d): %s\n", what, (int)s, gkm_last_error(g_gkm));
		std::abort();   // the reference has no error path; stop instead of continuing on a bad state
	}
}
} // namespace

// Replaces the 55 cudaMalloc'd device arrays of src/GPUAlloc.cu:3-68 by one handle (two state
// buffers, fluxes computed on the fly).  Reads the globals GetParams and segment set
// (src/FlowField.cpp:9-58, src/param.cpp:3-6).
DevAlloc::DevAlloc()
{
	d_W0 = d_W1 = d_W2 = d_W3 = d_W4 = nullptr;   // the handle owns the device memory
	if (nprocs != 1 || nc_segx != nc || nc_segy != nc || nc_segz != nc)
	{
		std::fprintf(stderr, "GPUupdate_b200: one rank holding the whole %d^3 cube is required (nprocs %d)\n", nc,
					 nprocs);
		std::abort();
	}
	gkm_config cfg;
	gkm_config_default(&cfg);
	cfg.params.n = nc_segx;
	cfg.params.gam = gam;
	cfg.params.den0 = den0;
	cfg.params.Mt = Mt;
	cfg.params.Re = Re;
	cfg.params.mu0 = mu0;
	cfg.params.p0 = p0;
	cfg.params.t0 = t0;
	cfg.cfl = kReferenceCfl;   // evolve() uses the caller's dt in any case
	gkm_check(gkm_create(&cfg, &g_gkm), "gkm_create");
}

DevAlloc::~DevAlloc()
{
	gkm_destroy(g_gkm);
	g_gkm = nullptr;
}

// src/GPUupdate.cu:79-219: W (host, Nt_seg values per component, ghosts of width 3) in, one
// Eulerian step with the caller's dt, W out with its ghosts already wrapped.  Pinned W
// (cudaHostAlloc, or cudaHostRegister on the reference's new[] arrays) pipelines the copies
// with the sweeps; pageable W takes one copy in and one out.
void evolve(ptype *W[5], DevAlloc * /*dev*/, ptype dt)
{
	gkm_check(gkm_evolve(g_gkm, W, dt), "gkm_evolve");
}
