// C ABI of libgkm_b200.so (declarations and contracts in include/gkm.h).
//
// One handle = one periodic cube resident on one GPU.  Two state buffers of
// 5 x nt^3 doubles alternate: the current state W and the accumulator A that
// the sweeps fill and the z sweep turns into the next state.  dt, t and the
// step count stay on the device (DevClock), so a step never waits for the
// host; with use_graphs the whole step is replayed as one CUDA graph per
// buffer parity.
#include "gkm.h"
#include "gkm_handle.h"

#include <cuda.h>   // CUtensorMap and its enums (the encoder comes from the driver at run time)

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using gkm::DevClock;
using gkm::FieldConst;
using gkm_host::cuda_fail;
using gkm_host::fail;

// Thomas tables of the spline line solves (arrays of N + 1): natural dp_1 = 4,
// m_i = 1/dp_{i-1}, dp_i = 4 - m_i; periodic (Sherman-Morrison, gamma = -4)
// dp_0 = 8, dp_i = b_i - m_i with b_{N-1} = 4.25, z = B^-1 (-4, 0, .., 0, 1).
void gkm::spline_line_tables(int N, int periodic, double* mt, double* dp, double* z, double* denom)
{
    for (int i = 0; i <= N; i++) mt[i] = dp[i] = z[i] = 0.0;
    *denom = 0.0;
    if (!periodic) {
        dp[1] = 4.0;
        for (int i = 2; i <= N - 2; i++) {
            mt[i] = 1.0 / dp[i - 1];
            dp[i] = 4.0 - mt[i];
        }
        return;
    }
    dp[0] = 8.0;
    for (int i = 1; i < N; i++) {
        mt[i] = 1.0 / dp[i - 1];
        dp[i] = ((i == N - 1) ? 4.25 : 4.0) - mt[i];
    }
    double rp = -4.0;
    z[0] = rp;
    for (int i = 1; i < N; i++) {
        double r = (i == N - 1) ? 1.0 : 0.0;
        rp = r - mt[i] * rp;
        z[i] = rp;
    }
    z[N - 1] = z[N - 1] / dp[N - 1];
    for (int i = N - 2; i >= 0; i--) z[i] = (z[i] - z[i + 1]) / dp[i];
    *denom = 1.0 + (z[0] + (-0.25) * z[N - 1]);
}

namespace {
constexpr int kStatsBlocks = 148 * 4;

enum GraphKind { kGraphEulerian = 0, kGraphFull = 1, kGraphParticles = 2 };
constexpr int kSplinePasses = 9;   // 3 components x 3 axes
}  // namespace

namespace {

void spline_tables(int N, int periodic, std::vector<double>& mt, std::vector<double>& dp, std::vector<double>& z,
                   double& denom)
{
    mt.assign(N + 1, 0.0);
    dp.assign(N + 1, 0.0);
    z.assign(N + 1, 0.0);
    gkm::spline_line_tables(N, periodic, mt.data(), dp.data(), z.data(), &denom);
}

gkm::SplineTables device_tables(const gkm_handle* h)
{
    const int N1 = h->grid.npts + 1;
    return gkm::SplineTables{h->tables, h->tables + N1, h->tables + 2 * N1, h->denom};
}

long long coef_count(const gkm_handle* h)
{
    long long M = h->grid.npts + h->grid.pad;
    return M * M * M;
}

void destroy_graphs(gkm_handle* h)
{
    for (int k = 0; k < 3; k++)
        for (int p = 0; p < 2; p++) {
            if (h->graph[k][p]) cudaGraphExecDestroy(h->graph[k][p]);
            h->graph[k][p] = nullptr;
            h->graph_np[k][p] = -1;
        }
}

// tensor maps, 4 per buffer and window variant: x slab, y slab, z brick, z slab box (the mixed
// form has the maps of its one window).  sweep_tmap: the map of buffer W for the slab copies of
// direction dir; sweep_tmap_acc: the map of buffer A for the z sweep's accumulator bricks;
// sweep_tmap_wb: the map of buffer W for the mixed z sweep's FP64 state bricks
const void* tmap_at(const gkm_handle* h, const double* buf, int variant, int kind)
{
    if (!h->d_tmaps) return nullptr;
    const int b = (buf == h->buf[0]) ? 0 : (buf == h->buf[1] ? 1 : -1);
    if (b < 0) return nullptr;
    return h->d_tmaps + sizeof(CUtensorMap) * (size_t)((b * gkm::kSweepVariants64 + variant) * 4 + kind);
}
const void* sweep_tmap(const gkm_handle* h, const double* W, int dir, int variant)
{
    return tmap_at(h, W, variant, dir == 2 ? 3 : dir);
}
const void* sweep_tmap_acc(const gkm_handle* h, const double* A, int dir, int variant)
{
    return dir == 2 ? tmap_at(h, A, variant, 2) : nullptr;
}
const void* sweep_tmap_wb(const gkm_handle* h, const double* W, int dir, int variant)
{
    return (dir == 2 && h->cfg.precision == GKM_PREC_MIXED) ? tmap_at(h, W, variant, 2) : nullptr;
}

// Encode the tensor maps: each buffer as a 4-D tensor (k, i, j, q) of doubles, dims (nt, nt, nt, 5);
// boxes (WB, 1, WA, 5) for the x sweep's slabs (window j x k at one i), (WB, WA, 1, 5) for the y
// sweep's (window i x k at one j), (2, TB, TA, 5) for the z sweep's accumulator bricks (two k-cells
// of the window i x j) and (2, WB, WA, 5) for its slabs (two k-planes of the window and its halo).
// The row strides must be multiples of 16 bytes, so nt must be even; otherwise (or without the
// driver entry point) the sweeps move every value with cp.async and plain loads and stores.
cudaError_t setup_tensor_maps(gkm_handle* h)
{
    if (h->fc.nt % 2) return cudaSuccess;
    const bool mixed = h->cfg.precision == GKM_PREC_MIXED;
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        cudaGetLastError();
        return cudaSuccess;
    }
    const Encode encode = reinterpret_cast<Encode>(fn);
    const cuuint64_t nt = (cuuint64_t)h->fc.nt;
    const cuuint64_t dims[4] = {nt, nt, nt, 5};
    const cuuint64_t strides[3] = {nt * 8, nt * nt * 8, nt * nt * nt * 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const int nmaps = 2 * gkm::kSweepVariants64 * 4;
    std::vector<CUtensorMap> maps((size_t)nmaps);
    for (int b = 0; b < 2; b++)
        for (int v = 0; v < (mixed ? gkm::kSweepVariants32 : gkm::kSweepVariants64); v++)
            for (int d = 0; d < 4; d++) {
                const gkm::SweepShape sh = gkm::sweep_shape(mixed, v);
                const cuuint32_t WB = (cuuint32_t)sh.TB + 2, WA = (cuuint32_t)sh.TA + 2;
                const cuuint32_t boxes[4][4] = {
                    {WB, 1u, WA, 5}, {WB, WA, 1u, 5}, {2u, (cuuint32_t)sh.TB, (cuuint32_t)sh.TA, 5}, {2u, WB, WA, 5}};
                const cuuint32_t* box = boxes[d];
                CUresult r = encode(&maps[(size_t)((b * gkm::kSweepVariants64 + v) * 4 + d)],
                                    CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, h->buf[b], dims, strides, box, estr,
                                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                if (r != CUDA_SUCCESS) return cudaSuccess;   // keep the cp.async path
            }
    cudaError_t e = cudaMalloc(&h->d_tmaps, sizeof(CUtensorMap) * (size_t)nmaps);
    if (e == cudaSuccess)
        e = cudaMemcpy(h->d_tmaps, maps.data(), sizeof(CUtensorMap) * (size_t)nmaps, cudaMemcpyHostToDevice);
    return e;
}

cudaError_t launch_sweep_any(gkm_handle* h, int dir, gkm::SweepArgs a)
{
    const SweepChoice& c = h->sweep[dir];
    a.seg_len = c.seg_len;
    a.tmap = sweep_tmap(h, a.W, dir, c.variant);
    a.tmap_acc = sweep_tmap_acc(h, a.A, dir, c.variant);
    a.tmap_wb = sweep_tmap_wb(h, a.W, dir, c.variant);
    a.wait_probe = h->cfg.test_wait_probe;
    if (h->cfg.precision == GKM_PREC_MIXED) return gkm::launch_sweep_mixed(dir, c.variant, a, c.nseg, h->stream);
    return gkm::launch_sweep(dir, c.variant, a, c.nseg, h->stream);
}

// segments along the sweep normal: enough CTAs for ~4 waves of the CTAs an SM holds
SweepChoice default_choice(const FieldConst& fc, bool mixed, int variant)
{
    const gkm::SweepShape sh = gkm::sweep_shape(mixed, variant);
    const long long tiles = (long long)((fc.n + sh.TB - 1) / sh.TB) * ((fc.n + sh.TA - 1) / sh.TA);
    long long nseg = (148LL * sh.ctas * 4 + tiles - 1) / tiles;
    long long maxseg = fc.n / 16 > 1 ? fc.n / 16 : 1;
    if (nseg > maxseg) nseg = maxseg;
    if (nseg < 1) nseg = 1;
    SweepChoice c;
    c.variant = variant;
    c.seg_len = (int)((fc.n + nseg - 1) / nseg);
    c.nseg = (fc.n + c.seg_len - 1) / c.seg_len;
    return c;
}

// enqueue one Eulerian step on h->stream (no host synchronisation)
cudaError_t enqueue_eulerian(gkm_handle* h)
{
    gkm::SweepArgs a{};
    a.W = h->buf[h->parity];
    a.A = h->buf[h->parity ^ 1];
    a.fc = h->fc;
    a.clock = h->clock;
    a.parity = h->parity;
    a.dt_fixed_mode = h->dt_fixed_mode;
    a.dt_fixed = h->dt_fixed;
    for (int d = 0; d < 3; d++) {
        cudaError_t e = launch_sweep_any(h, d, a);
        if (e != cudaSuccess) return e;
    }
    h->launches += 4;
    return gkm::launch_halo(h->buf[h->parity ^ 1], h->fc, h->clock, 1, h->parity ^ 1, h->dt_fixed_mode, h->dt_fixed,
                            h->stream);
}

cudaError_t enqueue_splines(gkm_handle* h, const double* W)
{
    if (h->spline_f32) {
        h->launches += kSplinePasses;
        return gkm::launch_spline_build_f32(W, h->fc, h->grid, device_tables(h), h->coef32[0], h->coef32[1],
                                            h->coef32[2], h->scratch, h->stream);
    }
    if (h->d_self && (W == h->buf[0] || W == h->buf[1])) {
        gkm::EnsembleWork w{};
        w.line0 = h->d_self_off;
        w.line1 = h->d_self_off + 2;
        w.warp2 = h->d_self_off + 4;
        h->launches += 3;
        return gkm::launch_ensemble_splines(h->d_self, w, h->self_totals, 1, W == h->buf[0] ? 0 : 1, h->stream);
    }
    h->launches += kSplinePasses;
    return gkm::launch_spline_build(W, h->fc, h->grid, device_tables(h), h->coef[0], h->coef[1], h->coef[2],
                                    h->scratch, h->stream);
}

// Set up the component-batched spline build where it pays: when one component's N^2 lines
// leave most of the GPU's thread slots (148 SMs x 2048) idle, and the device has room for two
// more scratch arrays.  Larger grids fill the GPU per component already.
cudaError_t setup_batched_splines(gkm_handle* h)
{
    const long long N = h->grid.npts, M = N + h->grid.pad;
    if (h->cfg.spline_build == 1 || h->spline_f32) return cudaSuccess;
    if (h->cfg.spline_build == 0 && 3 * N * N > 2LL * 148 * 2048) return cudaSuccess;
    const size_t scratch_bytes = sizeof(double) * (size_t)(M * M * N);
    size_t free_b = 0, total_b = 0;
    cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) return e;
    if (free_b < 2 * scratch_bytes + ((size_t)8 << 30)) return cudaSuccess;   // keep 8 GB for the caller
    for (int k = 0; k < 2; k++) {
        e = cudaMalloc(&h->scratch_extra[k], scratch_bytes);
        if (e != cudaSuccess) return e;
    }
    gkm::MemberDev md;
    std::memset(&md, 0, sizeof(md));
    md.buf[0] = h->buf[0];
    md.buf[1] = h->buf[1];
    md.clock = h->clock;
    md.fc = h->fc;
    md.grid = h->grid;
    md.tb = device_tables(h);
    for (int c = 0; c < 3; c++) md.coef[c] = h->coef[c];
    md.scratch[0] = h->scratch;
    md.scratch[1] = h->scratch_extra[0];
    md.scratch[2] = h->scratch_extra[1];
    const long long off[6] = {0, 3 * N * N, 0, 3 * M * N, 0, 3 * ((M * M + 31) / 32)};
    h->self_totals[0] = off[1];
    h->self_totals[1] = off[3];
    h->self_totals[2] = off[5];
    e = cudaMalloc(&h->d_self, sizeof(md));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_self_off, sizeof(off));
    if (e == cudaSuccess) e = cudaMemcpy(h->d_self, &md, sizeof(md), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_self_off, off, sizeof(off), cudaMemcpyHostToDevice);
    return e;
}

gkm::ParticleArrays arrays_of(double* const a[6])
{
    return gkm::ParticleArrays{{a[0], a[1], a[2], a[3], a[4], a[5]}};
}

// order the particles by spline-cell blocks (into the sorted copy), then Heun from the sorted
// copy back into the particle arrays with the dt of the last Eulerian step
cudaError_t enqueue_advect(gkm_handle* h)
{
    if (h->np <= 0) return cudaSuccess;
    int nl = 0;
    cudaError_t e = gkm::launch_particle_sort(h->grid, h->np, arrays_of(h->P), arrays_of(h->P_sorted), h->tag,
                                              h->tag_sorted, h->sort_keys, h->sort_counts, h->sort_temp, &nl,
                                              h->stream);
    h->launches += nl + 1;
    if (e != cudaSuccess) return e;
    h->launches += 1;
    if (h->spline_f32) {
        const float* c32[3] = {h->coef32[0], h->coef32[1], h->coef32[2]};
        return gkm::launch_particles_heun(c32, h->grid, h->clock, h->np, arrays_of(h->P_sorted), arrays_of(h->P),
                                          h->tag_sorted, h->tag, h->stream);
    }
    const double* c[3] = {h->coef[0], h->coef[1], h->coef[2]};
    return gkm::launch_particles_heun(c, h->grid, h->clock, h->np, arrays_of(h->P_sorted), arrays_of(h->P),
                                      h->tag_sorted, h->tag, h->stream);
}

// splines of the state W and Heun advection with the dt of the last Eulerian step
cudaError_t enqueue_particles(gkm_handle* h, const double* W)
{
    if (h->np <= 0) return cudaSuccess;
    cudaError_t e = enqueue_splines(h, W);
    if (e != cudaSuccess) return e;
    return enqueue_advect(h);
}

// the body of Evolve's loop: Eulerian step, splines of the new state, particles
cudaError_t enqueue_full(gkm_handle* h)
{
    cudaError_t e = enqueue_eulerian(h);
    if (e != cudaSuccess) return e;
    return enqueue_particles(h, h->buf[h->parity ^ 1]);
}

cudaError_t enqueue_kind(gkm_handle* h, int kind)
{
    if (kind == kGraphFull) return enqueue_full(h);
    if (kind == kGraphParticles) return enqueue_particles(h, h->buf[h->parity]);
    return enqueue_eulerian(h);
}

gkm_status run_steps(gkm_handle* h, int32_t nsteps, int kind)
{
    if (!h) return GKM_ERR_ARG;
    if (nsteps < 0) return fail(h, GKM_ERR_ARG, "nsteps < 0");
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    for (int s = 0; s < nsteps; s++) {
        const int p = h->parity;
        if (h->cfg.use_graphs) {
            if (!h->graph[kind][p] || h->graph_np[kind][p] != h->np) {
                if (h->graph[kind][p]) cudaGraphExecDestroy(h->graph[kind][p]);
                h->graph[kind][p] = nullptr;
                cudaGraph_t g = nullptr;
                const int64_t before = h->launches;
                CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
                cudaError_t e = enqueue_kind(h, kind);
                cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
                h->graph_kernels[kind][p] = h->launches - before;
                h->launches = before;   // counted when the graph is replayed
                if (e != cudaSuccess) return cuda_fail(h, e, "capture step");
                if (e2 != cudaSuccess) return cuda_fail(h, e2, "cudaStreamEndCapture");
                e = cudaGraphInstantiate(&h->graph[kind][p], g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
                h->graph_np[kind][p] = h->np;
            }
            CK(h, cudaGraphLaunch(h->graph[kind][p], h->stream));
            h->launches += h->graph_kernels[kind][p];
        } else {
            cudaError_t e = enqueue_kind(h, kind);
            if (e != cudaSuccess) return cuda_fail(h, e, "step launch");
        }
        if (kind != kGraphParticles) h->parity ^= 1;
        // the particle path leaves the splines of the current state built
        h->splines_valid = (kind != kGraphEulerian && h->np > 0);
    }
    return GKM_OK;
}

gkm_status reduce_wave(gkm_handle* h)
{
    h->launches += 1;
    CK(h, cudaMemsetAsync(&h->clock->wave[h->parity], 0, sizeof(unsigned long long), h->stream));
    CK(h, gkm::launch_wave_reduce(h->buf[h->parity], h->fc, h->clock, h->parity, h->stream));
    return GKM_OK;
}

gkm_status read_clock(gkm_handle* h, DevClock* c)
{
    CK(h, cudaMemcpyAsync(c, h->clock, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (c->status & 2) return fail(h, GKM_ERR_CUDA, "a bulk tensor copy of a sweep did not complete in time");
    if (c->status & 1) return fail(h, GKM_ERR_NONFINITE, "state holds a non-finite value or non-positive density");
    return GKM_OK;
}

gkm_status ensure_splines(gkm_handle* h)
{
    if (h->splines_valid) return GKM_OK;
    CK(h, enqueue_splines(h, h->buf[h->parity]));
    h->splines_valid = true;
    return GKM_OK;
}

// upload index of the particle in each device slot (the arrays are kept in spline-cell order)
gkm_status host_tags(gkm_handle* h, std::vector<long long>& tags)
{
    tags.resize((size_t)h->np);
    if (h->np == 0) return GKM_OK;
    CK(h, cudaMemcpyAsync(tags.data(), h->tag, sizeof(long long) * (size_t)h->np, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    for (long long t : tags)
        if (t < 0 || t >= h->np) return fail(h, GKM_ERR_STATE, "particle tags corrupted");
    return GKM_OK;
}

// the five further splines of the reference's 8-field generateSplines
// (src/update.cpp:1200-1233) and getParticleProp for every particle
// (src/ParticleTrack.cpp:99-113) into h->props; allocates on first use
gkm_status compute_props(gkm_handle* h)
{
    if (h->spline_f32)
        return fail(h, GKM_ERR_CONFIG, "particle properties need FP64 velocity-spline coefficients");
    gkm_status s = ensure_splines(h);
    if (s != GKM_OK) return s;
    const long long M = h->grid.npts + h->grid.pad;
    for (int c = 0; c < 5; c++)
        if (!h->prop_coef[c]) CK(h, cudaMalloc(&h->prop_coef[c], sizeof(double) * (size_t)(M * M * M)));
    if (!h->lap_nodes) CK(h, cudaMalloc(&h->lap_nodes, sizeof(double) * (size_t)h->fc.nt3));
    if (!h->props && h->cap > 0) CK(h, cudaMalloc(&h->props, sizeof(double) * gkm::kPropCount * (size_t)h->cap));
    const gkm::SplineTables tb = device_tables(h);
    const double* W = h->buf[h->parity];
    CK(h, gkm::launch_spline_source(W, h->fc, h->grid, tb, gkm::kSplineDensity, h->prop_coef[0], h->scratch,
                                    h->stream));
    CK(h, gkm::launch_spline_source(W, h->fc, h->grid, tb, gkm::kSplinePressure, h->prop_coef[1], h->scratch,
                                    h->stream));
    for (int f = 0; f < 3; f++) {
        CK(h, gkm::launch_lap_nodes(h->coef[f], h->grid, h->fc, h->lap_nodes, h->stream));
        CK(h, gkm::launch_spline_source(h->lap_nodes, h->fc, h->grid, tb, gkm::kSplinePlain, h->prop_coef[2 + f],
                                        h->scratch, h->stream));
    }
    h->launches += 2 * 3 + 3 * (1 + 3);
    if (h->np > 0) {
        const double* c8[8] = {h->prop_coef[0], h->coef[0], h->coef[1], h->coef[2],
                               h->prop_coef[1], h->prop_coef[2], h->prop_coef[3], h->prop_coef[4]};
        CK(h, gkm::launch_particle_props(c8, h->grid, h->np, h->P[0], h->P[1], h->P[2], h->props, h->stream));
        h->launches += 1;
    }
    return GKM_OK;
}

}  // namespace

// host copy of the property table, particle-major (np x kPropCount); used by the writers too
gkm_status gkm_host_props(gkm_handle* h, double* out)
{
    gkm_status s = compute_props(h);
    if (s != GKM_OK || h->np == 0) return s;
    std::vector<double> tmp((size_t)gkm::kPropCount * (size_t)h->np);
    CK(h, cudaMemcpyAsync(tmp.data(), h->props, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    std::vector<long long> tags;
    s = host_tags(h, tags);
    if (s != GKM_OK) return s;
    const size_t np = (size_t)h->np;
    for (size_t p = 0; p < np; p++)
        for (int q = 0; q < gkm::kPropCount; q++) out[(size_t)tags[p] * gkm::kPropCount + q] = tmp[(size_t)q * np + p];
    return GKM_OK;
}

extern "C" {

int gkm_abi_version(void) { return GKM_ABI_VERSION; }

void gkm_config_default(gkm_config* cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->cfl = 0.10;
    cfg->visc_law = GKM_VISC_SUTHERLAND;
    cfg->spline_mode = GKM_SPLINE_NATURAL_GHOST3;
    cfg->precision = GKM_PREC_FP64;
    cfg->device = 0;
    cfg->use_graphs = 1;
}

const char* gkm_last_error(const gkm_handle* h) { return h ? h->err.c_str() : "null handle"; }

int gkm_nt(const gkm_handle* h) { return h ? h->fc.nt : 0; }

gkm_status gkm_create(const gkm_config* cfg, gkm_handle** out)
{
    if (!cfg || !out) return GKM_ERR_ARG;
    *out = nullptr;
    const gkm_params& P = cfg->params;
    if (P.n < 4 || P.n > 2048) return GKM_ERR_CONFIG;
    if (!(P.gam > 1.0) || !(P.den0 > 0.0) || !(P.p0 > 0.0) || !(P.mu0 >= 0.0) || !(cfg->cfl > 0.0))
        return GKM_ERR_CONFIG;
    if (cfg->visc_law < 0 || cfg->visc_law > 1 || cfg->spline_mode < 0 || cfg->spline_mode > 1) return GKM_ERR_CONFIG;
    if (cfg->precision < GKM_PREC_FP64 || cfg->precision > GKM_PREC_MIXED || cfg->max_particles < 0)
        return GKM_ERR_CONFIG;
    if (cfg->spline_build < 0 || cfg->spline_build > 2) return GKM_ERR_CONFIG;
    if (cfg->test_wait_probe < 0 || cfg->test_wait_probe > 1) return GKM_ERR_CONFIG;
    if (cfg->spline_precision < GKM_SPLINE_COEF_FP64 || cfg->spline_precision > GKM_SPLINE_COEF_FP32)
        return GKM_ERR_CONFIG;
    const int K = (int)((5.0 - 3.0 * P.gam) / (P.gam - 1.0));   // src/FlowField.cpp:42
    if (K < 0) return GKM_ERR_CONFIG;

    gkm_handle* h = new gkm_handle();
    h->cfg = *cfg;
    FieldConst& fc = h->fc;
    fc.n = P.n;
    fc.nt = P.n + 6;
    fc.nt3 = (long long)fc.nt * fc.nt * fc.nt;
    fc.K = K;
    fc.visc = cfg->visc_law;
    fc.gam = P.gam;
    fc.gm1 = P.gam - 1;
    fc.dx = 2.0 * (std::atan(1.0) * 4.0) / P.n;   // src/FlowField.cpp:46
    fc.inv_dx = 1 / fc.dx;
    fc.mu0 = P.mu0;
    fc.T0 = P.p0 / (287.0 * P.den0);               // src/FlowField.cpp:47
    fc.cfl = cfg->cfl;
    // working units of the mixed-precision sweeps
    fc.p0 = P.p0;
    fc.u_s = std::sqrt(P.p0 / P.den0);
    fc.inv_rho_s = 1.0 / P.den0;
    fc.inv_m_s = 1.0 / (P.den0 * fc.u_s);
    fc.inv_E_s = 1.0 / P.p0;
    fc.inv_T0 = 1.0 / fc.T0;
    fc.eps_rho = 1e-10 * fc.inv_rho_s * fc.inv_rho_s;
    fc.eps_m = 1e-10 * fc.inv_m_s * fc.inv_m_s;
    fc.eps_T = 1e-10 * fc.inv_T0 * fc.inv_T0;
    fc.fscale[0] = P.den0 * fc.dx;
    fc.fscale[1] = fc.fscale[2] = fc.fscale[3] = P.den0 * fc.u_s * fc.dx;
    fc.fscale[4] = P.p0 * fc.dx;

    for (int d = 0; d < 3; d++) h->sweep[d] = default_choice(fc, cfg->precision == GKM_PREC_MIXED, 0);

    auto bail = [&](cudaError_t e, const char* where) {
        gkm_status s = cuda_fail(h, e, where);
        std::fprintf(stderr, "gkm_create: %s\n", h->err.c_str());
        gkm_destroy(h);
        return s;
    };
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) return bail(e, "cudaSetDevice");
    e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(e, "cudaStreamCreate");
    h->stream = h->own_stream;
    for (int b = 0; b < 2; b++) {
        e = cudaMalloc(&h->buf[b], sizeof(double) * 5 * (size_t)fc.nt3);
        if (e != cudaSuccess) return bail(e, "cudaMalloc(state)");
    }
    e = cudaMalloc(&h->clock, sizeof(DevClock));
    if (e != cudaSuccess) return bail(e, "cudaMalloc(clock)");
    e = cudaMemset(h->clock, 0, sizeof(DevClock));
    if (e != cudaSuccess) return bail(e, "cudaMemset(clock)");

    // splines
    h->grid.periodic = cfg->spline_mode == GKM_SPLINE_PERIODIC;
    h->grid.npts = h->grid.periodic ? fc.n : fc.nt;
    h->grid.pad = h->grid.periodic ? 3 : 2;
    if (h->grid.periodic) {
        h->grid.start = 0.5 * fc.dx;
        h->grid.dinv = 1.0 / fc.dx;
    } else {
        // src/Interpolation.cpp:11-26 with sta = 0; spacing (end-start)/(num-1)
        double s = (0 - 3) * fc.dx + 0.5 * fc.dx;
        double en = s + (fc.nt - 1) * fc.dx;
        h->grid.start = s;
        h->grid.dinv = 1.0 / ((en - s) / (double)(fc.nt - 1));
    }
    {
        std::vector<double> mt, dp, z;
        spline_tables(h->grid.npts, h->grid.periodic, mt, dp, z, h->denom);
        const size_t N1 = (size_t)h->grid.npts + 1;
        e = cudaMalloc(&h->tables, sizeof(double) * 3 * N1);
        if (e != cudaSuccess) return bail(e, "cudaMalloc(tables)");
        std::vector<double> all;
        all.insert(all.end(), mt.begin(), mt.end());
        all.insert(all.end(), dp.begin(), dp.end());
        all.insert(all.end(), z.begin(), z.end());
        e = cudaMemcpy(h->tables, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return bail(e, "cudaMemcpy(tables)");
    }
    const long long M = h->grid.npts + h->grid.pad, N = h->grid.npts;
    h->spline_f32 = cfg->spline_precision == GKM_SPLINE_COEF_FP32;
    for (int c = 0; c < 3; c++) {
        if (h->spline_f32) e = cudaMalloc(&h->coef32[c], sizeof(float) * (size_t)(M * M * M));
        else e = cudaMalloc(&h->coef[c], sizeof(double) * (size_t)(M * M * M));
        if (e != cudaSuccess) return bail(e, "cudaMalloc(spline coefficients)");
    }
    e = cudaMalloc(&h->scratch, sizeof(double) * (size_t)(M * M * N));
    if (e != cudaSuccess) return bail(e, "cudaMalloc(spline scratch)");
    // particles
    h->cap = cfg->max_particles;
    if (h->cap > 0) {
        for (int c = 0; c < 6; c++) {
            e = cudaMalloc(&h->P[c], sizeof(double) * (size_t)h->cap);
            if (e == cudaSuccess) e = cudaMalloc(&h->P_sorted[c], sizeof(double) * (size_t)h->cap);
            if (e != cudaSuccess) return bail(e, "cudaMalloc(particles)");
        }
        const long long nb = (h->grid.npts + 7) / 8, nkeys = nb * nb * nb;
        e = cudaMalloc(&h->tag, sizeof(long long) * (size_t)h->cap);
        if (e == cudaSuccess) e = cudaMalloc(&h->tag_sorted, sizeof(long long) * (size_t)h->cap);
        if (e == cudaSuccess) e = cudaMalloc(&h->sort_keys, sizeof(unsigned) * (size_t)h->cap);
        if (e == cudaSuccess) e = cudaMalloc(&h->sort_counts, sizeof(unsigned) * (size_t)nkeys);
        if (e == cudaSuccess) e = cudaMalloc(&h->sort_temp, sizeof(unsigned) * (size_t)gkm::scan_temp_size(nkeys));
        if (e != cudaSuccess) return bail(e, "cudaMalloc(particle ordering)");
    }
    e = cudaMalloc(&h->partials, sizeof(gkm::StatsPartial) * kStatsBlocks);
    if (e != cudaSuccess) return bail(e, "cudaMalloc(stats)");
    e = cudaMalloc(&h->stats_out, sizeof(double) * 32);
    if (e != cudaSuccess) return bail(e, "cudaMalloc(stats)");
    e = gkm::sweep_prepare();
    if (e == cudaSuccess) e = gkm::sweep_mixed_prepare();
    if (e != cudaSuccess) return bail(e, "sweep_prepare");
    e = setup_batched_splines(h);
    if (e != cudaSuccess) return bail(e, "batched spline build");
    e = setup_tensor_maps(h);
    if (e != cudaSuccess) return bail(e, "tensor maps");
    *out = h;
    return GKM_OK;
}

gkm_status gkm_destroy(gkm_handle* h)
{
    if (!h) return GKM_ERR_ARG;
    if (h->owner) return fail(h, GKM_ERR_STATE, "the handle belongs to an ensemble (gkm_ensemble_destroy frees it)");
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    destroy_graphs(h);
    for (int b = 0; b < 2; b++) cudaFree(h->buf[b]);
    cudaFree(h->clock);
    cudaFree(h->tables);
    for (int c = 0; c < 3; c++) {
        cudaFree(h->coef[c]);
        cudaFree(h->coef32[c]);
    }
    cudaFree(h->scratch);
    for (int k = 0; k < 2; k++) cudaFree(h->scratch_extra[k]);
    cudaFree(h->d_self);
    cudaFree(h->d_self_off);
    cudaFree(h->d_tmaps);
    for (int c = 0; c < 6; c++) {
        cudaFree(h->P[c]);
        cudaFree(h->P_sorted[c]);
    }
    cudaFree(h->tag);
    cudaFree(h->tag_sorted);
    cudaFree(h->sort_keys);
    cudaFree(h->sort_counts);
    cudaFree(h->sort_temp);
    for (int c = 0; c < 5; c++) cudaFree(h->prop_coef[c]);
    cudaFree(h->lap_nodes);
    cudaFree(h->props);
    for (cudaEvent_t e : h->pipe_ev) cudaEventDestroy(e);
    for (cudaStream_t s : {h->pipe_in, h->pipe_out, h->pipe_comp[0], h->pipe_comp[1], h->pipe_comp[2], h->pipe_comp[3],
                           h->pipe_halo})
        if (s) cudaStreamDestroy(s);
    cudaFree(h->partials);
    cudaFree(h->stats_out);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
    return GKM_OK;
}

gkm_status gkm_upload_state(gkm_handle* h, const double* const W[5])
{
    if (!h || !W) return GKM_ERR_ARG;
    for (int q = 0; q < 5; q++)
        if (!W[q]) return fail(h, GKM_ERR_ARG, "W[q] is NULL");
    const size_t bytes = sizeof(double) * (size_t)h->fc.nt3;
    double* dst = h->buf[h->parity];
    for (int q = 0; q < 5; q++)
        CK(h, cudaMemcpyAsync(dst + (size_t)q * h->fc.nt3, W[q], bytes, cudaMemcpyDefault, h->stream));
    h->launches += 1;
    CK(h, gkm::launch_halo(dst, h->fc, h->clock, 0, h->parity, 0, 0.0, h->stream));
    CK(h, cudaMemsetAsync(&h->clock->status, 0, sizeof(int), h->stream));
    gkm_status s = reduce_wave(h);
    if (s != GKM_OK) return s;
    h->state_loaded = true;
    h->splines_valid = false;
    return GKM_OK;
}

gkm_status gkm_download_state(gkm_handle* h, double* const W[5])
{
    if (!h || !W) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    const size_t bytes = sizeof(double) * (size_t)h->fc.nt3;
    const double* src = h->buf[h->parity];
    for (int q = 0; q < 5; q++) {
        if (!W[q]) return fail(h, GKM_ERR_ARG, "W[q] is NULL");
        CK(h, cudaMemcpyAsync(W[q], src + (size_t)q * h->fc.nt3, bytes, cudaMemcpyDefault, h->stream));
    }
    DevClock c;
    return read_clock(h, &c);
}

gkm_status gkm_timestep(gkm_handle* h, double* dt_out)
{
    if (!h) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    gkm_status s = reduce_wave(h);
    if (s != GKM_OK) return s;
    DevClock c;
    s = read_clock(h, &c);
    if (s != GKM_OK) return s;
    double mw;
    unsigned long long bits = c.wave[h->parity];
    std::memcpy(&mw, &bits, sizeof(mw));
    if (h->dt_fixed_mode) destroy_graphs(h);
    h->dt_fixed_mode = 0;
    if (dt_out) *dt_out = h->fc.cfl * h->fc.dx / mw;   // src/update.cpp:1053
    return GKM_OK;
}

gkm_status gkm_set_dt(gkm_handle* h, double dt)
{
    if (!h) return GKM_ERR_ARG;
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(h, GKM_ERR_ARG, "dt must be >= 0 and finite");
    h->dt_fixed_mode = dt > 0.0;
    h->dt_fixed = dt;
    destroy_graphs(h);
    return GKM_OK;
}

gkm_status gkm_evolve_eulerian(gkm_handle* h, int32_t nsteps) { return run_steps(h, nsteps, kGraphEulerian); }

gkm_status gkm_step(gkm_handle* h, int32_t nsteps) { return run_steps(h, nsteps, kGraphFull); }

gkm_status gkm_evolve_particles(gkm_handle* h) { return run_steps(h, 1, kGraphParticles); }

gkm_status gkm_step_timed(gkm_handle* h, int32_t nsteps, int32_t with_particles, double ms[7])
{
    if (!h || !ms || nsteps < 0) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    for (int k = 0; k < 7; k++) ms[k] = 0.0;
    cudaEvent_t ev[7];
    for (int k = 0; k < 7; k++) CK(h, cudaEventCreate(&ev[k]));
    gkm_status st = GKM_OK;
    for (int s = 0; s < nsteps && st == GKM_OK; s++) {
        gkm::SweepArgs a{};
        a.W = h->buf[h->parity];
        a.A = h->buf[h->parity ^ 1];
        a.fc = h->fc;
        a.clock = h->clock;
        a.parity = h->parity;
        a.dt_fixed_mode = h->dt_fixed_mode;
        a.dt_fixed = h->dt_fixed;
        cudaError_t e = cudaEventRecord(ev[0], h->stream);
        for (int d = 0; d < 3 && e == cudaSuccess; d++) {
            e = launch_sweep_any(h, d, a);
            if (e == cudaSuccess) e = cudaEventRecord(ev[d + 1], h->stream);
        }
        if (e == cudaSuccess)
            e = gkm::launch_halo(h->buf[h->parity ^ 1], h->fc, h->clock, 1, h->parity ^ 1, h->dt_fixed_mode,
                                 h->dt_fixed, h->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[4], h->stream);
        h->launches += 4;
        h->parity ^= 1;
        const bool parts = with_particles && h->np > 0;
        if (e == cudaSuccess && parts) e = enqueue_splines(h, h->buf[h->parity]);
        if (e == cudaSuccess) e = cudaEventRecord(ev[5], h->stream);
        if (e == cudaSuccess && parts) e = enqueue_advect(h);
        if (e == cudaSuccess) e = cudaEventRecord(ev[6], h->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[6]);
        if (e != cudaSuccess) {
            st = cuda_fail(h, e, "gkm_step_timed");
            break;
        }
        float t;
        for (int k = 0; k < 6; k++) {
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            ms[k] += t;
        }
        cudaEventElapsedTime(&t, ev[0], ev[6]);
        ms[6] += t;
        h->splines_valid = parts;
    }
    for (int k = 0; k < 7; k++) cudaEventDestroy(ev[k]);
    return st;
}

gkm_status gkm_autotune(gkm_handle* h, int32_t reps)
{
    if (!h || reps < 1) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    const bool mixed = h->cfg.precision == GKM_PREC_MIXED;
    const int nvar = mixed ? gkm::kSweepVariants32 : gkm::kSweepVariants64;
    // the sweeps leave W untouched (they write the accumulator A only); the clock
    // they also touch is saved here and put back afterwards
    DevClock saved;
    CK(h, cudaMemcpyAsync(&saved, h->clock, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    cudaEvent_t e0, e1;
    CK(h, cudaEventCreate(&e0));
    CK(h, cudaEventCreate(&e1));
    gkm::SweepArgs a{};
    a.W = h->buf[h->parity];
    a.A = h->buf[h->parity ^ 1];
    a.fc = h->fc;
    a.clock = h->clock;
    a.parity = h->parity;
    a.dt_fixed_mode = h->dt_fixed_mode;
    a.dt_fixed = h->dt_fixed;
    const int nsegs[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 24, 32};
    gkm_status st = GKM_OK;
    for (int d = 0; d < 3 && st == GKM_OK; d++) {
        SweepChoice best = h->sweep[d];
        float best_ms = 1e30f;
        for (int v = 0; v < nvar && st == GKM_OK; v++) {
            if (!mixed && v == 2 && !gkm::ws_ready()) continue;   // not available on this build
            int last_len = -1;
            for (int ns : nsegs) {
                SweepChoice c;
                c.variant = v;
                c.seg_len = (h->fc.n + ns - 1) / ns;
                if (c.seg_len < 8 || c.seg_len == last_len) continue;
                last_len = c.seg_len;
                c.nseg = (h->fc.n + c.seg_len - 1) / c.seg_len;
                h->sweep[d] = c;
                cudaError_t e = launch_sweep_any(h, d, a);   // warm-up
                if (e == cudaSuccess) e = cudaEventRecord(e0, h->stream);
                for (int r = 0; r < reps && e == cudaSuccess; r++) e = launch_sweep_any(h, d, a);
                if (e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0.f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                if (e != cudaSuccess) {
                    st = cuda_fail(h, e, "gkm_autotune");
                    break;
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best = c;
                }
            }
        }
        h->sweep[d] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemcpyAsync(h->clock, &saved, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream);
    cudaStreamSynchronize(h->stream);
    destroy_graphs(h);
    return st;
}

gkm_status gkm_sweep_config(const gkm_handle* h, int32_t out[12])
{
    if (!h || !out) return GKM_ERR_ARG;
    const bool mixed = h->cfg.precision == GKM_PREC_MIXED;
    for (int d = 0; d < 3; d++) {
        const gkm::SweepShape sh = gkm::sweep_shape(mixed, h->sweep[d].variant);
        out[4 * d + 0] = h->sweep[d].variant;
        out[4 * d + 1] = sh.TB;
        out[4 * d + 2] = sh.TA;
        out[4 * d + 3] = h->sweep[d].seg_len;
    }
    return GKM_OK;
}

gkm_status gkm_set_sweep_config(gkm_handle* h, const int32_t in[6])
{
    if (!h || !in) return GKM_ERR_ARG;
    const bool mixed = h->cfg.precision == GKM_PREC_MIXED;
    const int nvar = mixed ? gkm::kSweepVariants32 : gkm::kSweepVariants64;
    for (int d = 0; d < 3; d++) {
        const int v = in[2 * d], L = in[2 * d + 1];
        if (v < 0 || v >= nvar || L < 1) return fail(h, GKM_ERR_ARG, "sweep variant or segment length out of range");
        if (!mixed && v == 2 && !gkm::ws_ready())
            return fail(h, GKM_ERR_CONFIG, "the warp-specialized sweep is not available on this build");
    }
    for (int d = 0; d < 3; d++) {
        h->sweep[d].variant = in[2 * d];
        h->sweep[d].seg_len = in[2 * d + 1] < h->fc.n ? in[2 * d + 1] : h->fc.n;
        h->sweep[d].nseg = (h->fc.n + h->sweep[d].seg_len - 1) / h->sweep[d].seg_len;
    }
    destroy_graphs(h);
    return GKM_OK;
}

gkm_status gkm_launch_count(const gkm_handle* h, int64_t* count)
{
    if (!h || !count) return GKM_ERR_ARG;
    *count = h->launches;
    return GKM_OK;
}

gkm_status gkm_probe_fma_peak(int32_t device, double* fp64_tflops, double* fp32_tflops)
{
    if (!fp64_tflops || !fp32_tflops) return GKM_ERR_ARG;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = gkm::probe_fma_peak(fp64_tflops, fp32_tflops);
    return e == cudaSuccess ? GKM_OK : GKM_ERR_CUDA;
}

namespace {

// copy engines can read and write these asynchronously: pinned host or device memory
bool async_capable(const double* p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// The plug point evolve(W, dt) as a pipeline over chunks of y-planes: the host -> device copy of
// chunk c+1, the x/y/z sweeps of chunk c and the device -> host copy of chunk c-1 overlap.  A
// chunk's sweeps need the input planes within 3 of it (y stencil) with their ghosts; the input
// arrives in parts that end three planes into the next chunk, and a halo stream wraps each part's
// ghosts as it lands (the periodic y-ghost planes come from the last three interior planes,
// copied first, and from the first part), so chunk c waits for part c.  Each chunk writes only
// its own planes of the accumulator, so two compute streams run consecutive chunks concurrently.
// Results equal the one-shot path.
//
// Chunk boundaries (interior y-planes): the first and the last chunk hold 16 planes, so the
// sweeps start after a short copy and the copy after the last sweep is short; the others hold C
// planes.  Every boundary but n is a multiple of 16, and so of every window height.
std::vector<int> pipeline_chunks(int n, int C)
{
    std::vector<int> B{0};
    if (n <= 2 * C) {
        for (int j = C; j < n; j += C) B.push_back(j);
    } else {
        const int last = ((n - 1) / 16) * 16;   // the last chunk: 1..16 planes
        B.push_back(16);
        for (int j = 16 + C; j < last; j += C) B.push_back(j);
        if (B.back() != last) B.push_back(last);
    }
    B.push_back(n);
    return B;
}

gkm_status evolve_pipelined(gkm_handle* h, double* const W[5], double dt)
{
    const FieldConst& fc = h->fc;
    const int n = fc.n;
    const size_t plane = (size_t)fc.nt * fc.nt, nt3 = (size_t)fc.nt3;
    int C = h->pipe_chunk ? h->pipe_chunk : ((n / 8 + 15) / 16) * 16;   // a multiple of every window height
    if (C < 16) C = 16;
    const std::vector<int> B = pipeline_chunks(n, C);
    const int K = (int)B.size() - 1;
    const int S = h->pipe_streams;
    if (!h->pipe_in) {
        for (cudaStream_t* s : {&h->pipe_in, &h->pipe_out, &h->pipe_comp[0], &h->pipe_comp[1], &h->pipe_comp[2],
                                &h->pipe_comp[3], &h->pipe_halo})
            CK(h, cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
    }
    const size_t nev = 3 * (size_t)K + 2;
    while (h->pipe_ev.size() < nev) {
        cudaEvent_t e;
        CK(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->pipe_ev.push_back(e);
    }
    cudaEvent_t ev_start = h->pipe_ev[0], ev_done_out = h->pipe_ev[1];
    cudaEvent_t* ev_in = &h->pipe_ev[2];
    cudaEvent_t* ev_out = &h->pipe_ev[2 + K];
    cudaEvent_t* ev_cp = &h->pipe_ev[2 + 2 * K];   // copy of part c landed
    double* Wd = h->buf[h->parity];
    double* A = h->buf[h->parity ^ 1];
    DevClock* ck = h->clock;
    const bool mixed = h->cfg.precision == GKM_PREC_MIXED;

    // the clock: this step's dt, the next wave slot cleared (the z sweeps reduce into it), status
    CK(h, cudaMemcpyAsync(&ck->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemsetAsync(&ck->wave[h->parity ^ 1], 0, sizeof(unsigned long long), h->stream));
    CK(h, cudaMemsetAsync(&ck->status, 0, sizeof(int), h->stream));
    CK(h, cudaEventRecord(ev_start, h->stream));
    for (cudaStream_t s : {h->pipe_in, h->pipe_out, h->pipe_comp[0], h->pipe_comp[1], h->pipe_comp[2], h->pipe_comp[3],
                           h->pipe_halo})
        CK(h, cudaStreamWaitEvent(s, ev_start, 0));

    auto copy_in = [&](int J0, int J1) -> cudaError_t {
        for (int q = 0; q < 5; q++) {
            const size_t off = (size_t)q * nt3 + (size_t)J0 * plane;
            cudaError_t e = cudaMemcpyAsync(Wd + off, W[q] + (size_t)J0 * plane, sizeof(double) * (J1 - J0) * plane,
                                            cudaMemcpyDefault, h->pipe_in);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    auto copy_out = [&](int J0, int J1, cudaStream_t s) -> cudaError_t {
        for (int q = 0; q < 5; q++) {
            const size_t off = (size_t)q * nt3 + (size_t)J0 * plane;
            cudaError_t e = cudaMemcpyAsync(W[q] + (size_t)J0 * plane, A + off, sizeof(double) * (J1 - J0) * plane,
                                            cudaMemcpyDefault, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };

    // copy-in stream, copies only and back to back: the last three interior planes first, then one
    // part per chunk, planes [3 + B[c] + 3, 3 + B[c+1] + 3) (the first part from plane 3, the last
    // to n + 3): chunk c's planes after its first three, which came with part c-1, and the first
    // three planes of chunk c+1, all the y stencil of chunk c reaches beyond it.  One copy per
    // component and part: many small copies in both directions at once lose bus bandwidth.  The
    // halo stream wraps each part's ghosts once it has landed (a kernel between the copies would
    // leave the copy engine idle while it runs), and chunk c's sweeps wait for part c.
    auto part_end = [&](int c) { return c + 1 < K ? std::min(3 + B[c + 1] + 3, n + 3) : n + 3; };
    CK(h, copy_in(n, n + 3));
    for (int c = 0; c < K; c++) {
        const int P0 = c == 0 ? 3 : part_end(c - 1), P1 = part_end(c);
        const int P1c = std::min(P1, n);   // planes n..n+2 are already in
        if (P1c > P0) CK(h, copy_in(P0, P1c));
        CK(h, cudaEventRecord(ev_cp[c], h->pipe_in));
    }
    for (int c = 0; c < K; c++) {
        const int P0 = c == 0 ? 3 : part_end(c - 1), P1 = part_end(c);
        CK(h, cudaStreamWaitEvent(h->pipe_halo, ev_cp[c], 0));
        if (c == 0) {   // the y-ghost planes: images of planes n..n+2 (copied first) and of planes 3..5
            CK(h, gkm::launch_halo_planes(Wd, fc, 0, 3, h->pipe_halo));
            CK(h, gkm::launch_halo_planes(Wd, fc, n + 3, n + 6, h->pipe_halo));
            h->launches += 2;
        }
        if (P1 > P0) {
            CK(h, gkm::launch_halo_planes(Wd, fc, P0, P1, h->pipe_halo));
            h->launches += 1;
        }
        CK(h, cudaEventRecord(ev_in[c], h->pipe_halo));
    }

    // compute: chunk c on compute stream c % S, after its own planes and the first three of chunk c+1
    gkm::SweepArgs a{};
    a.W = Wd;
    a.A = A;
    a.fc = fc;
    a.clock = ck;
    a.parity = h->parity;
    a.dt_fixed_mode = 1;
    a.dt_fixed = dt;
    a.skip_clock_init = 1;
    for (int c = 0; c < K; c++) {
        cudaStream_t s = h->pipe_comp[c % S];
        CK(h, cudaStreamWaitEvent(s, ev_in[c], 0));
        const int j0 = B[c], j1 = B[c + 1];
        for (int d = 0; d < 3; d++) {
            gkm::SweepArgs ad = a;
            // y: one segment through the chunk; x, z: segments of at most C faces, so a chunk's
            // launch has enough CTAs to fill the SMs beside the other stream's (measured: 256^3
            // -2.5 %, 512^3 -8 % per pinned step against the whole-cube segment lengths)
            ad.seg_len = (d == 1) ? j1 - j0 : std::min(h->sweep[d].seg_len, C);
            const int v = h->sweep[d].variant;
            ad.tmap = sweep_tmap(h, ad.W, d, v);
            ad.tmap_acc = sweep_tmap_acc(h, ad.A, d, v);
            ad.tmap_wb = sweep_tmap_wb(h, ad.W, d, v);
            CK(h, mixed ? gkm::launch_sweep_mixed_rows(d, v, ad, j0, j1, s) : gkm::launch_sweep_rows(d, v, ad, j0, j1, s));
        }
        CK(h, gkm::launch_halo_planes(A, fc, 3 + j0, 3 + j1, s));
        h->launches += 4;
        CK(h, cudaEventRecord(ev_out[c], s));
        CK(h, cudaStreamWaitEvent(h->pipe_out, ev_out[c], 0));
        CK(h, copy_out(3 + j0, 3 + j1, h->pipe_out));
    }
    CK(h, cudaEventRecord(ev_done_out, h->pipe_out));

    // the y-ghost planes of the new state, the clock, the last copies
    for (int c = 0; c < K; c++) CK(h, cudaStreamWaitEvent(h->stream, ev_out[c], 0));
    CK(h, gkm::launch_halo_planes(A, fc, 0, 3, h->stream));
    CK(h, gkm::launch_halo_planes(A, fc, n + 3, n + 6, h->stream));
    CK(h, gkm::launch_clock_finish(ck, dt, h->stream));
    h->launches += 3;
    CK(h, copy_out(0, 3, h->stream));
    CK(h, copy_out(n + 3, n + 6, h->stream));
    CK(h, cudaStreamWaitEvent(h->stream, ev_done_out, 0));
    h->parity ^= 1;
    h->state_loaded = true;
    h->splines_valid = false;
    DevClock c;
    return read_clock(h, &c);
}

}  // namespace

gkm_status gkm_set_pipeline(gkm_handle* h, int32_t chunk_planes, int32_t compute_streams)
{
    if (!h) return GKM_ERR_ARG;
    if (chunk_planes < 0 || chunk_planes % 16 || compute_streams < 1 || compute_streams > 4)
        return fail(h, GKM_ERR_ARG, "chunk_planes: 0 or a multiple of 16; compute_streams: 1..4");
    h->pipe_chunk = chunk_planes;
    h->pipe_streams = compute_streams;
    return GKM_OK;
}

gkm_status gkm_evolve(gkm_handle* h, double* const W[5], double dt)
{
    if (!h || !W) return GKM_ERR_ARG;
    if (!(dt > 0.0)) return fail(h, GKM_ERR_ARG, "dt must be > 0");
    bool pipelined = true;
    for (int q = 0; q < 5; q++) pipelined = pipelined && W[q] && async_capable(W[q]);
    if (pipelined) return evolve_pipelined(h, W, dt);
    gkm_status s = gkm_upload_state(h, (const double* const*)W);
    if (s != GKM_OK) return s;
    const int mode = h->dt_fixed_mode;
    const double val = h->dt_fixed;
    h->dt_fixed_mode = 1;
    h->dt_fixed = dt;
    cudaError_t e = enqueue_eulerian(h);
    h->dt_fixed_mode = mode;
    h->dt_fixed = val;
    if (e != cudaSuccess) return cuda_fail(h, e, "evolve");
    h->parity ^= 1;
    h->splines_valid = false;
    return gkm_download_state(h, W);
}

gkm_status gkm_get_clock(gkm_handle* h, double* t, double* dt, int64_t* iter)
{
    if (!h) return GKM_ERR_ARG;
    DevClock c;
    gkm_status s = read_clock(h, &c);
    if (t) *t = c.t;
    if (dt) *dt = c.dt;
    if (iter) *iter = c.iter;
    return s;
}

gkm_status gkm_synchronize(gkm_handle* h)
{
    if (!h) return GKM_ERR_ARG;
    CK(h, cudaStreamSynchronize(h->stream));
    return GKM_OK;
}

gkm_status gkm_particles_upload(gkm_handle* h, int64_t np, const double* pos, const double* U)
{
    if (!h || (np > 0 && !pos)) return GKM_ERR_ARG;
    if (np < 0 || np > h->cap) return fail(h, GKM_ERR_ARG, "particle count exceeds max_particles");
    std::vector<double> tmp((size_t)np);
    for (int c = 0; c < 6; c++) {
        const double* src = c < 3 ? pos : U;
        if (!src) continue;
        for (int64_t p = 0; p < np; p++) tmp[(size_t)p] = src[3 * p + (c % 3)];
        CK(h, cudaMemcpyAsync(h->P[c], tmp.data(), sizeof(double) * (size_t)np, cudaMemcpyHostToDevice, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    if (np > 0) {   // tags: the upload order, restored by every download
        std::vector<long long> tags((size_t)np);
        for (int64_t p = 0; p < np; p++) tags[(size_t)p] = p;
        CK(h, cudaMemcpyAsync(h->tag, tags.data(), sizeof(long long) * (size_t)np, cudaMemcpyHostToDevice, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    h->np = np;
    if (!U && np > 0) {
        if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "U == NULL needs an uploaded state");
        gkm_status s = ensure_splines(h);
        if (s != GKM_OK) return s;
        const double* c[3] = {h->coef[0], h->coef[1], h->coef[2]};
        const float* c32[3] = {h->coef32[0], h->coef32[1], h->coef32[2]};
        h->launches += 1;
        if (h->spline_f32)
            CK(h, gkm::launch_particles_eval(c32, h->grid, np, h->P[0], h->P[1], h->P[2], h->P[3], h->P[4], h->P[5],
                                             h->stream));
        else
            CK(h, gkm::launch_particles_eval(c, h->grid, np, h->P[0], h->P[1], h->P[2], h->P[3], h->P[4], h->P[5],
                                             h->stream));
    }
    return GKM_OK;
}

gkm_status gkm_particles_download(gkm_handle* h, double* pos, double* U)
{
    if (!h) return GKM_ERR_ARG;
    std::vector<double> tmp((size_t)h->np);
    std::vector<long long> tags;
    gkm_status s = host_tags(h, tags);
    if (s != GKM_OK) return s;
    for (int c = 0; c < 6; c++) {
        double* dst = c < 3 ? pos : U;
        if (!dst) continue;
        CK(h, cudaMemcpyAsync(tmp.data(), h->P[c], sizeof(double) * (size_t)h->np, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (int64_t p = 0; p < h->np; p++) dst[3 * tags[(size_t)p] + (c % 3)] = tmp[(size_t)p];
    }
    DevClock c;
    return read_clock(h, &c);
}

gkm_status gkm_generate_splines(gkm_handle* h)
{
    if (!h) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    h->splines_valid = false;
    return ensure_splines(h);
}

gkm_status gkm_spline_coefs(gkm_handle* h, int32_t c, double* out, int64_t capacity)
{
    if (!h || !out || c < 0 || c > 2) return GKM_ERR_ARG;
    if (capacity < coef_count(h)) return fail(h, GKM_ERR_ARG, "capacity below (N+P)^3");
    gkm_status s = ensure_splines(h);
    if (s != GKM_OK) return s;
    if (h->spline_f32) {   // the stored floats, widened
        std::vector<float> tmp((size_t)coef_count(h));
        CK(h, cudaMemcpyAsync(tmp.data(), h->coef32[c], sizeof(float) * tmp.size(), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < tmp.size(); i++) out[i] = (double)tmp[i];
        return GKM_OK;
    }
    CK(h, cudaMemcpyAsync(out, h->coef[c], sizeof(double) * (size_t)coef_count(h), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return GKM_OK;
}

gkm_status gkm_stats_compute(gkm_handle* h, gkm_stats* out)
{
    if (!h || !out) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    gkm_status s = ensure_splines(h);
    if (s != GKM_OK) return s;
    const double* c[3] = {h->coef[0], h->coef[1], h->coef[2]};
    const float* c32[3] = {h->coef32[0], h->coef32[1], h->coef32[2]};
    h->launches += 4;
    if (h->spline_f32)
        CK(h, gkm::launch_stats(h->buf[h->parity], h->fc, h->grid, c32, h->partials, kStatsBlocks, h->stats_out,
                                h->stream));
    else
        CK(h, gkm::launch_stats(h->buf[h->parity], h->fc, h->grid, c, h->partials, kStatsBlocks, h->stats_out,
                                h->stream));
    double v[32];
    CK(h, cudaMemcpyAsync(v, h->stats_out, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    DevClock ck;
    s = read_clock(h, &ck);
    if (s != GKM_OK) return s;
    const gkm_params& P = h->cfg.params;
    const double gam = P.gam, Mt = P.Mt;
    out->t_over_t0 = ck.t / P.t0;
    out->TKE = v[0];
    out->Diss = v[1];
    out->SijSij = v[2];
    // src/update.cpp:793-798
    out->SKEWu = v[4] / std::pow(v[3], 1.5);
    out->SKEWv = v[7] / std::pow(v[6], 1.5);
    out->SKEWw = v[10] / std::pow(v[9], 1.5);
    out->KURTu = v[5] / std::pow(v[3], 2);
    out->KURTv = v[8] / std::pow(v[6], 2);
    out->KURTw = v[11] / std::pow(v[9], 2);
    // src/update.cpp:825-833
    out->Prms = v[16] / (gam * P.p0 * Mt * Mt);
    out->Trms = v[17] / ((gam - 1) * h->fc.T0 * Mt * Mt);
    out->Vrms = v[18] / (Mt * Mt / P.den0);
    return GKM_OK;
}

gkm_status gkm_particle_props(gkm_handle* h, double* props)
{
    if (!h || (h->np > 0 && !props)) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    return gkm_host_props(h, props);
}

gkm_status gkm_particle_stats_compute(gkm_handle* h, gkm_particle_stats* out)
{
    if (!h || !out) return GKM_ERR_ARG;
    if (!h->state_loaded) return fail(h, GKM_ERR_STATE, "no state uploaded");
    if (h->np <= 0) return fail(h, GKM_ERR_STATE, "no particles uploaded");
    gkm_status s = compute_props(h);
    if (s != GKM_OK) return s;
    h->launches += 2;
    CK(h, gkm::launch_particle_stats(h->props, h->np, h->partials, kStatsBlocks, h->stats_out, h->stream));
    double v[6];
    CK(h, cudaMemcpyAsync(v, h->stats_out, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    // src/update.cpp:1148-1155
    const double n = (double)h->np;
    out->TKE = v[0] / n;
    out->SijSij = v[1] / n;
    const double dudx2 = v[2] / n, dudx3 = v[3] / n, dwdz2 = v[4] / n, dwdz3 = v[5] / n;
    out->SKEWu = dudx3 / std::pow(dudx2, 1.5);
    out->SKEWw = dwdz3 / std::pow(dwdz2, 1.5);
    out->count = h->np;
    return GKM_OK;
}

gkm_status gkm_flux_faces(const double* in, int64_t nfaces, double gam, double dt, double dx, double* F)
{
    if (nfaces < 0 || (nfaces > 0 && (!in || !F))) return GKM_ERR_ARG;
    if (nfaces == 0) return GKM_OK;
    if (!(gam > 1.0)) return GKM_ERR_ARG;
    const int K = (int)((5.0 - 3.0 * gam) / (gam - 1.0));
    double *din = nullptr, *dF = nullptr;
    cudaError_t e = cudaMalloc(&din, sizeof(double) * 51 * (size_t)nfaces);
    if (e == cudaSuccess) e = cudaMalloc(&dF, sizeof(double) * 5 * (size_t)nfaces);
    if (e == cudaSuccess) e = cudaMemcpy(din, in, sizeof(double) * 51 * (size_t)nfaces, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = gkm::launch_flux_faces(din, nfaces, gam, K, dt, dx, dF, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(F, dF, sizeof(double) * 5 * (size_t)nfaces, cudaMemcpyDeviceToHost);
    cudaFree(din);
    cudaFree(dF);
    return e == cudaSuccess ? GKM_OK : GKM_ERR_CUDA;
}

gkm_status gkm_weno_faces(const double* stencils, int64_t n, double gam, double* Wl, double* Wr)
{
    if (n < 0 || (n > 0 && (!stencils || !Wl || !Wr))) return GKM_ERR_ARG;
    if (n == 0) return GKM_OK;
    double *ds = nullptr, *dl = nullptr, *dr = nullptr;
    cudaError_t e = cudaMalloc(&ds, sizeof(double) * 30 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dl, sizeof(double) * 5 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(double) * 5 * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(ds, stencils, sizeof(double) * 30 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = gkm::launch_weno_faces(ds, n, gam, dl, dr, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(Wl, dl, sizeof(double) * 5 * (size_t)n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(Wr, dr, sizeof(double) * 5 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(ds);
    cudaFree(dl);
    cudaFree(dr);
    return e == cudaSuccess ? GKM_OK : GKM_ERR_CUDA;
}

gkm_status gkm_set_stream(gkm_handle* h, void* stream)
{
    if (!h) return GKM_ERR_ARG;
    if (h->owner) return fail(h, GKM_ERR_STATE, "an ensemble member runs on the ensemble's stream");
    CK(h, cudaStreamSynchronize(h->stream));
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    destroy_graphs(h);
    return GKM_OK;
}

gkm_status gkm_device_state(gkm_handle* h, double** W)
{
    if (!h || !W) return GKM_ERR_ARG;
    *W = h->buf[h->parity];
    return GKM_OK;
}

}  // extern "C"
