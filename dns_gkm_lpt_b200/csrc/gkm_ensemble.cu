// Ensemble C ABI (declarations and contracts in include/gkm.h).
//
// An ensemble is a set of ordinary handles (one periodic cube each, any grid
// size) that share one stream.  Each stage of a step is one launch over the
// flattened work of all members: the device keeps an array of MemberDev (the
// members' buffers, clocks, constants and spline/particle arrays) and, per
// stage, prefix offsets of every member's work items; a kernel maps a global
// item to (member, local item) by binary search over the offsets.  The
// per-member arithmetic is the single-cube device code, so each member evolves
// exactly as it would alone.
//
// Sweeps: one window variant per direction for all members (one launch has one
// block shape), and a segment length per member (the autotuner picks one per
// grid size: short segments give many items, long ones load fewer extra slabs
// and compute fewer extra faces).  The work list holds the members with the
// longest items first and the persistent CTAs take items from a counter, so
// the short items fill the end of the launch.
#include "gkm_handle.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

using gkm::DevClock;
using gkm::MemberDev;

namespace {

// offset arrays in d_off, each nm + 1 long longs
// kOrderX..Z hold, per sweep direction, the member at each position of the work list
enum OffsetSet { kItemX = 0, kItemY, kItemZ, kGhost, kLine0, kLine1, kWarp2, kPart, kOrderX, kOrderY, kOrderZ,
                 kNumSets };

}  // namespace

struct gkm_ensemble {
    std::vector<gkm_handle*> mem;
    std::vector<double*> extra_scratch;   // two more spline scratch arrays per member (unless it has its own)
    bool mixed = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    SweepChoice sweep[3];                 // window variant shared by all members (seg_len unused)
    std::vector<int> seg[3];              // segment length of each member, per direction
    unsigned long long* d_next = nullptr; // work counters of the three sweep launches
    MemberDev* d_mem = nullptr;
    long long* d_off = nullptr;
    std::vector<long long> h_off;         // kNumSets x (nm + 1), as last uploaded
    long long total[kNumSets] = {};
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [with_particles][parity]
    int64_t graph_kernels[2][2] = {{0, 0}, {0, 0}};
    int64_t launches = 0;
    std::string err;
};

namespace {

gkm_status efail(gkm_ensemble* E, gkm_status s, const std::string& msg)
{
    if (E) E->err = msg;
    return s;
}

gkm_status ecuda(gkm_ensemble* E, cudaError_t e, const char* where)
{
    std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return efail(E, e == cudaErrorMemoryAllocation ? GKM_ERR_NOMEM : GKM_ERR_CUDA, m);
}

#define ECK(E, expr)                                         \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return ecuda(E, e_, #expr);   \
    } while (0)

int nm_of(const gkm_ensemble* E) { return (int)E->mem.size(); }

const long long* off_ptr(const gkm_ensemble* E, int set) { return E->d_off + (size_t)set * (E->mem.size() + 1); }

void destroy_graphs(gkm_ensemble* E)
{
    for (int k = 0; k < 2; k++)
        for (int p = 0; p < 2; p++) {
            if (E->graph[k][p]) cudaGraphExecDestroy(E->graph[k][p]);
            E->graph[k][p] = nullptr;
        }
}

// Members' device descriptors and work offsets from their current host state;
// uploads both (stream-ordered) and drops the step graphs when the offsets moved.
gkm_status refresh(gkm_ensemble* E, bool need_state)
{
    const int nm = nm_of(E);
    const int parity = E->mem[0]->parity;
    for (int m = 0; m < nm; m++) {
        const gkm_handle* h = E->mem[m];
        if (need_state && !h->state_loaded) return efail(E, GKM_ERR_STATE, "member " + std::to_string(m) + ": no state uploaded");
        if (h->parity != parity)
            return efail(E, GKM_ERR_STATE, "member " + std::to_string(m) + " was stepped outside the ensemble");
    }
    std::vector<MemberDev> hm((size_t)nm);
    std::vector<long long> off((size_t)kNumSets * (nm + 1), 0);
    std::vector<std::vector<long long>> items(3, std::vector<long long>((size_t)nm, 0));
    auto at = [&](int set, int m) -> long long& { return off[(size_t)set * (nm + 1) + m]; };
    for (int m = 0; m < nm; m++) {
        const gkm_handle* h = E->mem[m];
        MemberDev& md = hm[(size_t)m];
        std::memset(&md, 0, sizeof(md));
        md.buf[0] = h->buf[0];
        md.buf[1] = h->buf[1];
        md.clock = h->clock;
        md.fc = h->fc;
        md.dt_fixed_mode = h->dt_fixed_mode;
        md.dt_fixed = h->dt_fixed;
        const long long n = h->fc.n;
        for (int d = 0; d < 3; d++) {
            const gkm::SweepShape sh = gkm::sweep_shape(E->mixed, E->sweep[d].variant);
            int L = E->seg[d][(size_t)m];
            L = L < 1 ? 1 : (L > n ? (int)n : L);
            md.seg_len[d] = L;
            md.nseg[d] = (int)((n + L - 1) / L);
            md.tiles_b[d] = (int)((n + sh.TB - 1) / sh.TB);
            items[(size_t)d][(size_t)m] = (long long)md.tiles_b[d] * ((n + sh.TA - 1) / sh.TA) * md.nseg[d];
        }
        md.grid = h->grid;
        const int N1 = h->grid.npts + 1;
        md.tb = gkm::SplineTables{h->tables, h->tables + N1, h->tables + 2 * N1, h->denom};
        for (int c = 0; c < 3; c++) md.coef[c] = h->coef[c];
        md.scratch[0] = h->scratch;
        md.scratch[1] = h->scratch_extra[0] ? h->scratch_extra[0] : E->extra_scratch[2 * (size_t)m];
        md.scratch[2] = h->scratch_extra[1] ? h->scratch_extra[1] : E->extra_scratch[2 * (size_t)m + 1];
        for (int c = 0; c < 6; c++) md.P[c] = h->P[c];
        md.np = h->np;
        md.tmaps = h->d_tmaps;
        const long long N = h->grid.npts, M = N + h->grid.pad;
        const long long nt = h->fc.nt;
        const bool parts = h->np > 0;   // members without particles skip the spline work
        const long long count[kPart + 1] = {0,
                                            0,
                                            0,
                                            nt * nt * nt - n * n * n,
                                            parts ? 3 * N * N : 0,
                                            parts ? 3 * M * N : 0,
                                            parts ? 3 * ((M * M + 31) / 32) : 0,
                                            h->np};
        for (int s = kGhost; s <= kPart; s++) at(s, m + 1) = at(s, m) + count[s];
    }
    // sweep work lists: members in decreasing segment length (longest items first; a stable order,
    // so equal lengths keep the members' order), offsets by position
    for (int d = 0; d < 3; d++) {
        std::vector<int> ord((size_t)nm);
        for (int m = 0; m < nm; m++) ord[(size_t)m] = m;
        std::stable_sort(ord.begin(), ord.end(),
                         [&](int x, int y) { return hm[(size_t)x].seg_len[d] > hm[(size_t)y].seg_len[d]; });
        for (int p = 0; p < nm; p++) {
            at(kOrderX + d, p) = ord[(size_t)p];
            at(kItemX + d, p + 1) = at(kItemX + d, p) + items[(size_t)d][(size_t)ord[(size_t)p]];
        }
    }
    ECK(E, cudaMemcpyAsync(E->d_mem, hm.data(), sizeof(MemberDev) * (size_t)nm, cudaMemcpyHostToDevice, E->stream));
    if (off != E->h_off) {
        ECK(E, cudaMemcpyAsync(E->d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice, E->stream));
        E->h_off = off;
        for (int s = 0; s < kNumSets; s++) E->total[s] = at(s, nm);
        destroy_graphs(E);
    }
    // pageable sources: the copies above have been staged when they return
    return GKM_OK;
}

cudaError_t launch_sweep_dir(gkm_ensemble* E, int d, int parity)
{
    const SweepChoice& c = E->sweep[d];
    E->launches += 1;
    if (E->mixed)
        return gkm::launch_ensemble_sweep32(d, c.variant, E->d_mem, off_ptr(E, kItemX + d), off_ptr(E, kOrderX + d),
                                            nm_of(E), parity, E->d_next + d, E->stream);
    return gkm::launch_ensemble_sweep64(d, c.variant, E->d_mem, off_ptr(E, kItemX + d), off_ptr(E, kOrderX + d),
                                        nm_of(E), parity, E->d_next + d, E->stream);
}

cudaError_t launch_halo_all(gkm_ensemble* E, int parity)
{
    E->launches += 1;
    return gkm::launch_ensemble_halo(E->d_mem, off_ptr(E, kGhost), nm_of(E), E->total[kGhost], parity ^ 1, 1,
                                     E->stream);
}

cudaError_t launch_splines_all(gkm_ensemble* E, int parity)
{
    if (E->total[kLine0] == 0) return cudaSuccess;
    gkm::EnsembleWork w{};
    for (int d = 0; d < 3; d++) w.item[d] = off_ptr(E, kItemX + d);
    w.ghost = off_ptr(E, kGhost);
    w.line0 = off_ptr(E, kLine0);
    w.line1 = off_ptr(E, kLine1);
    w.warp2 = off_ptr(E, kWarp2);
    w.part = off_ptr(E, kPart);
    const long long totals[3] = {E->total[kLine0], E->total[kLine1], E->total[kWarp2]};
    E->launches += 3;
    return gkm::launch_ensemble_splines(E->d_mem, w, totals, nm_of(E), parity ^ 1, E->stream);
}

cudaError_t launch_particles_all(gkm_ensemble* E)
{
    if (E->total[kPart] == 0) return cudaSuccess;
    E->launches += 1;
    return gkm::launch_ensemble_heun(E->d_mem, off_ptr(E, kPart), nm_of(E), E->total[kPart], E->stream);
}

// one full step of every member from buffer `parity`
cudaError_t enqueue_step(gkm_ensemble* E, int parity, bool parts)
{
    for (int d = 0; d < 3; d++) {
        cudaError_t e = launch_sweep_dir(E, d, parity);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = launch_halo_all(E, parity);
    if (e != cudaSuccess || !parts) return e;
    e = launch_splines_all(E, parity);
    if (e != cudaSuccess) return e;
    return launch_particles_all(E);
}

void finish_step(gkm_ensemble* E, bool parts)
{
    for (gkm_handle* h : E->mem) {
        h->parity ^= 1;
        h->splines_valid = parts && h->np > 0;
    }
}

}  // namespace

extern "C" {

gkm_status gkm_ensemble_create(const gkm_config* members, int32_t n_members, gkm_ensemble** out)
{
    if (!members || !out || n_members < 1 || n_members > 65536) return GKM_ERR_ARG;
    *out = nullptr;
    for (int m = 1; m < n_members; m++)
        if (members[m].device != members[0].device || members[m].precision != members[0].precision)
            return GKM_ERR_CONFIG;
    for (int m = 0; m < n_members; m++)   // the ensemble's spline kernels store FP64 coefficients
        if (members[m].spline_precision != GKM_SPLINE_COEF_FP64) return GKM_ERR_CONFIG;
    gkm_ensemble* E = new gkm_ensemble();
    E->mixed = members[0].precision == GKM_PREC_MIXED;
    E->device = members[0].device;
    auto bail = [&](gkm_status s) {
        std::fprintf(stderr, "gkm_ensemble_create: %s\n", E->err.c_str());
        gkm_ensemble_destroy(E);
        return s;
    };
    cudaError_t e = cudaSetDevice(E->device);
    if (e != cudaSuccess) return bail(ecuda(E, e, "cudaSetDevice"));
    e = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(ecuda(E, e, "cudaStreamCreate"));
    int max_n = 0;
    for (int m = 0; m < n_members; m++) {
        gkm_handle* h = nullptr;
        gkm_status s = gkm_create(&members[m], &h);
        if (s != GKM_OK) return bail(efail(E, s, "member " + std::to_string(m) + ": gkm_create failed"));
        h->stream = E->stream;
        h->owner = E;
        E->mem.push_back(h);
        const long long M = h->grid.npts + h->grid.pad, N = h->grid.npts;
        for (int k = 0; k < 2; k++) {
            double* p = nullptr;   // the member's own second and third scratch when it has them
            if (!h->scratch_extra[k]) {
                e = cudaMalloc(&p, sizeof(double) * (size_t)(M * M * N));
                if (e != cudaSuccess) return bail(ecuda(E, e, "cudaMalloc(spline scratch)"));
            }
            E->extra_scratch.push_back(p);
        }
        if (h->fc.n > max_n) max_n = h->fc.n;
    }
    for (int d = 0; d < 3; d++) {
        E->sweep[d].variant = 0;
        E->sweep[d].seg_len = max_n < 16 ? max_n : 16;
        E->seg[d].assign((size_t)n_members, E->sweep[d].seg_len);
    }
    e = cudaMalloc(&E->d_next, 3 * sizeof(unsigned long long));
    if (e != cudaSuccess) return bail(ecuda(E, e, "cudaMalloc(work counters)"));
    e = cudaMalloc(&E->d_mem, sizeof(MemberDev) * (size_t)n_members);
    if (e != cudaSuccess) return bail(ecuda(E, e, "cudaMalloc(members)"));
    e = cudaMalloc(&E->d_off, sizeof(long long) * (size_t)kNumSets * (n_members + 1));
    if (e != cudaSuccess) return bail(ecuda(E, e, "cudaMalloc(offsets)"));
    *out = E;
    return GKM_OK;
}

gkm_status gkm_ensemble_destroy(gkm_ensemble* E)
{
    if (!E) return GKM_ERR_ARG;
    if (E->stream) cudaStreamSynchronize(E->stream);
    destroy_graphs(E);
    for (gkm_handle* h : E->mem) {
        h->owner = nullptr;
        h->stream = h->own_stream;
        gkm_destroy(h);
    }
    for (double* p : E->extra_scratch) cudaFree(p);
    cudaFree(E->d_mem);
    cudaFree(E->d_off);
    cudaFree(E->d_next);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
    return GKM_OK;
}

const char* gkm_ensemble_last_error(const gkm_ensemble* E) { return E ? E->err.c_str() : "null ensemble"; }

int32_t gkm_ensemble_size(const gkm_ensemble* E) { return E ? (int32_t)E->mem.size() : 0; }

gkm_handle* gkm_ensemble_member(gkm_ensemble* E, int32_t m)
{
    if (!E || m < 0 || m >= (int32_t)E->mem.size()) return nullptr;
    return E->mem[(size_t)m];
}

gkm_status gkm_ensemble_step(gkm_ensemble* E, int32_t nsteps, int32_t with_particles)
{
    if (!E || nsteps < 0) return GKM_ERR_ARG;
    ECK(E, cudaSetDevice(E->device));
    gkm_status s = refresh(E, true);
    if (s != GKM_OK) return s;
    const int k = with_particles ? 1 : 0;
    for (int it = 0; it < nsteps; it++) {
        const int p = E->mem[0]->parity;
        if (!E->graph[k][p]) {
            cudaGraph_t g = nullptr;
            const int64_t before = E->launches;
            ECK(E, cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = enqueue_step(E, p, k != 0);
            cudaError_t e2 = cudaStreamEndCapture(E->stream, &g);
            E->graph_kernels[k][p] = E->launches - before;
            E->launches = before;
            if (e != cudaSuccess) return ecuda(E, e, "capture ensemble step");
            if (e2 != cudaSuccess) return ecuda(E, e2, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&E->graph[k][p], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return ecuda(E, e, "cudaGraphInstantiate");
        }
        ECK(E, cudaGraphLaunch(E->graph[k][p], E->stream));
        E->launches += E->graph_kernels[k][p];
        finish_step(E, k != 0);
    }
    return GKM_OK;
}

gkm_status gkm_ensemble_step_timed(gkm_ensemble* E, int32_t nsteps, int32_t with_particles, double ms[7])
{
    if (!E || !ms || nsteps < 0) return GKM_ERR_ARG;
    ECK(E, cudaSetDevice(E->device));
    gkm_status s = refresh(E, true);
    if (s != GKM_OK) return s;
    for (int k = 0; k < 7; k++) ms[k] = 0.0;
    cudaEvent_t ev[7];
    for (int k = 0; k < 7; k++) ECK(E, cudaEventCreate(&ev[k]));
    gkm_status st = GKM_OK;
    for (int it = 0; it < nsteps; it++) {
        const int p = E->mem[0]->parity;
        cudaError_t e = cudaEventRecord(ev[0], E->stream);
        for (int d = 0; d < 3 && e == cudaSuccess; d++) {
            e = launch_sweep_dir(E, d, p);
            if (e == cudaSuccess) e = cudaEventRecord(ev[d + 1], E->stream);
        }
        if (e == cudaSuccess) e = launch_halo_all(E, p);
        if (e == cudaSuccess) e = cudaEventRecord(ev[4], E->stream);
        if (e == cudaSuccess && with_particles) e = launch_splines_all(E, p);
        if (e == cudaSuccess) e = cudaEventRecord(ev[5], E->stream);
        if (e == cudaSuccess && with_particles) e = launch_particles_all(E);
        if (e == cudaSuccess) e = cudaEventRecord(ev[6], E->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[6]);
        if (e != cudaSuccess) {
            st = ecuda(E, e, "gkm_ensemble_step_timed");
            break;
        }
        float t;
        for (int k = 0; k < 6; k++) {
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            ms[k] += t;
        }
        cudaEventElapsedTime(&t, ev[0], ev[6]);
        ms[6] += t;
        finish_step(E, with_particles != 0);
    }
    for (int k = 0; k < 7; k++) cudaEventDestroy(ev[k]);
    return st;
}

gkm_status gkm_ensemble_autotune(gkm_ensemble* E, int32_t reps)
{
    if (!E || reps < 1) return GKM_ERR_ARG;
    ECK(E, cudaSetDevice(E->device));
    gkm_status s = refresh(E, true);
    if (s != GKM_OK) return s;
    const int nm = nm_of(E);
    // the sweeps write only the accumulators; the clocks they touch are restored
    std::vector<DevClock> saved((size_t)nm);
    for (int m = 0; m < nm; m++)
        ECK(E, cudaMemcpyAsync(&saved[(size_t)m], E->mem[m]->clock, sizeof(DevClock), cudaMemcpyDeviceToHost,
                               E->stream));
    ECK(E, cudaStreamSynchronize(E->stream));
    // grid sizes of the members, largest first, and the candidate segment lengths
    std::vector<int> sizes;
    for (const gkm_handle* h : E->mem)
        if (std::find(sizes.begin(), sizes.end(), h->fc.n) == sizes.end()) sizes.push_back(h->fc.n);
    std::sort(sizes.begin(), sizes.end(), std::greater<int>());
    auto lens_upto = [](int n) {
        std::vector<int> v;
        for (int L : {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256})
            if (L < n) v.push_back(L);
        v.push_back(n);
        return v;
    };
    const std::vector<int> lens = lens_upto(sizes[0]);
    // the persistent kernel has the plain window variants only (variant 2 is single-cube)
    // FP64: 16 x 8, 16 x 16, and the warp-specialized 16 x 16 form where its kernels are usable
    const int nvar = E->mixed ? gkm::kSweepVariants32 : (gkm::ensemble_ws_ready() ? 3 : 2);
    const int p = E->mem[0]->parity;
    cudaEvent_t e0, e1;
    ECK(E, cudaEventCreate(&e0));
    ECK(E, cudaEventCreate(&e1));
    gkm_status st = GKM_OK;
    const int64_t launches0 = E->launches;
    // time of `reps` launches of direction d with the current shapes (one untimed launch first)
    auto time_dir = [&](int d, float* ms) -> gkm_status {
        gkm_status r = refresh(E, true);
        if (r != GKM_OK) return r;
        cudaError_t e = launch_sweep_dir(E, d, p);
        if (e == cudaSuccess) e = cudaEventRecord(e0, E->stream);
        for (int k = 0; k < reps && e == cudaSuccess; k++) e = launch_sweep_dir(E, d, p);
        if (e == cudaSuccess) e = cudaEventRecord(e1, E->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
        return e == cudaSuccess ? GKM_OK : ecuda(E, e, "gkm_ensemble_autotune");
    };
    for (int d = 0; d < 3 && st == GKM_OK; d++) {
        // 1. the window variant, with one segment length for every member
        int best_v = E->sweep[d].variant, best_L = E->sweep[d].seg_len;
        float best_ms = 1e30f;
        for (int v = 0; v < nvar && st == GKM_OK; v++)
            for (int L : lens) {
                E->sweep[d].variant = v;
                E->seg[d].assign((size_t)nm, L);
                float t = 0.f;
                st = time_dir(d, &t);
                if (st != GKM_OK) break;
                if (t < best_ms) {
                    best_ms = t;
                    best_v = v;
                    best_L = L;
                }
            }
        E->sweep[d].variant = best_v;
        E->sweep[d].seg_len = best_L;
        E->seg[d].assign((size_t)nm, best_L);
        // 2. one segment length per grid size, largest grids first, the other sizes held
        for (int n : sizes) {
            if (st != GKM_OK) break;
            std::vector<int> keep = E->seg[d];
            int best_n = -1;
            for (int L : lens_upto(n)) {
                for (int m = 0; m < nm; m++)
                    if (E->mem[m]->fc.n == n) E->seg[d][(size_t)m] = L;
                float t = 0.f;
                st = time_dir(d, &t);
                if (st != GKM_OK) break;
                if (t < best_ms) {
                    best_ms = t;
                    best_n = L;
                }
            }
            E->seg[d] = keep;
            if (best_n > 0)
                for (int m = 0; m < nm; m++)
                    if (E->mem[m]->fc.n == n) E->seg[d][(size_t)m] = best_n;
        }
    }
    E->launches = launches0;   // tuning launches are not steps
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int m = 0; m < nm; m++)
        cudaMemcpyAsync(E->mem[m]->clock, &saved[(size_t)m], sizeof(DevClock), cudaMemcpyHostToDevice, E->stream);
    cudaStreamSynchronize(E->stream);
    if (st != GKM_OK) return st;
    destroy_graphs(E);   // a variant of the same windows leaves the work offsets, and so the graphs, unchanged
    return refresh(E, true);
}

gkm_status gkm_ensemble_segments(const gkm_ensemble* E, int32_t* out, int64_t capacity)
{
    if (!E || !out) return GKM_ERR_ARG;
    const int nm = nm_of(E);
    if (capacity < 3LL * nm) return GKM_ERR_ARG;
    for (int d = 0; d < 3; d++)
        for (int m = 0; m < nm; m++) {
            const int n = E->mem[m]->fc.n, L = E->seg[d][(size_t)m];
            out[(size_t)d * nm + m] = L > n ? n : L;
        }
    return GKM_OK;
}

gkm_status gkm_ensemble_set_sweep_config(gkm_ensemble* E, const int32_t in[6])
{
    if (!E || !in) return GKM_ERR_ARG;
    const int nm = nm_of(E);
    const int nvar = E->mixed ? gkm::kSweepVariants32 : (gkm::ensemble_ws_ready() ? 3 : 2);
    for (int d = 0; d < 3; d++) {
        const int v = in[2 * d], L = in[2 * d + 1];
        if (L < 1) return efail(E, GKM_ERR_ARG, "segment length below 1");
        if (v < 0 || v >= nvar) return efail(E, GKM_ERR_CONFIG, "sweep variant not available for this ensemble");
    }
    for (int d = 0; d < 3; d++) {
        E->sweep[d].variant = in[2 * d];
        E->sweep[d].seg_len = in[2 * d + 1];
        E->seg[d].assign((size_t)nm, in[2 * d + 1]);
    }
    destroy_graphs(E);   // the captured steps launched the previous kernels
    return refresh(E, false);
}

gkm_status gkm_ensemble_sweep_config(const gkm_ensemble* E, int32_t out[12])
{
    if (!E || !out) return GKM_ERR_ARG;
    for (int d = 0; d < 3; d++) {
        const gkm::SweepShape sh = gkm::sweep_shape(E->mixed, E->sweep[d].variant);
        out[4 * d + 0] = E->sweep[d].variant;
        out[4 * d + 1] = sh.TB;
        out[4 * d + 2] = sh.TA;
        out[4 * d + 3] = E->sweep[d].seg_len;   // the length shared before per-size tuning

    }
    return GKM_OK;
}

gkm_status gkm_ensemble_launch_count(const gkm_ensemble* E, int64_t* count)
{
    if (!E || !count) return GKM_ERR_ARG;
    *count = E->launches;
    return GKM_OK;
}

gkm_status gkm_ensemble_synchronize(gkm_ensemble* E)
{
    if (!E) return GKM_ERR_ARG;
    ECK(E, cudaStreamSynchronize(E->stream));
    return GKM_OK;
}

gkm_status gkm_ensemble_stream(const gkm_ensemble* E, void** stream)
{
    if (!E || !stream) return GKM_ERR_ARG;
    *stream = (void*)E->stream;
    return GKM_OK;
}

}  // extern "C"
