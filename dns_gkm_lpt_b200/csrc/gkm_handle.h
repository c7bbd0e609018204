// Host-side state of one handle, shared by the single-cube C ABI
// (gkm_capi.cu) and the ensemble C ABI (gkm_ensemble.cu).  Not installed.
#pragma once

#include "gkm.h"
#include "gkm_internal.h"

#include <string>
#include <vector>

struct gkm_ensemble;

struct SweepChoice {
    int variant = 0;   // window variant (gkm::sweep_shape)
    int nseg = 1;      // CTAs along the sweep normal
    int seg_len = 1;   // faces per CTA along the normal
};

struct gkm_handle {
    gkm_config cfg{};
    gkm::FieldConst fc{};
    SweepChoice sweep[3];
    cudaStream_t own_stream = nullptr, stream = nullptr;
    double* buf[2] = {nullptr, nullptr};
    int parity = 0;
    gkm::DevClock* clock = nullptr;
    bool state_loaded = false;
    int dt_fixed_mode = 0;
    double dt_fixed = 0.0;
    gkm::SplineGrid grid{};
    double* tables = nullptr;  // mt | dp | z, each npts+1
    double denom = 0.0;
    double* coef[3] = {nullptr, nullptr, nullptr};
    float* coef32[3] = {nullptr, nullptr, nullptr};   // GKM_SPLINE_COEF_FP32: the coefficients, rounded
    bool spline_f32 = false;
    double* scratch = nullptr;
    // the three velocity splines built together (one launch per pass for all three components):
    // two more scratch arrays and a one-member descriptor for the ensemble spline kernels;
    // left out when the device lacks the memory (large grids), then one component at a time
    double* scratch_extra[2] = {nullptr, nullptr};
    gkm::MemberDev* d_self = nullptr;
    long long* d_self_off = nullptr;   // line0 | line1 | warp2 prefix offsets, 2 each
    long long self_totals[3] = {0, 0, 0};
    bool splines_valid = false;
    int64_t np = 0, cap = 0;
    double* P[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // y, x, z, u, v, w
    // particle ordering: the sorted copy, upload indices (tags) of both, keys and bucket counts
    double* P_sorted[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    long long* tag = nullptr;          // upload index of the particle in each slot of P
    long long* tag_sorted = nullptr;
    unsigned* sort_keys = nullptr;
    unsigned* sort_counts = nullptr;
    unsigned* sort_temp = nullptr;
    double* prop_coef[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};   // rho, p, lap u, lap v, lap w
    double* lap_nodes = nullptr;     // nt^3 Laplacian node values (one velocity component at a time)
    double* props = nullptr;         // [kPropCount][cap] particle properties
    gkm::StatsPartial* partials = nullptr;
    double* stats_out = nullptr;
    cudaGraphExec_t graph[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
    int64_t graph_np[3][2] = {{-1, -1}, {-1, -1}, {-1, -1}};
    int64_t graph_kernels[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    int64_t launches = 0;    // kernels launched (graph replays add the kernels they hold)
    // plug-point pipeline (gkm_evolve with pinned or device buffers): copy-in, copy-out and
    // two compute streams, and per-chunk events, created on first use
    cudaStream_t pipe_in = nullptr, pipe_out = nullptr, pipe_comp[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t pipe_halo = nullptr;   // ghost wrap of each part as it lands, off the copy-in stream
    std::vector<cudaEvent_t> pipe_ev;
    int pipe_chunk = 0;      // y-planes per chunk (multiple of 16); 0: about n/8
    // tensor maps of the two state buffers for the FP64 x / y sweeps' slab copies, in device
    // memory, index (buffer * kSweepVariants64 + variant) * 2 + direction; null when unavailable
    unsigned char* d_tmaps = nullptr;
    int pipe_streams = 2;    // compute streams
    std::string err;
    gkm_ensemble* owner = nullptr;   // set while the handle is a member of an ensemble
};

// particle property table on the host, particle-major np x kPropCount (gkm_capi.cu)
gkm_status gkm_host_props(gkm_handle* h, double* out);

namespace gkm_host {

inline gkm_status fail(gkm_handle* h, gkm_status s, const std::string& msg)
{
    if (h) h->err = msg;
    return s;
}

inline gkm_status cuda_fail(gkm_handle* h, cudaError_t e, const char* where)
{
    std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(h, e == cudaErrorMemoryAllocation ? GKM_ERR_NOMEM : GKM_ERR_CUDA, m);
}

#define CK(h, expr)                                         \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #expr); \
    } while (0)

}  // namespace gkm_host
