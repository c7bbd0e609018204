// Eulerian step on sm_100a: fused WENO reconstruction + gas-kinetic flux +
// conservative update, one sweep kernel per direction, plus the periodic halo
// wrap and the max(|u|+c) reduction that sets the next dt.
//
// Reference path replaced: evolveEulerian -> derivsX/Y/Z -> flux -> update
// (src/update.cpp:206-516), HaloTransfer (:855-1029), timestep (:1031-1054).
//
// Layout: the reference's own arrays, 5 components of nt^3 doubles (nt = n+6,
// index (j*nt + i)*nt + k, z fastest), ghosts refreshed on the device after
// every step, so every stencil read is in bounds and host<->device copies are
// plain memcpys of the reference's W[5].
//
// Per step: x sweep writes A = Fx(i) - Fx(i-1); y sweep A = (A + Fy(j)) - Fy(j-1);
// z sweep W' = W - (1/dx) ((A + Fz(k)) - Fz(k-1)) into A; the halo kernel
// wraps A's ghosts and the caller swaps W and A.  The additions run in the
// reference's left-to-right order with rounding-explicit intrinsics.
#include "sweep_impl.cuh"
#include "sweep_ws.cuh"

namespace gkm {
namespace {

using sweep_detail::block_max;
using sweep_detail::wave_speed;

__global__ void halo_kernel(double* __restrict__ W, FieldConst fc, DevClock* clock, int finish_step, int slot,
                            int dt_fixed_mode, double dt_fixed)
{
    const long long total = fc.nt3 - (long long)fc.n * fc.n * fc.n;
    if (finish_step && blockIdx.x == 0 && threadIdx.x == 0) {
        // src/update.cpp:167-169: timestep(W) of the new state, then t += dt
        clock->t += cfl_dt(fc, clock, slot, dt_fixed_mode, dt_fixed);
        clock->iter += 1;
    }
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x)
        halo_cell(W, fc, g);
}

// ghost cells of the y-planes [J0, J1): every cell with a coordinate outside the interior takes the
// value of its periodic image, which is interior in all three coordinates
__global__ void halo_planes_kernel(double* __restrict__ W, FieldConst fc, int J0, int J1)
{
    const int n = fc.n, nt = fc.nt;
    const long long nt2 = (long long)nt * nt, nt3 = fc.nt3;
    const long long total = (long long)(J1 - J0) * nt2;
    auto wrap = [n](int x) { return x < 3 ? x + n : (x >= n + 3 ? x - n : x); };
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int j = J0 + (int)(e / nt2);
        const long long rem = e - (long long)(j - J0) * nt2;
        const int i = (int)(rem / nt), k = (int)(rem - (long long)i * nt);
        const int wj = wrap(j), wi = wrap(i), wk = wrap(k);
        if (wj == j && wi == i && wk == k) continue;   // interior cell
        const long long dst = ((long long)j * nt + i) * nt + k;
        const long long src = ((long long)wj * nt + wi) * nt + wk;
#pragma unroll
        for (int q = 0; q < 5; q++) W[q * nt3 + dst] = W[q * nt3 + src];
    }
}

__global__ void clock_finish_kernel(DevClock* clock, double dt)
{
    clock->t += dt;   // src/update.cpp:167-168 with the next step's dt (the given one)
    clock->iter += 1;
}

__global__ void wave_reduce_kernel(const double* __restrict__ W, FieldConst fc, DevClock* clock, int slot)
{
    __shared__ double red[32];
    const int n = fc.n, nt = fc.nt;
    const long long nt3 = fc.nt3, total = (long long)n * n * n;
    double m = 0.0;
    bool bad = false;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(g / ((long long)n * n)), i = (int)((g / n) % n), k = (int)(g % n);
        const long long idx = ((long long)(j + 3) * nt + (i + 3)) * nt + (k + 3);
        double w[5];
#pragma unroll
        for (int q = 0; q < 5; q++) w[q] = W[q * nt3 + idx];
        double ws = wave_speed(w, fc.gam, fc.gm1);
        if (!isfinite(ws) || !(w[0] > 0.0)) bad = true;
        else m = ws > m ? ws : m;
    }
    m = block_max(m, red);
    if (threadIdx.x == 0 && m > 0.0) atomicMax(&clock->wave[slot], (unsigned long long)__double_as_longlong(m));
    if (bad) atomicOr(&clock->status, 1);
}

// Single-face entry with the same math as the sweep: per face 51 inputs
// WL[5] WR[5] Wl[5] Wr[5] DWxl DWxr DWyl DWyr DWzl DWzr [6x5] tau0.
__global__ void flux_faces_kernel(const double* __restrict__ in, long long nf, Phys<double> ph, double dt, double dx,
                                  double* __restrict__ F)
{
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const double* p = in + f * 51;
    FaceInput<double> fi;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        fi.WL_[q] = p[q];
        fi.WR_[q] = p[5 + q];
        fi.Wl_[q] = p[10 + q];
        fi.Wr_[q] = p[15 + q];
    }
#pragma unroll
    for (int v = 0; v < 6; v++)
#pragma unroll
        for (int q = 0; q < 5; q++) fi.DW_[v][q] = p[20 + 5 * v + q];
    double out[5];
    gks_flux<double>(fi, p[50], dt, dx, ph, out);
#pragma unroll
    for (int q = 0; q < 5; q++) F[f * 5 + q] = out[q];
}

__global__ void weno_faces_kernel(const double* __restrict__ s, long long n, Phys<double> ph, double* __restrict__ Wl,
                                  double* __restrict__ Wr)
{
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= n) return;
    const double* p = s + f * 30;   // 6 cells x 5 components
    double l[5], r[5], T[6];
#pragma unroll
    for (int o = 0; o < 6; o++) T[o] = temperature<double>(p[5 * o], p[5 * o + 1], p[5 * o + 2], p[5 * o + 3], p[5 * o + 4], ph);
#pragma unroll
    for (int q = 0; q < 4; q++)
        weno_scalar<double>(p[q], p[5 + q], p[10 + q], p[15 + q], p[20 + q], p[25 + q], kWenoEps, l[q], r[q]);
    double Tl, Tr;
    weno_scalar<double>(T[0], T[1], T[2], T[3], T[4], T[5], kWenoEps, Tl, Tr);
    l[4] = face_energy<double>(l[0], l[1], l[2], l[3], Tl, ph);
    r[4] = face_energy<double>(r[0], r[1], r[2], r[3], Tr, ph);
#pragma unroll
    for (int q = 0; q < 5; q++) {
        Wl[f * 5 + q] = l[q];
        Wr[f * 5 + q] = r[q];
    }
}

// the warp-specialized sweep may run only where its kernels were compiled to the register count
// its warpgroups' setmaxnreg split draws on (a smaller launch count would leave them waiting)
bool g_ws_ready = false;

template <int DIR, int MM>
cudaError_t ws_check(bool& ok)
{
    cudaFuncAttributes at;
    cudaError_t e = cudaFuncGetAttributes(&at, sweep_ws_kernel<DIR, SweepTile64b, MM>);
    if (e != cudaSuccess) return e;
    ok = ok && at.numRegs == 168;
    return cudaFuncSetAttribute(sweep_ws_kernel<DIR, SweepTile64b, MM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sweep_ws_detail::ws_smem_bytes<SweepTile64b>());
}

// the persistent ensemble form (x, y): the same register count check, its own shared-memory limit
template <int DIR>
cudaError_t ens_ws_check(bool& ok)
{
    cudaFuncAttributes at;
    cudaError_t e = cudaFuncGetAttributes(&at, ensemble_ws_kernel<DIR, SweepTile64b>);
    if (e != cudaSuccess) return e;
    ok = ok && at.numRegs == 168;
    return cudaFuncSetAttribute(ensemble_ws_kernel<DIR, SweepTile64b>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sweep_ws_detail::ws_smem_bytes<SweepTile64b>());
}
bool g_ens_ws_ready = false;

// x, y: the form with tensor copies when the launch carries a map; z: per-element copies
template <int DIR>
cudaError_t launch_ws(SweepArgs a, dim3 grid, cudaStream_t s)
{
    constexpr unsigned th = sweep_ws_detail::kThreads;
    const size_t smem = sweep_ws_detail::ws_smem_bytes<SweepTile64b>();
    if constexpr (DIR != 2) {
        if (a.tmap != nullptr) {
            sweep_ws_kernel<DIR, SweepTile64b, kMapsOn><<<grid, th, smem, s>>>(a);
            return cudaGetLastError();
        }
    }
    sweep_ws_kernel<DIR, SweepTile64b, kMapsOff><<<grid, th, smem, s>>>(a);
    return cudaGetLastError();
}

template <int DIR, class Tile>
cudaError_t launch_one(const SweepArgs& a, int nseg, cudaStream_t s)
{
    dim3 grid((a.fc.n + Tile::TB - 1) / Tile::TB, (a.fc.n + Tile::TA - 1) / Tile::TA, nseg);
    dim3 block(Tile::TB, Tile::TA);
    launch_form<DIR, double, Tile>(a, grid, block, s);
    return cudaGetLastError();
}

template <class Tile>
cudaError_t set_smem()
{
    cudaError_t e = set_form_smem<0, double, Tile>();
    if (e == cudaSuccess) e = set_form_smem<1, double, Tile>();
    if (e == cudaSuccess) e = set_form_smem<2, double, Tile>();
    return e;
}

}  // namespace

namespace {

// ensemble halo: every member's ghost cells as one flattened index space
__global__ void ensemble_halo_kernel(const MemberDev* __restrict__ mem, const long long* __restrict__ off, int nm,
                                     int buf, int finish_step)
{
    const long long total = off[nm];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int m = find_member(off, nm, g);
        const MemberDev& md = mem[m];
        const long long local = g - off[m];
        if (finish_step && local == 0) {
            md.clock->t += cfl_dt(md.fc, md.clock, buf, md.dt_fixed_mode, md.dt_fixed);   // src/update.cpp:167-169
            md.clock->iter += 1;
        }
        halo_cell(md.buf[buf], md.fc, local);
    }
}

}  // namespace

cudaError_t sweep_prepare()
{
    cudaError_t e = set_smem<SweepTile64a>();
    if (e == cudaSuccess) e = set_smem<SweepTile64b>();
    if (e == cudaSuccess) e = set_ensemble_smem<double, SweepTile64a>();
    if (e == cudaSuccess) e = set_ensemble_smem<double, SweepTile64b>();
    bool ok = true;
    if (e == cudaSuccess) e = ws_check<0, kMapsOn>(ok);
    if (e == cudaSuccess) e = ws_check<0, kMapsOff>(ok);
    if (e == cudaSuccess) e = ws_check<1, kMapsOn>(ok);
    if (e == cudaSuccess) e = ws_check<1, kMapsOff>(ok);
    if (e == cudaSuccess) e = ws_check<2, kMapsOff>(ok);
    g_ws_ready = e == cudaSuccess && ok;
    bool ens_ok = g_ws_ready;
    if (e == cudaSuccess) e = ens_ws_check<0>(ens_ok);
    if (e == cudaSuccess) e = ens_ws_check<1>(ens_ok);
    g_ens_ws_ready = e == cudaSuccess && ens_ok;
    return e;
}

bool ws_ready() { return g_ws_ready; }
bool ensemble_ws_ready() { return g_ens_ws_ready; }

cudaError_t launch_ensemble_sweep64(int dir, int variant, const MemberDev* mem, const long long* off,
                                    const long long* order, int nm, int parity, unsigned long long* next,
                                    cudaStream_t s)
{
    // variant 2: the persistent warp-specialized form for x and y (one CTA per SM); the z sweep, or a
    // build whose kernels missed the register count, runs it as variant 1
    if (variant == 2 && dir < 2 && g_ens_ws_ready) {
        cudaError_t e = cudaMemsetAsync(next, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
        const size_t smem = sweep_ws_detail::ws_smem_bytes<SweepTile64b>();
        if (dir == 0)
            ensemble_ws_kernel<0, SweepTile64b><<<148, sweep_ws_detail::kThreads, smem, s>>>(mem, off, order, nm, parity, next);
        else
            ensemble_ws_kernel<1, SweepTile64b><<<148, sweep_ws_detail::kThreads, smem, s>>>(mem, off, order, nm, parity, next);
        return cudaGetLastError();
    }
    if (variant >= 1)
        return launch_ensemble_sweep_t<double, SweepTile64b>(dir, mem, off, order, nm, parity, next, s);
    return launch_ensemble_sweep_t<double, SweepTile64a>(dir, mem, off, order, nm, parity, next, s);
}

cudaError_t launch_ensemble_halo(const MemberDev* mem, const long long* off, int nm, long long total, int buf,
                                 int finish_step, cudaStream_t s)
{
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    ensemble_halo_kernel<<<blocks, 256, 0, s>>>(mem, off, nm, buf, finish_step);
    return cudaGetLastError();
}

SweepShape sweep_shape(bool mixed, int variant)
{
    if (mixed) return {0, SweepTile32a::TB, SweepTile32a::TA, SweepTile32a::ctas};
    if (variant == 2) return {2, SweepTile64b::TB, SweepTile64b::TA, 1};
    if (variant == 1) return {1, SweepTile64b::TB, SweepTile64b::TA, SweepTile64b::ctas};
    return {0, SweepTile64a::TB, SweepTile64a::TA, SweepTile64a::ctas};
}

cudaError_t launch_sweep(int dir, int variant, const SweepArgs& a, int nseg, cudaStream_t s)
{
    if (variant == 2 && g_ws_ready) {
        const dim3 grid((a.fc.n + 15) / 16, (a.fc.n + 15) / 16, nseg);
        if (dir == 0) return launch_ws<0>(a, grid, s);
        if (dir == 1) return launch_ws<1>(a, grid, s);
        return launch_ws<2>(a, grid, s);
    }
    if (variant >= 1) {
        if (dir == 0) return launch_one<0, SweepTile64b>(a, nseg, s);
        if (dir == 1) return launch_one<1, SweepTile64b>(a, nseg, s);
        return launch_one<2, SweepTile64b>(a, nseg, s);
    }
    if (dir == 0) return launch_one<0, SweepTile64a>(a, nseg, s);
    if (dir == 1) return launch_one<1, SweepTile64a>(a, nseg, s);
    return launch_one<2, SweepTile64a>(a, nseg, s);
}

cudaError_t launch_sweep_rows(int dir, int variant, SweepArgs a, int j0, int j1, cudaStream_t s)
{
    // the pipelined plug point runs the plain kernels (variant 2 as variant 1)
    if (variant >= 1) return launch_sweep_rows_t<double, SweepTile64b>(dir, a, j0, j1, s);
    return launch_sweep_rows_t<double, SweepTile64a>(dir, a, j0, j1, s);
}

cudaError_t launch_halo_planes(double* W, const FieldConst& fc, int J0, int J1, cudaStream_t s)
{
    if (J0 < 0 || J1 > fc.nt || J0 >= J1) return cudaErrorInvalidValue;
    const long long total = (long long)(J1 - J0) * fc.nt * fc.nt;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    halo_planes_kernel<<<(unsigned)blocks, 256, 0, s>>>(W, fc, J0, J1);
    return cudaGetLastError();
}

cudaError_t launch_clock_finish(DevClock* clock, double dt, cudaStream_t s)
{
    clock_finish_kernel<<<1, 1, 0, s>>>(clock, dt);
    return cudaGetLastError();
}

cudaError_t launch_halo(double* W, const FieldConst& fc, DevClock* clock, int finish_step, int slot,
                        int dt_fixed_mode, double dt_fixed, cudaStream_t s)
{
    long long total = (long long)fc.nt * fc.nt * fc.nt - (long long)fc.n * fc.n * fc.n;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    halo_kernel<<<blocks, 256, 0, s>>>(W, fc, clock, finish_step, slot, dt_fixed_mode, dt_fixed);
    return cudaGetLastError();
}

cudaError_t launch_wave_reduce(const double* W, const FieldConst& fc, DevClock* clock, int slot, cudaStream_t s)
{
    long long total = (long long)fc.n * fc.n * fc.n;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    wave_reduce_kernel<<<blocks, 256, 0, s>>>(W, fc, clock, slot);
    return cudaGetLastError();
}

cudaError_t launch_flux_faces(const double* in, long long nfaces, double gam, int K, double dt, double dx, double* F,
                              cudaStream_t s)
{
    if (nfaces <= 0) return cudaSuccess;
    Phys<double> ph{gam, gam - 1.0, kR, K};
    flux_faces_kernel<<<(unsigned)((nfaces + 63) / 64), 64, 0, s>>>(in, nfaces, ph, dt, dx, F);
    return cudaGetLastError();
}

cudaError_t launch_weno_faces(const double* stencils, long long n, double gam, double* Wl, double* Wr, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    Phys<double> ph{gam, gam - 1.0, kR, 2};
    weno_faces_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(stencils, n, ph, Wl, Wr);
    return cudaGetLastError();
}

}  // namespace gkm
