// Host instantiation of the device numerics (dns_gkm_lpt_b200/csrc/gkm_numerics.cuh)
// for CPU tests: the FP64 flux/WENO exactly as the kernels formulate them, and
// the mixed-precision flux on non-dimensional single-precision values with the
// same unit conversions as the float sweeps.  Test infrastructure only.
#include <cmath>
#include "gkm_numerics.cuh"

using namespace gkm;

namespace {
template <class T>
struct Face {
    T WL_[5], WR_[5], Wl_[5], Wr_[5], DW_[6][5];
    T WL(int q) const { return WL_[q]; }
    T WR(int q) const { return WR_[q]; }
    T Wl(int q) const { return Wl_[q]; }
    T Wr(int q) const { return Wr_[q]; }
    T DW(int v, int q) const { return DW_[v][q]; }
};
}  // namespace

extern "C" {

// in: 51 doubles (WL WR Wl Wr DW[6x5] tau0), dimensional
void hn_flux_double(const double* in, double gam, double dt, double dx, double* F)
{
    Face<double> f;
    for (int q = 0; q < 5; q++) {
        f.WL_[q] = in[q];
        f.WR_[q] = in[5 + q];
        f.Wl_[q] = in[10 + q];
        f.Wr_[q] = in[15 + q];
    }
    for (int v = 0; v < 6; v++)
        for (int q = 0; q < 5; q++) f.DW_[v][q] = in[20 + 5 * v + q];
    const Phys<double> ph{gam, gam - 1.0, kR, (int)((5.0 - 3.0 * gam) / (gam - 1.0))};
    gks_flux<double>(f, in[50], dt, dx, ph, F);
}

// the same face with the reference's moment algebra (one MCal per table, weight and slope)
void hn_flux_double_mcal(const double* in, double gam, double dt, double dx, double* F)
{
    Face<double> f;
    for (int q = 0; q < 5; q++) {
        f.WL_[q] = in[q];
        f.WR_[q] = in[5 + q];
        f.Wl_[q] = in[10 + q];
        f.Wr_[q] = in[15 + q];
    }
    for (int v = 0; v < 6; v++)
        for (int q = 0; q < 5; q++) f.DW_[v][q] = in[20 + 5 * v + q];
    const Phys<double> ph{gam, gam - 1.0, kR, (int)((5.0 - 3.0 * gam) / (gam - 1.0))};
    gks_flux_mcal<double>(f, in[50], dt, dx, ph, F);
}

// the same face on the mixed-precision path: rho / rho0, m / (rho0 us), E / p0,
// lengths in dx, times in dx / us, us = sqrt(p0 / rho0); result back in dimensional FP64
void hn_flux_mixed(const double* in, double gam, double dt, double dx, double den0, double p0, double* F)
{
    const double us = std::sqrt(p0 / den0);
    const double sc[5] = {den0, den0 * us, den0 * us, den0 * us, p0};
    Face<float> f;
    for (int q = 0; q < 5; q++) {
        f.WL_[q] = float(in[q] / sc[q]);
        f.WR_[q] = float(in[5 + q] / sc[q]);
        f.Wl_[q] = float(in[10 + q] / sc[q]);
        f.Wr_[q] = float(in[15 + q] / sc[q]);
    }
    for (int v = 0; v < 6; v++)
        for (int q = 0; q < 5; q++) f.DW_[v][q] = float(in[20 + 5 * v + q] * dx / sc[q]);
    const Phys<float> ph{float(gam), float(gam - 1.0), 1.0f, (int)((5.0 - 3.0 * gam) / (gam - 1.0))};
    float Fr[5];
    gks_flux<float>(f, float(in[50] * us / dx), float(dt * us / dx), 1.0f, ph, Fr);
    const double fs[5] = {den0 * dx, den0 * us * dx, den0 * us * dx, den0 * us * dx, p0 * dx};
    for (int q = 0; q < 5; q++) F[q] = (double)Fr[q] * fs[q];
}

void hn_weno_double(const double* s, double eps, double* l, double* r)
{
    weno_scalar<double>(s[0], s[1], s[2], s[3], s[4], s[5], eps, *l, *r);
}

void hn_weno_float(const double* s, double eps, double* l, double* r)
{
    float a, b;
    weno_scalar<float>(float(s[0]), float(s[1]), float(s[2]), float(s[3]), float(s[4]), float(s[5]), float(eps), a, b);
    *l = a;
    *r = b;
}
}
