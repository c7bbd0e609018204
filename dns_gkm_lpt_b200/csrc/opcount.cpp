// Algorithmic operation count of one cell update, taken from the device
// numerics themselves: gkm_numerics.cuh is instantiated on the host with a
// scalar type that counts every arithmetic operation it performs, in the
// reference's formulation (GKM_REFERENCE_FORM 1: its moment algebra and its
// divisions) and with one reconstruction per face.  The count is the numerator
// of the FP64 roofline reported by bench.py, so it stays fixed when the kernels
// get cheaper.
//
// Per face (one reconstruction per face, as the sweep kernels do):
//   temperature of the cell entering the stencil window  1x
//   WENO-SYMOO on rho, rho u, rho v, rho w, T (two sides) 5x
//   face energy of the two reconstructed states           2x
//   the six slope vectors formed from the reconstructions 30 values
//   collision time of the left cell (c2p + Sutherland)    1x
//   gas-kinetic flux                                      1x
//   flux-difference accumulation (x: 1, y: 2, z: 4 ops per component, plus
//   the z sweep's |u|+c for the next dt)
// A cell update is three faces (x, y, z).
//
//   g++ -O1 -std=c++17 -I. opcount.cpp -o opcount && ./opcount > opcount.json
#include <cmath>
#include <cstdio>

struct Counts {
    long long add = 0, mul = 0, div = 0, sqrt = 0, exp = 0, erfc = 0, cmp = 0, pow = 0;
};
static Counts g_cnt;

struct Num {
    double v;
    Num() : v(0) {}
    Num(double x) : v(x) {}
};
inline Num operator+(Num a, Num b) { g_cnt.add++; return Num(a.v + b.v); }
inline Num operator-(Num a, Num b) { g_cnt.add++; return Num(a.v - b.v); }
inline Num operator*(Num a, Num b) { g_cnt.mul++; return Num(a.v * b.v); }
inline Num operator/(Num a, Num b) { g_cnt.div++; return Num(a.v / b.v); }
inline Num operator-(Num a) { return Num(-a.v); }   // a sign flip, free
inline Num& operator+=(Num& a, Num b) { a = a + b; return a; }
inline Num& operator-=(Num& a, Num b) { a = a - b; return a; }
inline bool operator>(Num a, Num b) { g_cnt.cmp++; return a.v > b.v; }
inline bool operator<(Num a, Num b) { g_cnt.cmp++; return a.v < b.v; }
inline Num fabs(Num a) { return Num(std::fabs(a.v)); }
inline Num fmax(Num a, Num b) { g_cnt.cmp++; return Num(std::fmax(a.v, b.v)); }

// count the gas-kinetic moments as the reference's MCal forms them
// (src/GKMflux.cpp:238-278: two multiplications per triple product) and its
// divisions; the kernels fold the moments, form reciprocals once and execute fewer
#define GKM_REFERENCE_FORM 1
#include "gkm_numerics.cuh"

namespace gkm {
template <>
struct Wide<Num> {
    using type = Num;
};
template <>
inline Num erfc_t<Num>(Num x) { g_cnt.erfc++; return Num(std::erfc(x.v)); }
template <>
inline Num exp_t<Num>(Num x) { g_cnt.exp++; return Num(std::exp(x.v)); }
template <>
inline Num sqrt_t<Num>(Num x) { g_cnt.sqrt++; return Num(std::sqrt(x.v)); }
}  // namespace gkm

// slopes formed from shared-memory reconstructions, as SmemFace does
struct CountingFace {
    Num WLv[5], WRv[5], Wlv[5], Wrv[5], N[10], S[10], Fw[10], B[10];
    Num inv_dx;
    Num WL(int q) const { return WLv[q]; }
    Num WR(int q) const { return WRv[q]; }
    Num Wl(int q) const { return Wlv[q]; }
    Num Wr(int q) const { return Wrv[q]; }
    Num DW(int v, int q) const
    {
        switch (v) {
            case 0: return Num(2.0) * (Wlv[q] - WLv[q]) * inv_dx;
            case 1: return Num(2.0) * (WRv[q] - Wrv[q]) * inv_dx;
            case 2: return Num(0.5) * (N[q] - S[q]) * inv_dx;
            case 3: return Num(0.5) * (N[5 + q] - S[5 + q]) * inv_dx;
            case 4: return Num(0.5) * (Fw[q] - B[q]) * inv_dx;
            default: return Num(0.5) * (Fw[5 + q] - B[5 + q]) * inv_dx;
        }
    }
};

static long long total(const Counts& c) { return c.add + c.mul + c.div + c.sqrt + c.exp + c.erfc; }

static void print(const char* name, const Counts& c, const char* sep)
{
    std::printf("    \"%s\": {\"add\": %lld, \"mul\": %lld, \"div\": %lld, \"sqrt\": %lld, \"exp\": %lld, "
                "\"erfc\": %lld, \"cmp\": %lld, \"flops\": %lld}%s\n",
                name, c.add, c.mul, c.div, c.sqrt, c.exp, c.erfc, c.cmp, total(c), sep);
}

int main()
{
    using namespace gkm;
    const Phys<Num> ph{Num(1.4), Num(0.4), Num(287.0), 2};
    // a representative state (values do not change the count: the code is branch-free)
    Num W[5] = {1.0, 100.0, -50.0, 30.0, 215250.0 + 0.5 * (100.0 * 100 + 50 * 50 + 30 * 30)};

    g_cnt = Counts();
    Num Tc = temperature<Num>(W[0], W[1], W[2], W[3], W[4], ph);
    (void)Tc;
    Counts c_temp = g_cnt;

    g_cnt = Counts();
    Num l, r;
    weno_scalar<Num>(W[0], W[0], W[0], W[0], W[0], W[0], Num(1e-10), l, r);
    Counts c_weno1 = g_cnt;

    g_cnt = Counts();
    Num e = face_energy<Num>(W[0], W[1], W[2], W[3], Num(300.0), ph);
    (void)e;
    Counts c_energy = g_cnt;

    // collision time of the left cell (sweep_kernel: c2p with one reciprocal, Sutherland with x*sqrt(x))
    g_cnt = Counts();
    {
        Num d = W[0], id = Num(1.0) / d;
        Num u = W[1] * id, v = W[2] * id, w = W[3] * id;
        Num p = (d * ph.gm1) * (W[4] * id - Num(0.5) * (u * u + v * v + w * w));
        Num T = p / (Num(287.0) * d);
        Num x = T / Num(300.0);
        Num mu = Num(1.0) * (x * sqrt_t<Num>(x)) * (Num(300.0) + Num(110.4)) / (T + Num(110.4));
        Num tau = mu / p;
        (void)tau;
    }
    Counts c_tau = g_cnt;

    CountingFace f;
    for (int q = 0; q < 5; q++) {
        f.WLv[q] = W[q];
        f.WRv[q] = W[q];
        f.Wlv[q] = W[q];
        f.Wrv[q] = W[q];
        f.N[q] = f.N[5 + q] = f.Fw[q] = f.Fw[5 + q] = W[q];
        f.S[q] = f.S[5 + q] = f.B[q] = f.B[5 + q] = W[q];
    }
    f.N[0] = f.N[5] = Num(1.001);
    f.inv_dx = Num(10.0);
    g_cnt = Counts();
    Num F[5];
    gks_flux<Num>(f, Num(1e-5), Num(3e-4), Num(0.1), ph, F);
    Counts c_flux = g_cnt;

    Counts acc;   // accumulation per face summed over x, y, z: 1 + 2 + 4 ops per component
    acc.add = 5 * (1 + 2 + 3);
    acc.mul = 5 * 1;
    Counts wave;  // |u|+c of the new cell (z sweep): 3 div, 3 mul, 2 add (|u|^2), 1 mul 1 div 1 mul 1 add (p),
                  // 1 mul 1 div (gam p / rho), 2 sqrt, 1 add
    wave.div = 5;
    wave.mul = 6;
    wave.add = 4;
    wave.sqrt = 2;

    Counts face;  // one face of one sweep, excluding the accumulation
    auto addc = [](Counts& a, const Counts& b, int k) {
        a.add += k * b.add; a.mul += k * b.mul; a.div += k * b.div; a.sqrt += k * b.sqrt;
        a.exp += k * b.exp; a.erfc += k * b.erfc; a.cmp += k * b.cmp;
    };
    addc(face, c_temp, 1);
    addc(face, c_weno1, 5);
    addc(face, c_energy, 2);
    addc(face, c_tau, 1);
    addc(face, c_flux, 1);
    Counts cell;
    addc(cell, face, 3);
    addc(cell, acc, 1);
    addc(cell, wave, 1);

    std::printf("{\n  \"what\": \"FP64 operations of one cell update (three faces): reference formulation of the moments, one reconstruction per face\",\n");
    std::printf("  \"per_call\": {\n");
    print("temperature", c_temp, ",");
    print("weno_scalar_both_sides", c_weno1, ",");
    print("face_energy", c_energy, ",");
    print("collision_time", c_tau, ",");
    print("gks_flux_incl_slopes", c_flux, "");
    std::printf("  },\n");
    print("per_face", face, ",");
    print("per_cell_update", cell, ",");
    std::printf("  \"flops_per_cell_update\": %lld,\n", total(cell));
    std::printf("  \"flops_per_face\": %lld\n}\n", total(face));
    return 0;
}
