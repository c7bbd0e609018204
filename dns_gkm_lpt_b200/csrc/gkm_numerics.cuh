// Device numerics of the gas-kinetic step: WENO-SYMOO reconstruction and the
// BGK flux integrated over one time step.  Templated on the arithmetic type T
// (double for the FP64 drop-in, float for the mixed-precision form).
//
// Mathematics follow the reference CPU path:
//   WENO-SYMOO        src/update.cpp:556-680
//   flux              src/GKMflux.cpp:11-229
//   moment products   src/GKMflux.cpp:238-278 (MCal)
//   slope solve       src/GKMflux.cpp:283-297
//   c2p               src/GKMflux.cpp:302-309
//
// Two forms of the flux.  gks_flux_mcal keeps the reference's moment algebra
// (one MCal per table, weight and slope vector) and is what the operation
// counter measures.  gks_flux_tau, the one the kernels run, takes the same
// moments of the same slope vectors as contractions of the normal tables with
// tangential functionals of each slope polynomial, and forms each reciprocal
// once (grouped divisions, one reciprocal square root per state).  The two
// forms and the reference differ only by rounding.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#define GKM_HD __host__ __device__ __forceinline__
#include "f32x2.cuh"
#else
// host-only compilation (op counting, CPU checks of the device numerics)
#include <algorithm>
#include <cmath>
#define GKM_HD inline
#endif

// GKM_REFERENCE_FORM 1 keeps the reference's arithmetic in the shared helpers
// (two divisions per WENO scalar, the divisions of temperature and face energy)
// and its MCal moment algebra; the operation counter compiles that form.  The
// kernels (0) form each reciprocal once and fold the moments.
#ifndef GKM_REFERENCE_FORM
#define GKM_REFERENCE_FORM 0
#endif

// Code shape of the flux: both half-Maxwellian sides unrolled (one copy of the
// side code per side) or one loop body.
#ifndef GKM_UNROLL_SIDES
#define GKM_UNROLL_SIDES 1
#endif

namespace gkm {

// single-precision arithmetic: float, and the packed pair F2 (f32x2.cuh)
template <class T>
struct single_t {
    static constexpr bool value = sizeof(T) == 4;
};
#ifdef __CUDACC__
template <>
struct single_t<F2> {
    static constexpr bool value = true;
};
#endif

constexpr double kR = 287.0;        // gas constant, src/param.h:21
constexpr double kPrandtl = 0.70;   // src/param.h:19
constexpr double kWenoEps = 1e-10;  // pow(10,-10), src/param.h:18

template <class T>
struct Phys {
    T gam;        // ratio of specific heats
    T gm1;        // gam - 1
    T Rg;         // gas constant in the working units
    int K;        // internal degrees of freedom (int((5-3g)/(g-1)))
};

// ---------------------------------------------------------------- WENO ----
// One scalar, both sides of the face between cells L (=a1) and R (=b1).
// a3, a2, a1 = cells L-2, L-1, L ; b1, b2, b3 = cells R, R+1, R+2.
// Linear weights 1/20, 9/20, 9/20, 1/20; IS_3 replaced by max(IS_0..IS_3);
// alpha_k = g_k / (eps + IS_k).  The normalised weights are formed with one
// division: w_k = g_k prod_{m!=k}(eps+IS_m) / sum_m g_m prod_{m'!=m}(eps+IS_m').
// ND: return the double-precision form's numerators and denominators (o0..o3 = Nl, Dl,
// Nr, Dr, so a caller can share one division among several scalars); else o0, o1 =
// the reconstructed left and right values.
template <class T, bool ND>
GKM_HD void weno_core(T a3, T a2, T a1, T b1, T b2, T b3, T eps, T& o0, T& o1, T& o2, T& o3)
{
    const T c13 = T(1.0 / 3.0), c76 = T(7.0 / 6.0), c116 = T(11.0 / 6.0), c16 = T(1.0 / 6.0), c56 = T(5.0 / 6.0);
    const T c1312 = T(13.0 / 12.0), c14 = T(0.25);
#if GKM_REFERENCE_FORM
    // candidate polynomials (left-biased "p", right-biased "n")
    T P0p = a3 * c13 - a2 * c76 + a1 * c116;
    T P0n = b3 * c13 - b2 * c76 + b1 * c116;
    T P1p = -a2 * c16 + a1 * c56 + b1 * c13;
    T P1n = -b2 * c16 + b1 * c56 + a1 * c13;
    T P2p = a1 * c13 + b1 * c56 - b2 * c16;
    T P2n = b1 * c13 + a1 * c56 - a2 * c16;
    T P3p = b1 * c116 - b2 * c76 + b3 * c13;
    T P3n = a1 * c116 - a2 * c76 + a3 * c13;
    // smoothness indicators
    T d;
    T e;
    d = a3 - T(2) * a2 + a1; e = a3 - T(4) * a2 + T(3) * a1; T I0p = c1312 * d * d + c14 * e * e;
    d = b3 - T(2) * b2 + b1; e = b3 - T(4) * b2 + T(3) * b1; T I0n = c1312 * d * d + c14 * e * e;
    d = a2 - T(2) * a1 + b1; e = b1 - a2;                    T I1p = c1312 * d * d + c14 * e * e;
    d = b2 - T(2) * b1 + a1; e = a1 - b2;                    T I1n = c1312 * d * d + c14 * e * e;
    d = a1 - T(2) * b1 + b2; e = -T(3) * a1 + T(4) * b1 - b2; T I2p = c1312 * d * d + c14 * e * e;
    d = b1 - T(2) * a1 + a2; e = -T(3) * b1 + T(4) * a1 - a2; T I2n = c1312 * d * d + c14 * e * e;
    d = b1 - T(2) * b2 + b3; e = -T(5) * b1 + T(8) * b2 - T(3) * b3; T I3p = c1312 * d * d + c14 * e * e;
    d = a1 - T(2) * a2 + a3; e = -T(5) * a1 + T(8) * a2 - T(3) * a3; T I3n = c1312 * d * d + c14 * e * e;
#else
    // the left-biased candidate k and the right-biased candidate 3-k are the same polynomial
    // of the same three cells, and so are the second differences of their indicators: four of
    // each instead of eight
    const T Pa = a3 * c13 - a2 * c76 + a1 * c116;   // P0p = P3n
    const T Pb = -a2 * c16 + a1 * c56 + b1 * c13;   // P1p = P2n
    const T Pc = a1 * c13 + b1 * c56 - b2 * c16;    // P2p = P1n
    const T Pd = b1 * c116 - b2 * c76 + b3 * c13;   // P3p = P0n
    const T P0p = Pa, P3n = Pa, P1p = Pb, P2n = Pb, P2p = Pc, P1n = Pc, P3p = Pd, P0n = Pd;
    const T dA = a3 - T(2) * a2 + a1, dB = a2 - T(2) * a1 + b1, dC = a1 - T(2) * b1 + b2, dD = b1 - T(2) * b2 + b3;
    const T qA = c1312 * dA * dA, qB = c1312 * dB * dB, qC = c1312 * dC * dC, qD = c1312 * dD * dD;
    T e;
    e = a3 - T(4) * a2 + T(3) * a1;         T I0p = qA + c14 * e * e;
    e = b3 - T(4) * b2 + T(3) * b1;         T I0n = qD + c14 * e * e;
    e = b1 - a2;                            T I1p = qB + c14 * e * e;
    e = a1 - b2;                            T I1n = qC + c14 * e * e;
    e = -T(3) * a1 + T(4) * b1 - b2;        T I2p = qC + c14 * e * e;
    e = -T(3) * b1 + T(4) * a1 - a2;        T I2n = qB + c14 * e * e;
    e = -T(5) * b1 + T(8) * b2 - T(3) * b3; T I3p = qD + c14 * e * e;
    e = -T(5) * a1 + T(8) * a2 - T(3) * a3; T I3n = qA + c14 * e * e;
#endif
    I3p = fmax(fmax(fmax(I0p, I1p), I2p), I3p);
    I3n = fmax(fmax(fmax(I0n, I1n), I2n), I3n);
    if constexpr (single_t<T>::value) {
        static_assert(!ND, "the single-precision form has no shared denominators");
        // single precision: products of three (eps + IS) underflow on flat stencils,
        // so form the alphas from reciprocals
        T a0 = T(1) / (eps + I0p), a1 = T(9) / (eps + I1p), a2 = T(9) / (eps + I2p), a3 = T(1) / (eps + I3p);
        o0 = (a0 * P0p + a1 * P1p + a2 * P2p + a3 * P3p) / (a0 + a1 + a2 + a3);
        a0 = T(1) / (eps + I0n);
        a1 = T(9) / (eps + I1n);
        a2 = T(9) / (eps + I2n);
        a3 = T(1) / (eps + I3n);
        o1 = (a0 * P0n + a1 * P1n + a2 * P2n + a3 * P3n) / (a0 + a1 + a2 + a3);
        return;
    }
    T Nl, Dl, Nr, Dr;
    {
        T e0 = eps + I0p, e1 = eps + I1p, e2 = eps + I2p, e3 = eps + I3p;
        T p01 = e0 * e1, p23 = e2 * e3;
        T n0 = e1 * p23, n1 = T(9) * e0 * p23, n2 = T(9) * p01 * e3, n3 = p01 * e2;
        Nl = n0 * P0p + n1 * P1p + n2 * P2p + n3 * P3p;
        Dl = n0 + n1 + n2 + n3;
    }
    {
        T e0 = eps + I0n, e1 = eps + I1n, e2 = eps + I2n, e3 = eps + I3n;
        T p01 = e0 * e1, p23 = e2 * e3;
        T n0 = e1 * p23, n1 = T(9) * e0 * p23, n2 = T(9) * p01 * e3, n3 = p01 * e2;
        Nr = n0 * P0n + n1 * P1n + n2 * P2n + n3 * P3n;
        Dr = n0 + n1 + n2 + n3;
    }
    if constexpr (ND) {
        o0 = Nl;
        o1 = Dl;
        o2 = Nr;
        o3 = Dr;
        return;
    }
#if GKM_REFERENCE_FORM
    o0 = Nl / Dl;
    o1 = Nr / Dr;
#else
    // both sides with one division: D ranges from 4 eps^3 (flat stencil) to about IS_max^3,
    // so Dl Dr stays far inside the double range for any physical state
    const T inv = T(1) / (Dl * Dr);
    o0 = Nl * (Dr * inv);
    o1 = Nr * (Dl * inv);
#endif
}

template <class T>
GKM_HD void weno_scalar(T a3, T a2, T a1, T b1, T b2, T b3, T eps, T& fl, T& fr)
{
    T u0, u1;
    weno_core<T, false>(a3, a2, a1, b1, b2, b3, eps, fl, fr, u0, u1);
}

// numerators and denominators of both sides (double precision), fl = Nl / Dl, fr = Nr / Dr
template <class T>
GKM_HD void weno_nd(T a3, T a2, T a1, T b1, T b2, T b3, T eps, T& Nl, T& Dl, T& Nr, T& Dr)
{
    weno_core<T, true>(a3, a2, a1, b1, b2, b3, eps, Nl, Dl, Nr, Dr);
}

// temperature of a conserved state, src/update.cpp:615-620
template <class T>
GKM_HD T temperature(T r, T m1, T m2, T m3, T E, const Phys<T>& ph)
{
    T ir = T(1) / r;
#if GKM_REFERENCE_FORM
    return ph.gm1 * (E * ir - T(0.5) * (m1 * m1 + m2 * m2 + m3 * m3) * ir * ir) / ph.Rg;
#else
    return (E * ir - T(0.5) * (m1 * m1 + m2 * m2 + m3 * m3) * ir * ir) * (ph.gm1 / ph.Rg);
#endif
}

// face energy from reconstructed rho, momentum and temperature, src/update.cpp:673-674
template <class T>
GKM_HD T face_energy(T r, T m1, T m2, T m3, T Tf, const Phys<T>& ph)
{
#if GKM_REFERENCE_FORM
    return r * ph.Rg * Tf / ph.gm1 + T(0.5) * (m1 * m1 + m2 * m2 + m3 * m3) / r;
#else
    return r * Tf * (ph.Rg / ph.gm1) + T(0.5) * (m1 * m1 + m2 * m2 + m3 * m3) / r;
#endif
}

// face energy with 1/r given (the sweeps form the two sides' reciprocals together)
template <class T>
GKM_HD T face_energy_ir(T r, T ir, T m1, T m2, T m3, T Tf, const Phys<T>& ph)
{
    return r * Tf * (ph.Rg / ph.gm1) + T(0.5) * (m1 * m1 + m2 * m2 + m3 * m3) * ir;
}

// ------------------------------------------------------ moment tables ----
// Maxwellian moments of one state: x half-space table H (and H2 for the
// equilibrium state's other half), full tables X (x), Y (y), Z (z).
// src/GKMflux.cpp:45-68 (l, r) and :85-103 (e).
// The tangential tables enter the moments only as products Y[b] Z[c] with
// b + c <= 5, so they are kept as that 21-entry product table: every triple
// product of MCal then costs one multiplication instead of two.
// (GKM_SHARED_YZ 0 keeps the separate tables and forms every triple product
// with two multiplications as the reference's MCal does; the operation counter
// uses that to count the reference formulation.)
#ifndef GKM_SHARED_YZ
#define GKM_SHARED_YZ (!GKM_REFERENCE_FORM)
#endif
constexpr int kYZ = 21;
GKM_HD constexpr int yz(int b, int c) { return 6 * c - c * (c - 1) / 2 + b; }

template <class T>
struct Moments {
    T H[7];
    T X[7];
#if GKM_SHARED_YZ
    T YZ[kYZ];
#else
    T Y[6], Z[6];
#endif
    T Ie2, Ie4;
};

template <class T>
GKM_HD T erfc_t(T x);
template <>
GKM_HD double erfc_t<double>(double x) { return ::erfc(x); }
template <>
GKM_HD float erfc_t<float>(float x) { return erfcf(x); }
template <class T>
GKM_HD T exp_t(T x);
template <>
GKM_HD double exp_t<double>(double x) { return exp(x); }
template <>
GKM_HD float exp_t<float>(float x) { return expf(x); }
template <class T>
GKM_HD T sqrt_t(T x);
template <>
GKM_HD double sqrt_t<double>(double x) { return sqrt(x); }
template <>
GKM_HD float sqrt_t<float>(float x) { return sqrtf(x); }
// 1 / sqrt(x): the device's reciprocal square root (within 1 ulp), on the host 1 / sqrt
template <class T>
GKM_HD T rsqrt_t(T x);
template <>
GKM_HD double rsqrt_t<double>(double x)
{
#ifdef __CUDA_ARCH__
    return rsqrt(x);
#else
    return 1.0 / sqrt(x);
#endif
}
template <>
GKM_HD float rsqrt_t<float>(float x)
{
#ifdef __CUDA_ARCH__
    return rsqrtf(x);
#else
    return 1.0f / sqrtf(x);
#endif
}

// half: +1 positive-u half space (erfc(-sqrt(lam) u)/2), -1 negative half
template <class T>
GKM_HD void half_table(T* H, T U0, T lam, T inv2lam, int half)
{
    const T pi = T(3.14159265358979323846);
    T sl = sqrt_t<T>(lam);
    T g = T(0.5) * exp_t<T>(-lam * U0 * U0) / sqrt_t<T>(lam * pi);
    if (half > 0) {
        H[0] = T(0.5) * erfc_t<T>(-sl * U0);
        H[1] = U0 * H[0] + g;
    } else {
        H[0] = T(0.5) * erfc_t<T>(sl * U0);
        H[1] = U0 * H[0] - g;
    }
#pragma unroll
    for (int i = 2; i < 7; i++) H[i] = U0 * H[i - 1] + H[i - 2] * (T(i - 1) * inv2lam);
}

template <class T, int N>
GKM_HD void full_table(T* F, T U, T inv2lam)
{
    F[0] = T(1);
    F[1] = U;
#pragma unroll
    for (int i = 2; i < N; i++) F[i] = U * F[i - 1] + F[i - 2] * (T(i - 1) * inv2lam);
}

template <class T>
GKM_HD void build_moments(Moments<T>& M, const T U[3], T lam, int K, int half)
{
    T inv2lam = T(1) / (T(2) * lam);
    M.Ie2 = T(K) * inv2lam;
    M.Ie4 = T(3 * K + K * (K - 1)) * inv2lam * inv2lam;
    half_table<T>(M.H, U[0], lam, inv2lam, half);
    full_table<T, 7>(M.X, U[0], inv2lam);
#if GKM_SHARED_YZ
    T Y[6], Z[6];
    full_table<T, 6>(Y, U[1], inv2lam);
    full_table<T, 6>(Z, U[2], inv2lam);
#pragma unroll
    for (int c = 0; c < 6; c++)
#pragma unroll
        for (int b = 0; b + c < 6; b++) M.YZ[yz(b, c)] = Y[b] * Z[c];
#else
    full_table<T, 6>(M.Y, U[1], inv2lam);
    full_table<T, 6>(M.Z, U[2], inv2lam);
#endif
}

#if GKM_SHARED_YZ
#define GKM_TABLES(S) S.YZ
#define TM(A, B, C) (I[k + (A)] * YZ[yz(l + (B), m + (C))])
#define GKM_YZ_PARAM const T* YZ
#else
#define GKM_TABLES(S) S.Y, S.Z
#define TM(A, B, C) (I[k + (A)] * Y[l + (B)] * Z[m + (C)])
#define GKM_YZ_PARAM const T* Y, const T* Z
#endif

// ----------------------------------------------------------- MCal -----
// <psi (u^k v^l w^m) (a0 + a1 u + a2 v + a3 w + a4 psi4)> with psi = (1,u,v,w,psi4),
// psi4 = (u^2+v^2+w^2+xi^2)/2; I = normal table (full or half), Y, Z tangential.
template <int k, int l, int m, class T>
GKM_HD void mcal(T M[5], const T* I, GKM_YZ_PARAM, T Ie2, T Ie4, const T a[5])
{
    T t000 = TM(0, 0, 0), t100 = TM(1, 0, 0), t010 = TM(0, 1, 0), t001 = TM(0, 0, 1);
    T t200 = TM(2, 0, 0), t020 = TM(0, 2, 0), t002 = TM(0, 0, 2);
    T t110 = TM(1, 1, 0), t101 = TM(1, 0, 1), t011 = TM(0, 1, 1);
    T v0 = T(0.5) * (t200 + t020 + t002 + t000 * Ie2);
    T v1 = T(0.5) * (TM(3, 0, 0) + TM(1, 2, 0) + TM(1, 0, 2) + t100 * Ie2);
    T v2 = T(0.5) * (TM(2, 1, 0) + TM(0, 3, 0) + TM(0, 1, 2) + t010 * Ie2);
    T v3 = T(0.5) * (TM(2, 0, 1) + TM(0, 2, 1) + TM(0, 0, 3) + t001 * Ie2);
    M[0] = a[0] * t000 + a[1] * t100 + a[2] * t010 + a[3] * t001 + a[4] * v0;
    M[1] = a[0] * t100 + a[1] * t200 + a[2] * t110 + a[3] * t101 + a[4] * v1;
    M[2] = a[0] * t010 + a[1] * t110 + a[2] * t020 + a[3] * t011 + a[4] * v2;
    M[3] = a[0] * t001 + a[1] * t101 + a[2] * t011 + a[3] * t002 + a[4] * v3;
    M[4] = T(0.25) * a[4] *
               (TM(4, 0, 0) + TM(0, 4, 0) + TM(0, 0, 4) + t000 * Ie4 +
                T(2) * (TM(2, 2, 0) + TM(2, 0, 2) + t200 * Ie2 + TM(0, 2, 2) + t020 * Ie2 + t002 * Ie2)) +
           a[0] * v0 + a[1] * v1 + a[2] * v2 + a[3] * v3;
}

template <int k, int l, int m, class T>
GKM_HD void mcal0(T M[5], const T* I, GKM_YZ_PARAM, T Ie2)
{
    M[0] = TM(0, 0, 0);
    M[1] = TM(1, 0, 0);
    M[2] = TM(0, 1, 0);
    M[3] = TM(0, 0, 1);
    M[4] = T(0.5) * (TM(2, 0, 0) + TM(0, 2, 0) + TM(0, 0, 2) + TM(0, 0, 0) * Ie2);
}

template <class T>
GKM_HD void axpy5(T* acc, T s, const T* M)
{
#pragma unroll
    for (int q = 0; q < 5; q++) acc[q] += s * M[q];
}

// ----------------------------------------------------- slope solver ---
// Solve the 5x5 moment system for the Maxwellian slope coefficients, with the
// Prandtl-number correction on the energy component (src/GKMflux.cpp:283-297).
template <class T>
struct SlopeState {
    T U[3];
    T lam2;     // 2 lam
    T usqc;     // u.u + (K+3)/(2 lam)
    T a4fac;    // (1/Pr) (4 lam^2) / (K+3)
};

template <class T>
GKM_HD SlopeState<T> slope_state(const T U[3], T lam, int K)
{
    SlopeState<T> s;
    s.U[0] = U[0];
    s.U[1] = U[1];
    s.U[2] = U[2];
    s.lam2 = T(2) * lam;
    s.usqc = U[0] * U[0] + U[1] * U[1] + U[2] * U[2] + T(K + 3) / s.lam2;
    s.a4fac = T(1.0 / kPrandtl) * (T(4) * lam * lam) / T(K + 3);
    return s;
}

template <class T>
GKM_HD void slope_solve(const T b[5], const SlopeState<T>& s, T a[5])
{
    T r2 = b[1] - s.U[0] * b[0];
    T r3 = b[2] - s.U[1] * b[0];
    T r4 = b[3] - s.U[2] * b[0];
    T r5 = T(2) * b[4] - b[0] * s.usqc;
    a[4] = s.a4fac * (r5 - T(2) * (s.U[0] * r2 + s.U[1] * r3 + s.U[2] * r4));
    a[3] = s.lam2 * r4 - s.U[2] * a[4];
    a[2] = s.lam2 * r3 - s.U[1] * a[4];
    a[1] = s.lam2 * r2 - s.U[0] * a[4];
    a[0] = b[0] - a[1] * s.U[0] - a[2] * s.U[1] - a[3] * s.U[2] - T(0.5) * a[4] * s.usqc;
}

template <class T>
GKM_HD void c2p(const T W[5], T gm1, T& den, T U[3], T& P)
{
    den = W[0];
    T ir = T(1) / den;
    U[0] = W[1] * ir;
    U[1] = W[2] * ir;
    U[2] = W[3] * ir;
    P = (den * gm1) * (W[4] * ir - T(0.5) * (U[0] * U[0] + U[1] * U[1] + U[2] * U[2]));
}

// ------------------------------------------------- time coefficients ----
// Integrals over [0, dt] of the BGK relaxation, src/GKMflux.cpp:162-167,197-204.
// With e = exp(-dt/tau) the coefficients are differences of nearly equal terms
// when dt/tau is small, so they are always formed in double precision
// (wide_t), whatever type the flux itself runs in.
template <class T>
struct Wide {
    using type = double;
};
template <class T>
using wide_t = typename Wide<T>::type;

template <class D>
struct TimeCoefs {
    D gm1, gm2, gm3, gm4, gm5, p0, p1, p2, p3, p4, p5;
};

// BGK time integrals over [0, dt] with e = exp(-dt/tau) (src/GKMflux.cpp:162-167,197-204).
// EXPM1: 1 - e as -expm1(-dt/tau), exact where dt/tau is small (the mixed form,
// whose flux runs in FP32 and gets these FP64 coefficients); otherwise the
// reference's 1 - e.
template <class D, bool EXPM1 = false>
GKM_HD TimeCoefs<D> time_coefs(D tau, D dt)
{
    TimeCoefs<D> c;
    D ex = exp_t<D>(-dt / tau);
    D omx;
    if constexpr (EXPM1) omx = -expm1(-dt / tau);
    else omx = D(1) - ex;
    D gm0 = dt - tau * omx;
    D igm0 = D(1) / gm0;
    c.gm1 = -omx * igm0;
    c.gm2 = (-dt + D(2) * tau * omx - dt * ex) * igm0;
    c.gm3 = -c.gm1;
    c.gm4 = (dt * ex - tau * omx) * igm0;
    c.gm5 = tau * c.gm3;
    D Pc = tau * omx;                               // -tau (e - 1)
    D Qc = -tau * dt * ex + tau * tau * omx;        // -tau dt e - tau^2 (e - 1)
    c.p0 = dt - Pc;
    c.p1 = D(0.5) * dt * dt - tau * c.p0;
    c.p2 = -tau * c.p0 + Qc;
    c.p3 = Pc;
    c.p4 = -Qc - tau * Pc;
    c.p5 = -tau * Pc;
    return c;
}

// --------------------------------------------------------- the flux ----
// The face inputs come from a provider so that the 30 slope values are formed
// where they are consumed instead of being held in registers.  A provider has
//   T WL(int q), WR(int q)   cell averages left/right of the face
//   T Wl(int q), Wr(int q)   reconstructed face states
//   T DW(int v, int q)       slope vectors v = 0..5: DWxl, DWxr, DWyl, DWyr, DWzl, DWzr
// all in the face frame (slot 1 = normal momentum).  tau0 = mu(T_L)/p_L of the
// left cell.  Output F[5] = flux integrated over [0, dt] (not divided by dt).
template <class T>
struct FaceInput {
    T WL_[5], WR_[5], Wl_[5], Wr_[5];
    T DW_[6][5];
    GKM_HD T WL(int q) const { return WL_[q]; }
    GKM_HD T WR(int q) const { return WR_[q]; }
    GKM_HD T Wl(int q) const { return Wl_[q]; }
    GKM_HD T Wr(int q) const { return Wr_[q]; }
    GKM_HD T DW(int v, int q) const { return DW_[v][q]; }
};

// The flux with the reference's moment algebra: one MCal (25 triple products
// and their sums) per table, weight and slope vector.  The operation counter
// instantiates this form; the kernels run gks_flux_tau below.
template <class T, class Prov>
GKM_HD void gks_flux_mcal(const Prov& in, T tau0, T dt, T dx, const Phys<T>& ph, T F[5])
{
    const int K = ph.K;
    T denl, Ul[3], Pl, denr, Ur[3], Pr;
    {
        T wl[5], wr[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            wl[q] = in.Wl(q);
            wr[q] = in.Wr(q);
        }
        c2p<T>(wl, ph.gm1, denl, Ul, Pl);
        c2p<T>(wr, ph.gm1, denr, Ur, Pr);
    }
    T laml = T(0.5) * denl / Pl;
    T lamr = T(0.5) * denr / Pr;

    // collision time with the pressure-jump correction, src/GKMflux.cpp:156-157
    T ql = denl / laml, qr = denr / lamr;
    const TimeCoefs<wide_t<T>> tc = time_coefs<wide_t<T>, (sizeof(T) < sizeof(wide_t<T>))>(
        wide_t<T>(tau0) + wide_t<T>(dt) * wide_t<T>(fabs(ql - qr) / fabs(ql + qr)), wide_t<T>(dt));
    const T gm1 = T(tc.gm1), gm2 = T(tc.gm2), gm3 = T(tc.gm3), gm4 = T(tc.gm4), gm5 = T(tc.gm5);
    const T p0 = T(tc.p0), p1 = T(tc.p1), p2 = T(tc.p2), p3 = T(tc.p3), p4 = T(tc.p4), p5 = T(tc.p5);

    T We[5] = {0, 0, 0, 0, 0};      // equilibrium state at the face, src/GKMflux.cpp:73-77
    T by_[5] = {0, 0, 0, 0, 0}, bz_[5] = {0, 0, 0, 0, 0};
    T Bacc[5] = {0, 0, 0, 0, 0};   // B_ * dene, without the gm1/gm3 terms
    T Facc[5] = {0, 0, 0, 0, 0};
    T M[5];

    const T cB = gm4 + gm5;
    // ---------------- one side (l: positive half with left state, r: negative half with right state)
#if GKM_UNROLL_SIDES
#pragma unroll
#else
#pragma unroll 1
#endif
    for (int side = 0; side < 2; side++) {
        const T den = side == 0 ? denl : denr;
        const T* Us = side == 0 ? Ul : Ur;
        const T lam = side == 0 ? laml : lamr;
        Moments<T> S;
        build_moments<T>(S, Us, lam, K, side == 0 ? +1 : -1);
        SlopeState<T> ss = slope_state<T>(Us, lam, K);
        T iden = T(1) / den;
        mcal0<0, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2);
        axpy5<T>(We, den, M);
        T Bs[5] = {0, 0, 0, 0, 0};   // -(Mf100 ax + Mf010 ay + Mf001 az)
        T b[5], a[5];
        // normal slope
#pragma unroll
        for (int q = 0; q < 5; q++) b[q] = in.DW(0 + side, q) * iden;
        slope_solve<T>(b, ss, a);
        mcal<1, 0, 0, T>(M, S.X, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Bs, T(-1), M);
        mcal<1, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Bacc, cB * den, M);
        mcal<2, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Facc, p4 * den, M);
        // first tangential slope
#pragma unroll
        for (int q = 0; q < 5; q++) b[q] = in.DW(2 + side, q) * iden;
        slope_solve<T>(b, ss, a);
        mcal<0, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(by_, T(1), M);
        mcal<0, 1, 0, T>(M, S.X, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Bs, T(-1), M);
        mcal<0, 1, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Bacc, cB * den, M);
        mcal<1, 1, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Facc, p4 * den, M);
        // second tangential slope
#pragma unroll
        for (int q = 0; q < 5; q++) b[q] = in.DW(4 + side, q) * iden;
        slope_solve<T>(b, ss, a);
        mcal<0, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(bz_, T(1), M);
        mcal<0, 0, 1, T>(M, S.X, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Bs, T(-1), M);
        mcal<0, 0, 1, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Bacc, cB * den, M);
        mcal<1, 0, 1, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Facc, p4 * den, M);
        // time slope of this side, src/GKMflux.cpp:145-151
        slope_solve<T>(Bs, ss, a);
        mcal<0, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Bacc, gm5 * den, M);
        mcal<1, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2, S.Ie4, a);
        axpy5<T>(Facc, p5 * den, M);
        // free transport of the initial half-Maxwellian
        mcal0<1, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2);
        axpy5<T>(Facc, p3 * den, M);
    }

    // ---------------- equilibrium part
    T dene, Ue[3], Pe;
    c2p<T>(We, ph.gm1, dene, Ue, Pe);
    T lame = T(0.5) * dene / Pe;
    Moments<T> E;
    build_moments<T>(E, Ue, lame, K, +1);
    T H2[7];
    {
        T inv2lam = T(1) / (T(2) * lame);
        half_table<T>(H2, Ue[0], lame, inv2lam, -1);
    }
    SlopeState<T> se = slope_state<T>(Ue, lame, K);
    T b[5], a[5];
    const T idx2 = T(2) / (dene * dx);
    // normal equilibrium slopes from the cell averages, src/GKMflux.cpp:115-116
#pragma unroll
    for (int q = 0; q < 5; q++) b[q] = (We[q] - in.WL(q)) * idx2;
    slope_solve<T>(b, se, a);
    mcal<1, 0, 0, T>(M, E.H, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Bacc, gm2 * dene, M);
    mcal<2, 0, 0, T>(M, E.H, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Facc, p2 * dene, M);
#pragma unroll
    for (int q = 0; q < 5; q++) b[q] = (in.WR(q) - We[q]) * idx2;
    slope_solve<T>(b, se, a);
    mcal<1, 0, 0, T>(M, H2, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Bacc, gm2 * dene, M);
    mcal<2, 0, 0, T>(M, H2, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Facc, p2 * dene, M);
    // tangential equilibrium slopes
    slope_solve<T>(by_, se, a);
    mcal<0, 1, 0, T>(M, E.X, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Bacc, gm2 * dene, M);
    mcal<1, 1, 0, T>(M, E.X, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Facc, p2 * dene, M);
    slope_solve<T>(bz_, se, a);
    mcal<0, 0, 1, T>(M, E.X, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Bacc, gm2 * dene, M);
    mcal<1, 0, 1, T>(M, E.X, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Facc, p2 * dene, M);
    // time derivative of the equilibrium, src/GKMflux.cpp:183-191
    mcal0<0, 0, 0, T>(M, E.X, GKM_TABLES(E), E.Ie2);
    T idene = T(1) / dene;
#pragma unroll
    for (int q = 0; q < 5; q++) b[q] = (gm1 * dene * M[q] + Bacc[q] + gm3 * We[q]) * idene;
    slope_solve<T>(b, se, a);
    mcal<1, 0, 0, T>(M, E.X, GKM_TABLES(E), E.Ie2, E.Ie4, a);
    axpy5<T>(Facc, p1 * dene, M);
    mcal0<1, 0, 0, T>(M, E.X, GKM_TABLES(E), E.Ie2);
    axpy5<T>(Facc, p0 * dene, M);
#pragma unroll
    for (int q = 0; q < 5; q++) F[q] = Facc[q];
}

#if GKM_SHARED_YZ
// ------------------------------------------------ moment functionals ----
// Every moment the flux takes is <u^k psi_i P>_N for a table N (full or half
// space) and a polynomial P built from slope vectors: P = psi.a, or
// G = u (psi.a_n) + v (psi.a_y) + w (psi.a_z).  Writing P = sum_p u^p Q_p(v, w, xi^2),
//   <u^k psi_i P>_N = sum_p N[p + k] tau_i(Q_p)          (i = 0, 2, 3)
//   <u^k psi_1 P>_N = sum_p N[p + k + 1] tau_0(Q_p)
//   <u^k psi_4 P>_N = sum_p (N[p + k + 2] tau_0(Q_p) / 2 + N[p + k] tau_4(Q_p))
// with the tangential functionals tau_0 = <Q>, tau_2 = <v Q>, tau_3 = <w Q>,
// tau_4 = <(v^2 + w^2 + xi^2) Q> / 2.  They involve the tangential tables only,
// so one set serves the full and the half-space table and the weights u^0 and
// u^1: a contraction costs 24 multiply-adds where MCal forms 25 triple
// products and their sums again.  Same moments, summed in another order.
template <class T>
struct Tau {
    T c0[4], cv[4], cw[4], c4[4];   // tau_0, tau_2, tau_3, tau_4 of Q_0 .. Q_3
};

template <bool ADD, class T, class V>
GKM_HD void put(T& x, const V& v)
{
    if constexpr (ADD) x += v;
    else x = v;
}

// mu(q, r, s) = <v^q w^r xi^(2s)>
template <int Q, int R, int S, class T>
GKM_HD T mu(const Moments<T>& M)
{
    static_assert(Q + R <= 5 && S <= 2, "tangential moment beyond the tables");
    if constexpr (S == 0) return M.YZ[yz(Q, R)];
    else if constexpr (S == 1) return M.YZ[yz(Q, R)] * M.Ie2;
    else return M.YZ[yz(Q, R)] * M.Ie4;
}

// <v^q w^r xi^(2s) R(a)>, R(a) = a0 + a2 v + a3 w + (a4/2)(v^2 + w^2 + xi^2) the u-free part of psi.a
template <int Q, int R, int S, class T>
GKM_HD T rho_moment(const T a[5], T h4, const Moments<T>& M)
{
    return a[0] * mu<Q, R, S>(M) + a[2] * mu<Q + 1, R, S>(M) + a[3] * mu<Q, R + 1, S>(M) +
           h4 * (mu<Q + 2, R, S>(M) + mu<Q, R + 2, S>(M) + mu<Q, R, S + 1>(M));
}

// functionals of Q = v^q w^r R(a) into entry p
template <bool ADD, int Q, int R, int P, class T>
GKM_HD void tau_R(Tau<T>& t, const T a[5], T h4, const Moments<T>& M)
{
    put<ADD>(t.c0[P], rho_moment<Q, R, 0>(a, h4, M));
    put<ADD>(t.cv[P], rho_moment<Q + 1, R, 0>(a, h4, M));
    put<ADD>(t.cw[P], rho_moment<Q, R + 1, 0>(a, h4, M));
    put<ADD>(t.c4[P], T(0.5) * (rho_moment<Q + 2, R, 0>(a, h4, M) + rho_moment<Q, R + 2, 0>(a, h4, M) +
                                rho_moment<Q, R, 1>(a, h4, M)));
}

// functionals of Q = c v^q w^r into entry p
template <bool ADD, int Q, int R, int P, class T>
GKM_HD void tau_mono(Tau<T>& t, T c, const Moments<T>& M)
{
    put<ADD>(t.c0[P], c * mu<Q, R, 0>(M));
    put<ADD>(t.cv[P], c * mu<Q + 1, R, 0>(M));
    put<ADD>(t.cw[P], c * mu<Q, R + 1, 0>(M));
    put<ADD>(t.c4[P], (T(0.5) * c) * (mu<Q + 2, R, 0>(M) + mu<Q, R + 2, 0>(M) + mu<Q, R, 1>(M)));
}

// functionals of psi.a: Q_0 = R(a), Q_1 = a1, Q_2 = a4/2
template <class T>
GKM_HD void tau_psi(Tau<T>& t, const T a[5], const Moments<T>& M)
{
    const T h4 = T(0.5) * a[4];
    tau_R<false, 0, 0, 0>(t, a, h4, M);
    tau_mono<false, 0, 0, 1>(t, a[1], M);
    tau_mono<false, 0, 0, 2>(t, h4, M);
}

// out_i = <u^k psi_i P>_N, P = sum_{p = P0..P1} u^p Q_p
template <int K, int P0, int P1, class T>
GKM_HD void contract(T out[5], const T* N, const Tau<T>& t)
{
    static_assert(P1 + K + 2 <= 6, "normal moment beyond the table");
    T o0 = N[P0 + K] * t.c0[P0];
    T o1 = N[P0 + K + 1] * t.c0[P0];
    T o2 = N[P0 + K] * t.cv[P0];
    T o3 = N[P0 + K] * t.cw[P0];
    T o4 = N[P0 + K] * t.c4[P0] + T(0.5) * N[P0 + K + 2] * t.c0[P0];
#pragma unroll
    for (int p = P0 + 1; p <= P1; p++) {
        o0 += N[p + K] * t.c0[p];
        o1 += N[p + K + 1] * t.c0[p];
        o2 += N[p + K] * t.cv[p];
        o3 += N[p + K] * t.cw[p];
        o4 += N[p + K] * t.c4[p] + T(0.5) * N[p + K + 2] * t.c0[p];
    }
    out[0] = o0;
    out[1] = o1;
    out[2] = o2;
    out[3] = o3;
    out[4] = o4;
}

// Primitive values of a state with the reciprocals the flux reuses: 1/rho,
// lam = rho / (2 p) and 1 / (2 lam) = p / rho.
template <class T>
struct Prim {
    T den, ir, U[3], P, lam, inv2lam;
};

// both face states together, with pd = p rho = (gamma - 1)(E rho - |m|^2 / 2) known before any
// division: 1/rho_l, 1/rho_r, 1/p_l, 1/p_r and 1/(p_l + p_r) (the collision-time ratio) all
// from one reciprocal of rho_l rho_r pd_l pd_r S, S = pd_l rho_r + pd_r rho_l = (p_l + p_r) rho_l rho_r
template <class T>
GKM_HD void prim_pair(const T wl[5], const T wr[5], T gm1, Prim<T>& l, Prim<T>& r, T& inv_psum)
{
    l.den = wl[0];
    r.den = wr[0];
    const T pdl = gm1 * (wl[4] * l.den - T(0.5) * (wl[1] * wl[1] + wl[2] * wl[2] + wl[3] * wl[3]));
    const T pdr = gm1 * (wr[4] * r.den - T(0.5) * (wr[1] * wr[1] + wr[2] * wr[2] + wr[3] * wr[3]));
    const T dd = l.den * r.den, pp = pdl * pdr;
    const T S = pdl * r.den + pdr * l.den;
    const T inv = T(1) / ((dd * pp) * S);
    const T ppS = pp * S * inv;   // 1 / dd
    l.ir = r.den * ppS;
    r.ir = l.den * ppS;
    const T ddS = dd * S * inv;   // 1 / pp
    const T iPl = l.den * (pdr * ddS), iPr = r.den * (pdl * ddS);   // rho / pd
    inv_psum = dd * (dd * pp * inv);
    Prim<T>* st[2] = {&l, &r};
    const T* w[2] = {wl, wr};
    const T pd[2] = {pdl, pdr}, iP[2] = {iPl, iPr};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        Prim<T>& s = *st[k];
        s.U[0] = w[k][1] * s.ir;
        s.U[1] = w[k][2] * s.ir;
        s.U[2] = w[k][3] * s.ir;
        s.P = pd[k] * s.ir;
        s.lam = T(0.5) * s.den * iP[k];
        s.inv2lam = s.P * s.ir;
    }
}

// one state with one division: 1/rho = pd / (rho pd), 1/p = rho^2 / (rho pd)
template <class T>
GKM_HD Prim<T> prim(const T W[5], T gm1)
{
    Prim<T> s;
    s.den = W[0];
    const T pd = gm1 * (W[4] * s.den - T(0.5) * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]));
    const T inv = T(1) / (s.den * pd);
    s.ir = pd * inv;
    s.U[0] = W[1] * s.ir;
    s.U[1] = W[2] * s.ir;
    s.U[2] = W[3] * s.ir;
    s.P = pd * s.ir;
    s.lam = T(0.5) * s.den * (s.den * s.den * inv);
    s.inv2lam = s.P * s.ir;
    return s;
}

// moment tables of a state (build_moments) with sqrt(lam) and 1/sqrt(lam pi) from one
// reciprocal square root
template <class T>
GKM_HD void build_moments_prim(Moments<T>& M, const Prim<T>& st, int K, int half)
{
    const T inv2lam = st.inv2lam, U0 = st.U[0];
    M.Ie2 = T(K) * inv2lam;
    M.Ie4 = T(3 * K + K * (K - 1)) * inv2lam * inv2lam;
    const T isl = rsqrt_t<T>(st.lam);
    const T sl = st.lam * isl;
    const T g = T(0.28209479177387814347) * exp_t<T>(-st.lam * U0 * U0) * isl;   // 1 / (2 sqrt(pi))
    if (half > 0) {
        M.H[0] = T(0.5) * erfc_t<T>(-sl * U0);
        M.H[1] = U0 * M.H[0] + g;
    } else {
        M.H[0] = T(0.5) * erfc_t<T>(sl * U0);
        M.H[1] = U0 * M.H[0] - g;
    }
#pragma unroll
    for (int i = 2; i < 7; i++) M.H[i] = U0 * M.H[i - 1] + M.H[i - 2] * (T(i - 1) * inv2lam);
    full_table<T, 7>(M.X, U0, inv2lam);
    T Y[6], Z[6];
    full_table<T, 6>(Y, st.U[1], inv2lam);
    full_table<T, 6>(Z, st.U[2], inv2lam);
#pragma unroll
    for (int c = 0; c < 6; c++)
#pragma unroll
        for (int b = 0; b + c < 6; b++) M.YZ[yz(b, c)] = Y[b] * Z[c];
}

// slope_state without divisions: (K+3)/(2 lam) = (K+3) inv2lam; iK3 = 1/(K+3)
template <class T>
GKM_HD SlopeState<T> slope_state_prim(const Prim<T>& st, T iK3, int K)
{
    SlopeState<T> s;
    s.U[0] = st.U[0];
    s.U[1] = st.U[1];
    s.U[2] = st.U[2];
    s.lam2 = T(2) * st.lam;
    s.usqc = st.U[0] * st.U[0] + st.U[1] * st.U[1] + st.U[2] * st.U[2] + T(K + 3) * st.inv2lam;
    s.a4fac = T(1.0 / kPrandtl) * (T(4) * st.lam * st.lam) * iK3;
    return s;
}

// The equilibrium part of the flux (src/GKMflux.cpp:73-229 after the two half-Maxwellians):
// the equilibrium state We at the face, its slopes from the cell averages and the tangential
// slopes by_, bz_ the sides gathered, the time derivative from Bacc, and the flux moments added to
// Facc.  gm1..p2 are the time coefficients of src/GKMflux.cpp:162-167,197-204.
template <class T, class Prov>
GKM_HD void gks_equilibrium_part(const Prov& in, const T We[5], const T by_[5], const T bz_[5], T Bacc[5], T Facc[5],
                                 T gm1, T gm2, T gm3, T p0, T p1, T p2, T iK3, T dx, const Phys<T>& ph, T F[5])
{
    const int K = ph.K;
    T M[5];
    const Prim<T> ste = prim<T>(We, ph.gm1);
    const T dene = ste.den;
    Moments<T> E;
    build_moments_prim<T>(E, ste, K, +1);
    // the negative half space of the equilibrium: full table minus the positive half
    T H2[7];
#pragma unroll
    for (int i = 0; i < 7; i++) H2[i] = E.X[i] - E.H[i];
    SlopeState<T> se = slope_state_prim<T>(ste, iK3, K);
    Tau<T> tp;
    T b[5], a[5];
    const T idx2 = (T(2) / dx) * ste.ir;
    // normal equilibrium slopes from the cell averages, src/GKMflux.cpp:115-116
#pragma unroll
    for (int q = 0; q < 5; q++) b[q] = (We[q] - in.WL(q)) * idx2;
    slope_solve<T>(b, se, a);
    tau_psi<T>(tp, a, E);
    contract<1, 0, 2>(M, E.H, tp);
    axpy5<T>(Bacc, gm2 * dene, M);
    contract<2, 0, 2>(M, E.H, tp);
    axpy5<T>(Facc, p2 * dene, M);
#pragma unroll
    for (int q = 0; q < 5; q++) b[q] = (in.WR(q) - We[q]) * idx2;
    slope_solve<T>(b, se, a);
    tau_psi<T>(tp, a, E);
    contract<1, 0, 2>(M, H2, tp);
    axpy5<T>(Bacc, gm2 * dene, M);
    contract<2, 0, 2>(M, H2, tp);
    axpy5<T>(Facc, p2 * dene, M);
    // tangential equilibrium slopes: G_E = v (psi.a_y) + w (psi.a_z),
    //   Q_0 = v R(a_y) + w R(a_z), Q_1 = a1y v + a1z w, Q_2 = (a4y/2) v + (a4z/2) w
    slope_solve<T>(by_, se, a);
    {
        const T h4 = T(0.5) * a[4];
        tau_R<false, 1, 0, 0>(tp, a, h4, E);
        tau_mono<false, 1, 0, 1>(tp, a[1], E);
        tau_mono<false, 1, 0, 2>(tp, h4, E);
    }
    slope_solve<T>(bz_, se, a);
    {
        const T h4 = T(0.5) * a[4];
        tau_R<true, 0, 1, 0>(tp, a, h4, E);
        tau_mono<true, 0, 1, 1>(tp, a[1], E);
        tau_mono<true, 0, 1, 2>(tp, h4, E);
    }
    contract<0, 0, 2>(M, E.X, tp);
    axpy5<T>(Bacc, gm2 * dene, M);
    contract<1, 0, 2>(M, E.X, tp);
    axpy5<T>(Facc, p2 * dene, M);
    // time derivative of the equilibrium, src/GKMflux.cpp:183-191
    mcal0<0, 0, 0, T>(M, E.X, GKM_TABLES(E), E.Ie2);
    const T idene = ste.ir;
#pragma unroll
    for (int q = 0; q < 5; q++) b[q] = (gm1 * dene * M[q] + Bacc[q] + gm3 * We[q]) * idene;
    slope_solve<T>(b, se, a);
    tau_psi<T>(tp, a, E);
    contract<1, 0, 2>(M, E.X, tp);
    axpy5<T>(Facc, p1 * dene, M);
    mcal0<1, 0, 0, T>(M, E.X, GKM_TABLES(E), E.Ie2);
    axpy5<T>(Facc, p0 * dene, M);
#pragma unroll
    for (int q = 0; q < 5; q++) F[q] = Facc[q];
}

// The flux of gks_flux_mcal with the moment functionals above: the same
// moments of the same slope vectors (src/GKMflux.cpp:11-229), grouped per
// polynomial instead of per MCal call.
template <class T, class Prov>
GKM_HD void gks_flux_tau(const Prov& in, T tau0, T dt, T dx, const Phys<T>& ph, T F[5])
{
    const int K = ph.K;
    const T iK3 = T(1) / T(K + 3);
    Prim<T> stl, str;
    T inv_psum;
    {
        T wl[5], wr[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            wl[q] = in.Wl(q);
            wr[q] = in.Wr(q);
        }
        prim_pair<T>(wl, wr, ph.gm1, stl, str, inv_psum);
    }

    // collision time with the pressure-jump correction, src/GKMflux.cpp:156-157:
    // |rho_l/lam_l - rho_r/lam_r| / |rho_l/lam_l + rho_r/lam_r| with rho/lam = 2 p (p > 0)
    const TimeCoefs<wide_t<T>> tc = time_coefs<wide_t<T>, (sizeof(T) < sizeof(wide_t<T>))>(
        wide_t<T>(tau0) + wide_t<T>(dt) * wide_t<T>(fabs(stl.P - str.P) * inv_psum), wide_t<T>(dt));
    const T gm1 = T(tc.gm1), gm2 = T(tc.gm2), gm3 = T(tc.gm3), gm4 = T(tc.gm4), gm5 = T(tc.gm5);
    const T p0 = T(tc.p0), p1 = T(tc.p1), p2 = T(tc.p2), p3 = T(tc.p3), p4 = T(tc.p4), p5 = T(tc.p5);

    T We[5] = {0, 0, 0, 0, 0};      // equilibrium state at the face, src/GKMflux.cpp:73-77
    T by_[5] = {0, 0, 0, 0, 0}, bz_[5] = {0, 0, 0, 0, 0};
    T Bacc[5] = {0, 0, 0, 0, 0};   // B_ * dene, without the gm1/gm3 terms
    T Facc[5] = {0, 0, 0, 0, 0};
    T M[5];

    const T cB = gm4 + gm5;
    // ---------------- one side (l: positive half with left state, r: negative half with right state)
#if GKM_UNROLL_SIDES
#pragma unroll
#else
#pragma unroll 1
#endif
    for (int side = 0; side < 2; side++) {
        const Prim<T>& st = side == 0 ? stl : str;
        const T den = st.den;
        Moments<T> S;
        build_moments_prim<T>(S, st, K, side == 0 ? +1 : -1);
        SlopeState<T> ss = slope_state_prim<T>(st, iK3, K);
        const T iden = st.ir;
        mcal0<0, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2);
        axpy5<T>(We, den, M);
        // G = u (psi.a_n) + v (psi.a_y) + w (psi.a_z):
        //   Q_0 = v R(a_y) + w R(a_z), Q_1 = R(a_n) + a1y v + a1z w,
        //   Q_2 = a1n + (a4y/2) v + (a4z/2) w, Q_3 = a4n/2
        Tau<T> tg, tp;
        T b[5], a[5];
        // normal slope
#pragma unroll
        for (int q = 0; q < 5; q++) b[q] = in.DW(0 + side, q) * iden;
        slope_solve<T>(b, ss, a);
        {
            const T h4 = T(0.5) * a[4];
            tau_R<false, 0, 0, 1>(tg, a, h4, S);
            tau_mono<false, 0, 0, 2>(tg, a[1], S);
            tau_mono<false, 0, 0, 3>(tg, h4, S);
        }
        // first tangential slope: <psi (psi.a_y)>_H feeds the equilibrium's y slope
#pragma unroll
        for (int q = 0; q < 5; q++) b[q] = in.DW(2 + side, q) * iden;
        slope_solve<T>(b, ss, a);
        {
            const T h4 = T(0.5) * a[4];
            tau_psi<T>(tp, a, S);
            contract<0, 0, 2>(M, S.H, tp);
            axpy5<T>(by_, T(1), M);
            tau_R<false, 1, 0, 0>(tg, a, h4, S);
            tau_mono<true, 1, 0, 1>(tg, a[1], S);
            tau_mono<true, 1, 0, 2>(tg, h4, S);
        }
        // second tangential slope
#pragma unroll
        for (int q = 0; q < 5; q++) b[q] = in.DW(4 + side, q) * iden;
        slope_solve<T>(b, ss, a);
        {
            const T h4 = T(0.5) * a[4];
            tau_psi<T>(tp, a, S);
            contract<0, 0, 2>(M, S.H, tp);
            axpy5<T>(bz_, T(1), M);
            tau_R<true, 0, 1, 0>(tg, a, h4, S);
            tau_mono<true, 0, 1, 1>(tg, a[1], S);
            tau_mono<true, 0, 1, 2>(tg, h4, S);
        }
        // -<psi G>_X is the right-hand side of this side's time slope, src/GKMflux.cpp:145-151
        contract<0, 0, 3>(M, S.X, tg);
#pragma unroll
        for (int q = 0; q < 5; q++) b[q] = -M[q];
        contract<0, 0, 3>(M, S.H, tg);
        axpy5<T>(Bacc, cB * den, M);
        contract<1, 0, 3>(M, S.H, tg);
        axpy5<T>(Facc, p4 * den, M);
        // time slope of this side
        slope_solve<T>(b, ss, a);
        tau_psi<T>(tp, a, S);
        contract<0, 0, 2>(M, S.H, tp);
        axpy5<T>(Bacc, gm5 * den, M);
        contract<1, 0, 2>(M, S.H, tp);
        axpy5<T>(Facc, p5 * den, M);
        // free transport of the initial half-Maxwellian
        mcal0<1, 0, 0, T>(M, S.H, GKM_TABLES(S), S.Ie2);
        axpy5<T>(Facc, p3 * den, M);
    }
    gks_equilibrium_part<T>(in, We, by_, bz_, Bacc, Facc, gm1, gm2, gm3, p0, p1, p2, iK3, dx, ph, F);
}

#endif

// The flux the kernels run: the functional form where the tangential product
// table exists (GKM_SHARED_YZ), else the reference's MCal form.
template <class T, class Prov>
GKM_HD void gks_flux(const Prov& in, T tau0, T dt, T dx, const Phys<T>& ph, T F[5])
{
#if GKM_SHARED_YZ
    gks_flux_tau<T>(in, tau0, dt, dx, ph, F);
#else
    gks_flux_mcal<T>(in, tau0, dt, dx, ph, F);
#endif
}

}  // namespace gkm
