// Packed single precision for sm_100a: a pair of FP32 values in one register
// pair, added, multiplied or fused-multiply-added by one instruction
// (add/mul/fma .rn.f32x2).  The mixed-precision sweeps are issue-bound, so
// evaluating two independent lanes of the same arithmetic per instruction (two
// WENO scalars of a cell, both sides' face energies) frees issue slots; each
// lane is rounded as the scalar operation would be.
//
// F2 works in the templated numerics (gkm_numerics.cuh) like a scalar: a * b
// yields an F2Mul that stays unevaluated until it is added (one fma.f32x2, as
// the compiler contracts a * b + c for scalars) or used as an F2 (one mul.f32x2).
// Division, square roots and the special functions act on each lane.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace gkm {

struct F2Mul;

struct F2 {
    float2 v;
    __device__ __forceinline__ F2() {}
    // both lanes the same value; explicit, so that a scalar never turns into a pair unasked
    __device__ __forceinline__ explicit F2(float a) : v(make_float2(a, a)) {}
    __device__ __forceinline__ explicit F2(double a) : v(make_float2((float)a, (float)a)) {}
    __device__ __forceinline__ explicit F2(int a) : v(make_float2((float)a, (float)a)) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ F2(float2 x) : v(x) {}
    __device__ __forceinline__ F2(const F2Mul& m);
    __device__ __forceinline__ float lo() const { return v.x; }
    __device__ __forceinline__ float hi() const { return v.y; }
    // lane by lane; friends found through their F2 arguments only, so they hide no scalar fmax / fabs
    friend __device__ __forceinline__ F2 fmax(F2 x, F2 y) { return F2(fmaxf(x.v.x, y.v.x), fmaxf(x.v.y, y.v.y)); }
    friend __device__ __forceinline__ F2 fabs(F2 x) { return F2(fabsf(x.v.x), fabsf(x.v.y)); }
};

// a product not yet rounded: becomes one fma.f32x2 when added, one mul.f32x2 otherwise
struct F2Mul {
    float2 a, b;
};

__device__ __forceinline__ float2 neg2(float2 x) { return make_float2(-x.x, -x.y); }
__device__ __forceinline__ F2::F2(const F2Mul& m) : v(__fmul2_rn(m.a, m.b)) {}

__device__ __forceinline__ F2Mul operator*(F2 x, F2 y) { return {x.v, y.v}; }
__device__ __forceinline__ F2Mul operator*(const F2Mul& m, F2 y) { return {__fmul2_rn(m.a, m.b), y.v}; }
__device__ __forceinline__ F2Mul operator*(F2 y, const F2Mul& m) { return {y.v, __fmul2_rn(m.a, m.b)}; }
__device__ __forceinline__ F2Mul operator*(const F2Mul& m, const F2Mul& n)
{
    return {__fmul2_rn(m.a, m.b), __fmul2_rn(n.a, n.b)};
}

__device__ __forceinline__ F2 operator+(F2 x, F2 y) { return F2(__fadd2_rn(x.v, y.v)); }
__device__ __forceinline__ F2 operator-(F2 x, F2 y) { return F2(__fadd2_rn(x.v, neg2(y.v))); }
__device__ __forceinline__ F2 operator-(F2 x) { return F2(neg2(x.v)); }
__device__ __forceinline__ F2Mul operator-(const F2Mul& m) { return {neg2(m.a), m.b}; }

__device__ __forceinline__ F2 operator+(const F2Mul& m, F2 c) { return F2(__ffma2_rn(m.a, m.b, c.v)); }
__device__ __forceinline__ F2 operator+(F2 c, const F2Mul& m) { return F2(__ffma2_rn(m.a, m.b, c.v)); }
__device__ __forceinline__ F2 operator-(const F2Mul& m, F2 c) { return F2(__ffma2_rn(m.a, m.b, neg2(c.v))); }
__device__ __forceinline__ F2 operator-(F2 c, const F2Mul& m) { return F2(__ffma2_rn(neg2(m.a), m.b, c.v)); }
__device__ __forceinline__ F2 operator+(const F2Mul& m, const F2Mul& n)
{
    return F2(__ffma2_rn(m.a, m.b, __fmul2_rn(n.a, n.b)));
}
__device__ __forceinline__ F2 operator-(const F2Mul& m, const F2Mul& n)
{
    return F2(__ffma2_rn(m.a, m.b, neg2(__fmul2_rn(n.a, n.b))));
}

__device__ __forceinline__ F2& operator+=(F2& x, F2 y) { return x = x + y; }
__device__ __forceinline__ F2& operator+=(F2& x, const F2Mul& m) { return x = m + x; }
__device__ __forceinline__ F2& operator-=(F2& x, F2 y) { return x = x - y; }
__device__ __forceinline__ F2& operator-=(F2& x, const F2Mul& m) { return x = x - m; }
__device__ __forceinline__ F2& operator*=(F2& x, F2 y) { return x = F2(x * y); }

// lane by lane
__device__ __forceinline__ F2 operator/(F2 x, F2 y) { return F2(x.v.x / y.v.x, x.v.y / y.v.y); }

}  // namespace gkm
