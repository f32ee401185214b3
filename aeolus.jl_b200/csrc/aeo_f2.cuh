// aeo_f2.cuh -- two FP32 lanes computed by the paired FP32 instructions of
// sm_100 (__fadd2_rn, __fmul2_rn, __ffma2_rn: one instruction for both lanes).
//
// F2 is the value type of the paired sweep: every stencil expression of the
// scalar code runs unchanged on two x-adjacent cells.  A product is kept
// unevaluated (F2M) until it meets a sum or a difference, which then issues
// one fused multiply-add, as the compiler contracts the scalar code; a product
// that is stored or multiplied again is rounded there.
#pragma once

#include <cuda_runtime.h>

__device__ __forceinline__ float2 f2neg(float2 x) { return make_float2(-x.x, -x.y); }

struct F2 {
    float2 v;
    F2() = default;
    __device__ __forceinline__ F2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ explicit F2(double s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ explicit F2(int s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
};

// a product a*b not yet rounded
struct F2M {
    float2 a, b;
    __device__ __forceinline__ operator F2() const { return F2(__fmul2_rn(a, b)); }
};

__device__ __forceinline__ F2 operator+(F2 x, F2 y) { return F2(__fadd2_rn(x.v, y.v)); }
__device__ __forceinline__ F2 operator-(F2 x, F2 y) { return F2(__fadd2_rn(x.v, f2neg(y.v))); }
__device__ __forceinline__ F2 operator-(F2 x) { return F2(f2neg(x.v)); }

__device__ __forceinline__ F2M operator*(F2 x, F2 y) { return F2M{x.v, y.v}; }
__device__ __forceinline__ F2M operator*(F2M m, F2 y) { return F2M{__fmul2_rn(m.a, m.b), y.v}; }
__device__ __forceinline__ F2M operator*(F2 y, F2M m) { return F2M{y.v, __fmul2_rn(m.a, m.b)}; }
__device__ __forceinline__ F2M operator*(F2M m, F2M n) { return F2M{__fmul2_rn(m.a, m.b), __fmul2_rn(n.a, n.b)}; }
__device__ __forceinline__ F2M operator-(F2M m) { return F2M{f2neg(m.a), m.b}; }

__device__ __forceinline__ F2 operator+(F2M m, F2 c) { return F2(__ffma2_rn(m.a, m.b, c.v)); }
__device__ __forceinline__ F2 operator+(F2 c, F2M m) { return F2(__ffma2_rn(m.a, m.b, c.v)); }
__device__ __forceinline__ F2 operator-(F2M m, F2 c) { return F2(__ffma2_rn(m.a, m.b, f2neg(c.v))); }
__device__ __forceinline__ F2 operator-(F2 c, F2M m) { return F2(__ffma2_rn(f2neg(m.a), m.b, c.v)); }
__device__ __forceinline__ F2 operator+(F2M m, F2M n) { return F2(__ffma2_rn(m.a, m.b, __fmul2_rn(n.a, n.b))); }
__device__ __forceinline__ F2 operator-(F2M m, F2M n) { return F2(__ffma2_rn(m.a, m.b, f2neg(__fmul2_rn(n.a, n.b)))); }

__device__ __forceinline__ F2& operator+=(F2& x, F2 y) { return x = x + y; }
__device__ __forceinline__ F2& operator+=(F2& x, F2M y) { return x = x + y; }
__device__ __forceinline__ F2& operator-=(F2& x, F2 y) { return x = x - y; }
__device__ __forceinline__ F2& operator-=(F2& x, F2M y) { return x = x - y; }

__device__ __forceinline__ F2 sqrt(F2 x) { return F2(sqrtf(x.v.x), sqrtf(x.v.y)); }

// c sqrt(b / a) where a > 0, else 0, lane by lane
__device__ __forceinline__ F2 sqrt_ratio_or_zero(F2 b, F2 a, float c) {
    return F2(a.v.x > 0.f ? c * sqrtf(b.v.x / a.v.x) : 0.f, a.v.y > 0.f ? c * sqrtf(b.v.y / a.v.y) : 0.f);
}

// the FP32 RK3 stage combination x + ca*(s - x) on a pair (rk_combine of
// aeo_common.cuh: weights that sum to one exactly)
__device__ __forceinline__ F2 rk_combine(float ca, float, F2 s, F2 x) { return x + F2(ca) * (s - x); }
