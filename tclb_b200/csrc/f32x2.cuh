// Two FP32 lanes as one value, for the two-nodes-per-thread kernels.
//
// Blackwell (sm_100) issues FP32 add, multiply and fused multiply-add on a
// pair of lanes as one instruction (__fadd2_rn, __fmul2_rn, __ffma2_rn). The
// collision code of the models is written once, templated on its value type;
// instantiated with F2 it updates two nodes per instruction. Each lane is an
// ordinary IEEE FP32 operation with round-to-nearest, as in the scalar code.
//
// Contraction: the scalar code is compiled with FMA contraction, a*b + c
// becoming one fused operation. F2 keeps that: a product is held unevaluated
// (F2Prod) and fused into the add or subtract that consumes it; a product that
// is stored or multiplied again is rounded with one packed multiply.
#pragma once
#include <cuda_runtime.h>

namespace tclb {

struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ F2(float2 x) : v(x) {}
  __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
  // broadcast of a constant or a per-launch scalar
  __device__ __forceinline__ F2(double c) : v(make_float2((float)c, (float)c)) {}
  __device__ __forceinline__ F2(float c) : v(make_float2(c, c)) {}
  __device__ __forceinline__ F2(int c) : v(make_float2((float)c, (float)c)) {}
};

__device__ __forceinline__ float2 neg2(float2 x) { return make_float2(-x.x, -x.y); }

struct F2Prod {
  float2 a, b;
  __device__ __forceinline__ operator F2() const { return F2(__fmul2_rn(a, b)); }
};

__device__ __forceinline__ F2Prod operator*(F2 x, F2 y) { return {x.v, y.v}; }
__device__ __forceinline__ F2Prod operator*(F2Prod p, F2 y) { return {F2(p).v, y.v}; }
__device__ __forceinline__ F2Prod operator*(F2 x, F2Prod p) { return {x.v, F2(p).v}; }
__device__ __forceinline__ F2Prod operator*(F2Prod p, F2Prod q) { return {F2(p).v, F2(q).v}; }

__device__ __forceinline__ F2 operator+(F2 x, F2 y) { return F2(__fadd2_rn(x.v, y.v)); }
__device__ __forceinline__ F2 operator-(F2 x, F2 y) { return F2(__fadd2_rn(x.v, neg2(y.v))); }
__device__ __forceinline__ F2 operator-(F2 x) { return F2(neg2(x.v)); }
__device__ __forceinline__ F2Prod operator-(F2Prod p) { return {neg2(p.a), p.b}; }

__device__ __forceinline__ F2 operator+(F2Prod p, F2 c) { return F2(__ffma2_rn(p.a, p.b, c.v)); }
__device__ __forceinline__ F2 operator+(F2 c, F2Prod p) { return F2(__ffma2_rn(p.a, p.b, c.v)); }
__device__ __forceinline__ F2 operator-(F2Prod p, F2 c) { return F2(__ffma2_rn(p.a, p.b, neg2(c.v))); }
__device__ __forceinline__ F2 operator-(F2 c, F2Prod p) { return F2(__ffma2_rn(neg2(p.a), p.b, c.v)); }
__device__ __forceinline__ F2 operator+(F2Prod p, F2Prod q) { return F2(__ffma2_rn(p.a, p.b, F2(q).v)); }
__device__ __forceinline__ F2 operator-(F2Prod p, F2Prod q) { return F2(__ffma2_rn(p.a, p.b, neg2(F2(q).v))); }

__device__ __forceinline__ F2& operator+=(F2& x, F2 y) { return x = x + y; }
__device__ __forceinline__ F2& operator-=(F2& x, F2 y) { return x = x - y; }
__device__ __forceinline__ F2& operator*=(F2& x, F2 y) { return x = F2(x * y); }
__device__ __forceinline__ F2& operator+=(F2& x, F2Prod p) { return x = p + x; }
__device__ __forceinline__ F2& operator-=(F2& x, F2Prod p) { return x = x - p; }

// 1 / x per lane (IEEE division, as R(1) / x in the scalar code)
__device__ __forceinline__ F2 recip(F2 x) { return F2(1.0f / x.v.x, 1.0f / x.v.y); }
template <class R>
__device__ __forceinline__ R recip(R x) { return R(1) / x; }

}  // namespace tclb
