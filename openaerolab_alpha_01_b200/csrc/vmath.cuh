// vmath.cuh — one arithmetic vocabulary for three lane types: float, double and F2 (two float
// lanes in a 64-bit register, operated on with sm_100a's packed f32x2 instructions). Collision
// code written once against these helpers runs one cell per thread (float, double) or two cells
// per thread (F2) with the same operation sequence per lane. The library is compiled with
// -fmad=false, so the scalar forms fuse only the multiply-adds written explicitly; ptxas may still
// contract a packed multiply and the packed add that consumes it into one packed FMA, so the F2
// form agrees with the scalar forms to rounding, not bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace oal {

struct F2 {
  unsigned long long v;
};

__device__ __forceinline__ F2 f2(float a, float b) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2split(F2 r, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r.v)); }
__device__ __forceinline__ float f2lo(F2 r) { float a, b; f2split(r, a, b); return a; }
__device__ __forceinline__ float f2hi(F2 r) { float a, b; f2split(r, a, b); return b; }

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { F2 r; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { F2 r; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { F2 r; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 operator-(F2 a) { return f2(-f2lo(a), -f2hi(a)); }
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { a = a + b; return a; }

// ---- lane-type traits ------------------------------------------------------------------------
template <class V> struct Lane;
template <> struct Lane<float> { using S = float; static constexpr int N = 1; };
template <> struct Lane<double> { using S = double; static constexpr int N = 1; };
template <> struct Lane<F2> { using S = float; static constexpr int N = 2; };

template <class V> __device__ __forceinline__ V splat(typename Lane<V>::S c);
template <> __device__ __forceinline__ float splat<float>(float c) { return c; }
template <> __device__ __forceinline__ double splat<double>(double c) { return c; }
template <> __device__ __forceinline__ F2 splat<F2>(float c) { return f2(c, c); }

// fused multiply-add a*b + c, round to nearest
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double vfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ F2 vfma(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double vmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ F2 vmax(F2 a, F2 b) { return f2(fmaxf(f2lo(a), f2lo(b)), fmaxf(f2hi(a), f2hi(b))); }
__device__ __forceinline__ float vmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double vmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ F2 vmin(F2 a, F2 b) { return f2(fminf(f2lo(a), f2lo(b)), fminf(f2hi(a), f2hi(b))); }

// reciprocal and square root: single-instruction approximations in float (<= 2 ulp), exact in double
__device__ __forceinline__ float frcp(float x) { float r; asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
__device__ __forceinline__ float fsqrt(float x) { float r; asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
__device__ __forceinline__ float vrcp(float x) { return frcp(x); }
__device__ __forceinline__ double vrcp(double x) { return 1.0 / x; }
__device__ __forceinline__ F2 vrcp(F2 x) { return f2(frcp(f2lo(x)), frcp(f2hi(x))); }
__device__ __forceinline__ float vsqrt(float x) { return fsqrt(x); }
__device__ __forceinline__ double vsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ F2 vsqrt(F2 x) { return f2(fsqrt(f2lo(x)), fsqrt(f2hi(x))); }

// per-lane select: (a > b) ? x : y
__device__ __forceinline__ float vsel_gt(float a, float b, float x, float y) { return a > b ? x : y; }
__device__ __forceinline__ double vsel_gt(double a, double b, double x, double y) { return a > b ? x : y; }
__device__ __forceinline__ F2 vsel_gt(F2 a, F2 b, F2 x, F2 y) {
  return f2(f2lo(a) > f2lo(b) ? f2lo(x) : f2lo(y), f2hi(a) > f2hi(b) ? f2hi(x) : f2hi(y));
}
// clamp to [lo, hi] per lane (lo <= hi assumed), NaN-propagating like the reference's clamp
__device__ __forceinline__ float vclamp(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ double vclamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ F2 vclamp(F2 v, F2 lo, F2 hi) {
  return f2(vclamp(f2lo(v), f2lo(lo), f2lo(hi)), vclamp(f2hi(v), f2hi(lo), f2hi(hi)));
}
// max(v, c) with the reference's NaN behaviour of Julia max (NaN wins)
__device__ __forceinline__ float vmaxc(float v, float c) { return v > c ? v : (v != v ? v : c); }
__device__ __forceinline__ double vmaxc(double v, double c) { return v > c ? v : (v != v ? v : c); }
__device__ __forceinline__ F2 vmaxc(F2 v, float c) { return f2(vmaxc(f2lo(v), c), vmaxc(f2hi(v), c)); }

// any lane true
__device__ __forceinline__ bool vany_gt(float a, float b) { return a > b; }
__device__ __forceinline__ bool vany_gt(double a, double b) { return a > b; }
__device__ __forceinline__ bool vany_gt(F2 a, F2 b) { return f2lo(a) > f2lo(b) || f2hi(a) > f2hi(b); }

}  // namespace oal
