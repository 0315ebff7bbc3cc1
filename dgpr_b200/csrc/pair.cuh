// f2: two FP32 values of two elements that run in lockstep in one thread,
// with Blackwell's packed FP32x2 arithmetic (__fadd2_rn, __fmul2_rn,
// __ffma2_rn: one instruction for both lanes, each lane rounded as the
// scalar operation).  The templated kernels and pointwise physics take it as
// their compute type T, so a thread computes the same point of two elements
// with one instruction stream.  Comparisons used as branch conditions are
// for values both lanes share (mu, kq); lane-dependent choices go through
// select() (the Roe entropy fix).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <type_traits>

// Products are kept unrounded (f2mul) until they meet an addition, which
// then becomes one __ffma2_rn: `a * b + c` contracts into a fused
// multiply-add as the scalar compiler does for float.  Anywhere else an
// f2mul rounds to f2 (one __fmul2_rn).  DGB_PAIR_CONTRACT 0 keeps every
// product rounded.
#ifndef DGB_PAIR_CONTRACT
#define DGB_PAIR_CONTRACT 1
#endif

namespace dgb {

// the scalar overloads stay visible beside the f2 ones declared below
using ::fabs;
using ::fma;
using ::sqrt;

struct f2 {
  float2 v;
  f2() = default;
  __host__ __device__ constexpr f2(float a, float b) : v{a, b} {}
  __host__ __device__ constexpr explicit f2(float a) : v{a, a} {}
  __host__ __device__ constexpr explicit f2(double a) : v{(float)a, (float)a} {}
  __host__ __device__ constexpr explicit f2(int a) : v{(float)a, (float)a} {}
  __host__ __device__ float lane(int l) const { return l ? v.y : v.x; }
};

template <class T>
struct is_pair : std::false_type {};
template <>
struct is_pair<f2> : std::true_type {};

__host__ __device__ inline f2 operator+(f2 a, f2 b)
{
#ifdef __CUDA_ARCH__
  const float2 r = __fadd2_rn(a.v, b.v);
  return f2(r.x, r.y);
#else
  return f2(a.v.x + b.v.x, a.v.y + b.v.y);
#endif
}
#if DGB_PAIR_CONTRACT
struct f2mul;
__host__ __device__ inline f2mul operator*(f2 a, f2 b);
#else
__host__ __device__ inline f2 operator*(f2 a, f2 b)
{
#ifdef __CUDA_ARCH__
  const float2 r = __fmul2_rn(a.v, b.v);
  return f2(r.x, r.y);
#else
  return f2(a.v.x * b.v.x, a.v.y * b.v.y);
#endif
}
#endif
__host__ __device__ inline f2 operator-(f2 a) { return f2(-a.v.x, -a.v.y); }
__host__ __device__ inline f2 operator-(f2 a, f2 b) { return a + (-b); }
__host__ __device__ inline f2 operator/(f2 a, f2 b) { return f2(a.v.x / b.v.x, a.v.y / b.v.y); }
__host__ __device__ inline f2& operator+=(f2& a, f2 b) { return a = a + b; }
__host__ __device__ inline f2& operator-=(f2& a, f2 b) { return a = a - b; }
__host__ __device__ inline f2& operator*=(f2& a, f2 b)
{
#ifdef __CUDA_ARCH__
  const float2 r = __fmul2_rn(a.v, b.v);
  return a = f2(r.x, r.y);
#else
  return a = f2(a.v.x * b.v.x, a.v.y * b.v.y);
#endif
}
// branch conditions on values both lanes share
__host__ __device__ inline bool operator!=(f2 a, f2 b) { return a.v.x != b.v.x || a.v.y != b.v.y; }
__host__ __device__ inline bool operator==(f2 a, f2 b) { return !(a != b); }

__host__ __device__ inline f2 fma(f2 a, f2 b, f2 c)
{
#ifdef __CUDA_ARCH__
  const float2 r = __ffma2_rn(a.v, b.v, c.v);
  return f2(r.x, r.y);
#else
  return f2(a.v.x * b.v.x + c.v.x, a.v.y * b.v.y + c.v.y);
#endif
}
__host__ __device__ inline f2 sqrt(f2 a) { return f2(sqrtf(a.v.x), sqrtf(a.v.y)); }
__host__ __device__ inline f2 fabs(f2 a) { return f2(fabsf(a.v.x), fabsf(a.v.y)); }

#if DGB_PAIR_CONTRACT
struct f2mul {
  f2 a, b;
  __host__ __device__ operator f2() const
  {
#ifdef __CUDA_ARCH__
    const float2 r = __fmul2_rn(a.v, b.v);
    return f2(r.x, r.y);
#else
    return f2(a.v.x * b.v.x, a.v.y * b.v.y);
#endif
  }
};
__host__ __device__ inline f2mul operator*(f2 a, f2 b) { return f2mul{a, b}; }
__host__ __device__ inline f2 operator+(f2mul p, f2 c) { return fma(p.a, p.b, c); }
__host__ __device__ inline f2 operator+(f2 c, f2mul p) { return fma(p.a, p.b, c); }
__host__ __device__ inline f2 operator+(f2mul p, f2mul q) { return fma(p.a, p.b, f2(q)); }
__host__ __device__ inline f2 operator-(f2mul p, f2 c) { return fma(p.a, p.b, -c); }
__host__ __device__ inline f2 operator-(f2 c, f2mul p) { return fma(-p.a, p.b, c); }
__host__ __device__ inline f2 operator-(f2mul p, f2mul q) { return fma(p.a, p.b, -f2(q)); }
__host__ __device__ inline f2mul operator-(f2mul p) { return f2mul{-p.a, p.b}; }
__host__ __device__ inline f2mul operator*(f2mul p, f2 c) { return f2mul{f2(p), c}; }
__host__ __device__ inline f2mul operator*(f2 c, f2mul p) { return f2mul{c, f2(p)}; }
__host__ __device__ inline f2mul operator*(f2mul p, f2mul q) { return f2mul{f2(p), f2(q)}; }
__host__ __device__ inline f2 operator/(f2mul p, f2 c) { return f2(p) / c; }
__host__ __device__ inline f2 operator/(f2 c, f2mul p) { return c / f2(p); }
__host__ __device__ inline f2 operator/(f2mul p, f2mul q) { return f2(p) / f2(q); }
__host__ __device__ inline f2& operator+=(f2& a, f2mul p) { return a = fma(p.a, p.b, a); }
__host__ __device__ inline f2& operator-=(f2& a, f2mul p) { return a = fma(-p.a, p.b, a); }
__host__ __device__ inline f2& operator*=(f2& a, f2mul p) { return a *= f2(p); }
__host__ __device__ inline f2 sqrt(f2mul a) { return sqrt(f2(a)); }
__host__ __device__ inline f2 fabs(f2mul a) { return fabs(f2(a)); }
#endif

// lane-wise: a < b ? x : y
__host__ __device__ inline f2 select_lt(f2 a, f2 b, f2 x, f2 y)
{
  return f2(a.v.x < b.v.x ? x.v.x : y.v.x, a.v.y < b.v.y ? x.v.y : y.v.y);
}
__host__ __device__ inline bool any_lt(f2 a, f2 b) { return a.v.x < b.v.x || a.v.y < b.v.y; }

}  // namespace dgb
