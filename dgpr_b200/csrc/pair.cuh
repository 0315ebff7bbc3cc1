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
__host__ __device__ inline f2 operator*(f2 a, f2 b)
{
#ifdef __CUDA_ARCH__
  const float2 r = __fmul2_rn(a.v, b.v);
  return f2(r.x, r.y);
#else
  return f2(a.v.x * b.v.x, a.v.y * b.v.y);
#endif
}
__host__ __device__ inline f2 operator-(f2 a) { return f2(-a.v.x, -a.v.y); }
__host__ __device__ inline f2 operator-(f2 a, f2 b) { return a + (-b); }
__host__ __device__ inline f2 operator/(f2 a, f2 b) { return f2(a.v.x / b.v.x, a.v.y / b.v.y); }
__host__ __device__ inline f2& operator+=(f2& a, f2 b) { return a = a + b; }
__host__ __device__ inline f2& operator-=(f2& a, f2 b) { return a = a - b; }
__host__ __device__ inline f2& operator*=(f2& a, f2 b) { return a = a * b; }
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

// lane-wise: a < b ? x : y
__host__ __device__ inline f2 select_lt(f2 a, f2 b, f2 x, f2 y)
{
  return f2(a.v.x < b.v.x ? x.v.x : y.v.x, a.v.y < b.v.y ? x.v.y : y.v.y);
}
__host__ __device__ inline bool any_lt(f2 a, f2 b) { return a.v.x < b.v.x || a.v.y < b.v.y; }

}  // namespace dgb
