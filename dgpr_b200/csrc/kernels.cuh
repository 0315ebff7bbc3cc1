// Residual / RK-stage kernels for affine hexahedral elements, templated on the
// polynomial size P = p + 1 and on the compute type T of the residual:
//   T = double : the plain FP64 form
//   T = float  : the mixed form -- contractions, traces and the pointwise
//                Roe / viscous fluxes in FP32; the inverse mass matrix, the RK
//                update and the state in HBM stay FP64
//
// One CTA per element.  The tensor-product structure of the basis (equispaced
// Lagrange, basis.cpp:64-170) and of the quadrature (P Gauss points per
// direction, geometry_common.cpp:176-177) is used throughout: every
// interpolation / projection is a sequence of 1D P x P contractions on
// shared-memory element tiles (sum factorisation), never the dense nb x nqv
// tables the reference streams from HBM.
//
// Pipeline (state layout U[e][r][b], the reference's):
//   trace_kernel : U -> face traces T[e][lf][10][P*P] (5 conserved values and
//                  the viscous normal flux A(U, grad U).n_out at every face
//                  quadrature point); once per dgb_step call
//   stage_kernel : U_s, T_s -> R (volume + source + faces), f = -Minv R, the
//                  RK update U_{s+1}, and in its epilogue the traces T_{s+1}
//                  of U_{s+1} for the next stage; one launch per RK stage
// The face kernel of the reference (solve.cpp:393-794) is folded into the
// stage kernel: each element evaluates its own six faces from its own traces
// and its neighbours' traces, so no per-face residual slots are written
// (the reference's FACERESID gather, solve_cuda.cu:1192-1210).
#pragma once

#include <cuda_runtime.h>

#include "kernels.hpp"
#include "physics.cuh"

#ifndef DGB_STAGE_REGS
#define DGB_STAGE_REGS 96
#endif
#ifndef DGB_STAGE_REGS_F32
#define DGB_STAGE_REGS_F32 64
#endif
// faces the stage and trace kernels process per pass: 3 (two passes; measured
// faster at p = 3) or 6 (one pass, 6 P^2 threads busy)
#ifndef DGB_FACES_PER_PASS
#define DGB_FACES_PER_PASS 3
#endif
// L2 prefetch, at the start of each stage CTA, of the face traces (own and
// neighbours') and RK operands it reads later
#ifndef DGB_PREFETCH_L2
#define DGB_PREFETCH_L2 1
#endif

namespace dgb {

// ------------------------------------------------------------ configuration

template <int P>
struct Cfg {
  static constexpr int NB = P * P * P;  // nodes = volume quadrature points
  static constexpr int NQF = P * P;     // face quadrature points
  static constexpr int NH = 3 * NQF;    // face points of half an element (3 faces)
  static constexpr int NT = (((NB > NH ? NB : NH) + 31) / 32) * 32;
  // stage and trace kernels: FPP faces per pass (all six, or three at a time)
  static constexpr int FPP = DGB_FACES_PER_PASS;
  static constexpr int NF = FPP * NQF;
  static constexpr int NTS = (((NB > NF ? NB : NF) + 31) / 32) * 32;
  // operator table: B Bd Dq M1i Bi (P*P each), E0 E1 D0 D1 Wb w (P each), cend[2],
  // EL0 EL1 DL0 DL1 (P each: value / derivative at xi = 0, 1 of the Lagrange
  // polynomials through the Gauss points, for the Gauss-point stage kernel)
  static constexpr int oB = 0, oBd = P * P, oDq = 2 * P * P, oMi = 3 * P * P, oBi = 4 * P * P;
  static constexpr int oE = 5 * P * P, oD = oE + 2 * P, oWb = oD + 2 * P, oW = oWb + P;
  static constexpr int oC = oW + P;
  static constexpr int oEh = oC + 2, oDh = oEh + 2 * P;
  static constexpr int OPS = oDh + 2 * P;
};

constexpr int align16(int bytes) { return (bytes + 15) & ~15; }

// Resident CTAs per SM the stage kernel is compiled for: caps registers at
// about DGB_STAGE_REGS (FP64) / DGB_STAGE_REGS_F32 (FP32) per thread so
// occupancy is not register-limited.
template <int P, class T>
struct MinBlocks {
  static constexpr int REGS = sizeof(T) == 8 ? DGB_STAGE_REGS : DGB_STAGE_REGS_F32;
  static constexpr int RAW = 65536 / (Cfg<P>::NTS * REGS);
  static constexpr int value = RAW < 1 ? 1 : (RAW > 16 ? 16 : RAW);
};

// ------------------------------------------------------------ L2 prefetch

__device__ __forceinline__ void prefetch_l2(const void* p)
{
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// every 128-byte line of [p, p + bytes), spread over the CTA's threads
__device__ __forceinline__ void prefetch_range(const void* p, long bytes, int first, int stride)
{
  const char* c = reinterpret_cast<const char*>(p);
  for (long o = (long)first * 128; o < bytes; o += (long)stride * 128) prefetch_l2(c + o);
}

// ------------------------------------------------------------ strided loads

// Entries [0, N) of an FP64 array spread over NT threads (thread t takes
// t, t + NT, ...), loaded into registers with all the loads in flight
// together, for the caller to store afterwards: a loop that stores each
// entry before it loads the next has the loads wait one after another.
template <int N, int NT>
__device__ __forceinline__ void load_spread(const double* __restrict__ src, int t, double (&v)[(N + NT - 1) / NT])
{
#pragma unroll
  for (int k = 0; k < (N + NT - 1) / NT; ++k) {
    const int i = t + k * NT;
    v[k] = i < N ? src[i] : 0.;
  }
}

// ------------------------------------------------------------ index helpers

// node index from the coordinate along face axis a and the two tangential
// coordinates (t1 < t2 in axis order: x faces (y,z), y faces (x,z), z faces (x,y))
template <int P>
__device__ __forceinline__ int face_node(int a, int ia, int t1, int t2)
{
  return a == 0 ? ia + P * (t1 + P * t2) : a == 1 ? t1 + P * (ia + P * t2) : t1 + P * (t2 + P * ia);
}

// P consecutive values from shared memory p[0..P-1] (p aligned to P values):
// 16-byte vector loads for FP64 lines of even length, so a line costs P/2
// load instructions instead of P.  (FP32 lines stay scalar: float4 loads
// measured 1.7% slower in the mixed stage kernel, which then spills.)
template <int P, class T>
__device__ __forceinline__ void load_line(const T* p, T* v)
{
  if constexpr (std::is_same<T, double>::value && P % 2 == 0) {
#pragma unroll
    for (int k = 0; k < P; k += 2) {
      const double2 q = *reinterpret_cast<const double2*>(p + k);
      v[k] = q.x;
      v[k + 1] = q.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < P; ++k) v[k] = p[k];
  }
}

// one output point o of a 1D contraction along axis AX for all 5 variables:
//   out[r][o] (+)= scale * sum_k M(a, k) in[r][o with coordinate AX replaced by k]
// M(a,k) = Mat[a*P+k], or Mat[k*P+a] when TR.  Along x (AX = 0) the P inputs
// of a line are contiguous and aligned, as is an operator row when !TR.
template <int P, int AX, bool TR, bool ACC, class T>
__device__ __forceinline__ void contract(const T* __restrict__ Mat, const T* in, T* out, int o,
                                         T scale = T(1))
{
  constexpr int NB = P * P * P;
  constexpr int S = AX == 0 ? 1 : (AX == 1 ? P : P * P);
  const int a = (o / S) % P;
  const int base = o - a * S;
  T m[P];
  if constexpr (!TR && std::is_same<T, double>::value && P % 2 == 0) {
    load_line<P>(Mat + a * P, m);
  } else {
#pragma unroll
    for (int k = 0; k < P; ++k) m[k] = TR ? Mat[k * P + a] : Mat[a * P + k];
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    T s = T(0);
    if constexpr (AX == 0 && std::is_same<T, double>::value && P % 2 == 0) {
      T x[P];
      load_line<P>(in + r * NB + base, x);
#pragma unroll
      for (int k = 0; k < P; ++k) s = fma(m[k], x[k], s);
    } else {
#pragma unroll
      for (int k = 0; k < P; ++k) s = fma(m[k], in[r * NB + base + k * S], s);
    }
    s *= scale;
    out[r * NB + o] = ACC ? out[r * NB + o] + s : s;
  }
}

// same, result returned in registers
template <int P, int AX, bool TR, class T>
__device__ __forceinline__ void contract_reg(const T* __restrict__ Mat, const T* in, int o, T* res)
{
  constexpr int NB = P * P * P;
  constexpr int S = AX == 0 ? 1 : (AX == 1 ? P : P * P);
  const int a = (o / S) % P;
  const int base = o - a * S;
  T m[P];
  if constexpr (!TR && std::is_same<T, double>::value && P % 2 == 0) {
    load_line<P>(Mat + a * P, m);
  } else {
#pragma unroll
    for (int k = 0; k < P; ++k) m[k] = TR ? Mat[k * P + a] : Mat[a * P + k];
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    T s = T(0);
    if constexpr (AX == 0 && std::is_same<T, double>::value && P % 2 == 0) {
      T x[P];
      load_line<P>(in + r * NB + base, x);
#pragma unroll
      for (int k = 0; k < P; ++k) s = fma(m[k], x[k], s);
    } else {
#pragma unroll
      for (int k = 0; k < P; ++k) s = fma(m[k], in[r * NB + base + k * S], s);
    }
    res[r] = s;
  }
}

// Dual-consistency test coefficients of one face point: with
// dc = A(S, d n^T) (solve.cpp:509-546, 720-741) the face term -grad(phi) . dc fJ w
// becomes sum_i d(phi)/d(xi_i) b_i with b_i = -fw sum_c Jinv[i][c] dc[c].
// Written for variables 1..4 (dc has no mass component): fb[(i*4 + r-1)*stride].
template <class T>
__device__ __forceinline__ void dual_consistency_ref(const T* S, const T* d, const T* n, T mu, const T* Ji,
                                                     T fw, T* fb, int stride, T kq)
{
  const T lam = -(T(2) / T(3)) * mu;
  const T ir = T(1) / S[0];
  const T vel[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  T a[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) a[i] = (d[1 + i] - d[0] * vel[i]) * ir;
  const T an = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
  T tau[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) tau[k][c] = mu * (a[k] * n[c] + a[c] * n[k]) + (k == c ? lam * an : T(0));
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    T en = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T m = Ji[3 * i] * tau[k][0] + Ji[3 * i + 1] * tau[k][1] + Ji[3 * i + 2] * tau[k][2];
      fb[(i * 4 + k) * stride] = -fw * m;
      en += vel[k] * m;
    }
    fb[(i * 4 + 3) * stride] = -fw * en;
  }
  if (kq != T(0)) {  // the heat flux kq Y(d) n of the energy row
    const T h = kq * heat_y(S, d);
#pragma unroll
    for (int i = 0; i < 3; ++i)
      fb[(i * 4 + 3) * stride] -= fw * h * (Ji[3 * i] * n[0] + Ji[3 * i + 1] * n[1] + Ji[3 * i + 2] * n[2]);
  }
}

// ------------------------------------------------------------- face traces

// The trace of one face point: the 5 values S and A(S, grad S).n_out from
// the reference-space gradient g[c][r] = dS_r/dxi_c, into Te[(lf*10 + r)*NQF + fq].
template <int P, class T, bool CV>
__device__ __forceinline__ void trace_point_store(int lf, int fq, const T* S, const T (*g)[5], const T* sg,
                                                  const double* __restrict__ gfe, T mu, T kq,
                                                  T* __restrict__ Te)
{
  constexpr int NQF = P * P;
  T Qn[5] = {T(0), T(0), T(0), T(0), T(0)};
  if (mu != T(0)) {
    T Ji[9], n[3];
    if constexpr (CV) {
      const double* gp = gfe + lf * kFaceC * NQF + fq;
#pragma unroll
      for (int c = 0; c < 9; ++c) Ji[c] = T(gp[c * NQF]);
#pragma unroll
      for (int c = 0; c < 3; ++c) n[c] = T(gp[(kFaceN + c) * NQF]);
    } else {
#pragma unroll
      for (int c = 0; c < 9; ++c) Ji[c] = sg[kGeoJinv + c];
#pragma unroll
      for (int c = 0; c < 3; ++c) n[c] = sg[kGeoN + 3 * lf + c];
    }
    T G[3][5], Q[3][5];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 5; ++r) G[c][r] = Ji[c] * g[0][r] + Ji[3 + c] * g[1][r] + Ji[6 + c] * g[2][r];
    visc_flux(S, G, mu, Q, kq);
#pragma unroll
    for (int r = 0; r < 5; ++r) Qn[r] = Q[0][r] * n[0] + Q[1][r] * n[1] + Q[2][r] * n[2];
  }
  T* Tq = Te + lf * 10 * NQF;
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    Tq[r * NQF + fq] = S[r];
    Tq[(5 + r) * NQF + fq] = Qn[r];
  }
}

// Traces of a nodal state sUx[5][NB] (shared memory) on the FPP faces
// lf = FPP*half + j, j < FPP: at every face quadrature point the 5 conserved values
// and the viscous normal flux A(U, grad U).n_out, written to
// Te[(lf*10 + r)*NQF + fq] (Te = this element's slice of the trace buffer).
// Threads tid < 3*NQF each own one face point.  Scratch: sN[3][10][NQF],
// sY[3][15][NQF].  Both the trace kernel and the stage kernel's epilogue call
// this, so a trace is bit-identical whichever of them produced it.
// sg: element geometry record in T (Jinv, detJ, normals, surface Jacobians).
// CV (curved elements): the inverse Jacobian and normal of each face point
// come from gfe, this element's per-point face geometry [6][kFaceC][P*P].
template <int P, class T, bool CV>
__device__ __forceinline__ void trace_half(int half, const T* sUx, T* sN, T* sY, const T* so, const T* sg,
                                           T mu, T kq, T* __restrict__ Te, const double* __restrict__ gfe)
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NF, FPP = C::FPP;
  const int tid = threadIdx.x;
  const T* B = so + C::oB;
  const T* Bd = so + C::oBd;
  if (tid < NH) {  // along the face normal: value and normal derivative
    const int j = tid / NQF, lf = FPP * half + j, fq = tid % NQF, t1 = fq % P, t2 = fq / P;
    const int a = lf >> 1, end = lf & 1;
    const T* Ev = so + C::oE + end * P;
    const T* Dv = so + C::oD + end * P;
    T* out = sN + j * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      T v = T(0), dn = T(0);
#pragma unroll
      for (int ia = 0; ia < P; ++ia) {
        const T u = sUx[r * NB + face_node<P>(a, ia, t1, t2)];
        v = fma(Ev[ia], u, v);
        dn = fma(Dv[ia], u, dn);
      }
      out[r * NQF + fq] = v;
      out[(5 + r) * NQF + fq] = dn;
    }
  }
  __syncthreads();
  if (tid < NH) {  // first tangential direction (index q1 = fq % P)
    const int j = tid / NQF, fq = tid % NQF, q1 = fq % P, t2 = fq / P;
    const T* in = sN + j * 10 * NQF;
    T* out = sY + j * 15 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      T yv = T(0), yd = T(0), yn = T(0);
#pragma unroll
      for (int t1 = 0; t1 < P; ++t1) {
        const T v = in[r * NQF + t1 + P * t2];
        yv = fma(B[q1 * P + t1], v, yv);
        yd = fma(Bd[q1 * P + t1], v, yd);
        yn = fma(B[q1 * P + t1], in[(5 + r) * NQF + t1 + P * t2], yn);
      }
      out[r * NQF + fq] = yv;
      out[(5 + r) * NQF + fq] = yd;
      out[(10 + r) * NQF + fq] = yn;
    }
  }
  __syncthreads();
  if (tid < NH) {  // second tangential direction, physical gradient, A(U, grad U).n
    const int j = tid / NQF, lf = FPP * half + j, fq = tid % NQF, q1 = fq % P, q2 = fq / P, a = lf >> 1;
    const T* in = sY + j * 15 * NQF;
    T S[5], g[3][5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      T v = T(0), d1 = T(0), d2 = T(0), dn = T(0);
#pragma unroll
      for (int t2 = 0; t2 < P; ++t2) {
        const T bv = B[q2 * P + t2], bd = Bd[q2 * P + t2];
        const T yv = in[r * NQF + q1 + P * t2];
        v = fma(bv, yv, v);
        d2 = fma(bd, yv, d2);
        d1 = fma(bv, in[(5 + r) * NQF + q1 + P * t2], d1);
        dn = fma(bv, in[(10 + r) * NQF + q1 + P * t2], dn);
      }
      S[r] = v;
      g[0][r] = a == 0 ? dn : d1;
      g[1][r] = a == 0 ? d1 : (a == 1 ? dn : d2);
      g[2][r] = a == 2 ? dn : d2;
    }
    trace_point_store<P, T, CV>(lf, fq, S, g, sg, gfe, mu, kq, Te);
  }
}

template <int P, class T>
struct TraceSmem {
  using C = Cfg<P>;
  static constexpr int oOps = 0;
  static constexpr int oGeo = align16(C::OPS * (int)sizeof(T));
  static constexpr int oU = oGeo + align16(kGeoStride * (int)sizeof(T));
  static constexpr int oN = oU + align16(5 * C::NB * (int)sizeof(T));
  static constexpr int oY = oN + align16(10 * C::FPP * C::NQF * (int)sizeof(T));
  static constexpr int TOTAL = oY + align16(15 * C::FPP * C::NQF * (int)sizeof(T));
};

// Face traces of U (FP64 in HBM) into Tr[e][lf][10][P*P] (type T).
// HT: with the heat flux (prm.kq); without it the heat terms compile away.
template <int P, class T, bool CV, bool HT>
__global__ void __launch_bounds__(Cfg<P>::NTS)
trace_kernel(long E, const double* __restrict__ U, const T* __restrict__ opsg, const double* __restrict__ geo,
             const double* __restrict__ gf, T* __restrict__ Tr, DevParams prm)
{
  using C = Cfg<P>;
  using L = TraceSmem<P, T>;
  constexpr int NB = C::NB, NQF = C::NQF;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw + L::oOps);
  T* sg = reinterpret_cast<T*>(smraw + L::oGeo);
  T* sU = reinterpret_cast<T*>(smraw + L::oU);
  T* sN = reinterpret_cast<T*>(smraw + L::oN);
  T* sY = reinterpret_cast<T*>(smraw + L::oY);
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  for (int i = tid; i < C::OPS; i += blockDim.x) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += blockDim.x) sg[i] = T(geo[e * kGeoStride + i]);
  const double* Ue = U + e * 5 * NB;
  for (int i = tid; i < 5 * NB; i += blockDim.x) sU[i] = T(Ue[i]);
  __syncthreads();
  T* Te = Tr + e * 60 * NQF;
#pragma unroll 1
  for (int half = 0; half < 6 / C::FPP; ++half) {
    if (half) __syncthreads();  // the scratch of the previous pass is reused
    trace_half<P, T, CV>(half, sU, sN, sY, so, sg, T(prm.mu), HT ? T(prm.kq) : T(0), Te, CV ? gf + e * 6 * kFaceC * NQF : nullptr);
  }
}

// ------------------------------------------------------------- face fluxes

// The face terms of one face point (lf, fq) of an element (solve.cpp:393-794):
// fa[r * OS] = the coefficient of the test function phi (Roe or boundary
// flux, minus the viscous normal flux, plus the BR2 lifting), times fJ w;
// fb[(i * 4 + r - 1) * OS] = the dual-consistency coefficient of
// d(phi)/d(xi_i) for variables 1..4.  Uo, Qo: the element's trace (values,
// viscous normal flux) at the point; nb = nbr[e][lf]; for nb >= 0 also the
// neighbour's (Un, Qn) and its lifting scale lift_n.  VO: the viscous terms
// alone (no Roe or boundary Euler flux), for the derivative of the residual
// in the viscosity, in which it is linear.  Shared by the nodal,
// the Gauss-point and the paired Gauss-point stage kernels, so their face
// arithmetic is the same; a pair (T = f2) takes interior faces only.
template <int P, class T, bool CV, int OS = P * P, bool VO = false>
__device__ __forceinline__ void face_point_fluxes(int lf, int fq, int nb, const T* Uo, const T* Qo, const T* Un,
                                                  const T* Qn, T lift_n, const T* so, const T* sg,
                                                  const double* __restrict__ gfe, const DevParams& prm, T gamma,
                                                  T mu, T kq, T detJ, const T* Ji, int* flag, T* fa, T* fb)
{
  using C = Cfg<P>;
  constexpr int NQF = C::NQF;
  const int q1 = fq % P, q2 = fq / P, end = lf & 1;
  const T* w1 = so + C::oW;
  const T eta = T(prm.eta);
  // geometry of this face point (affine elements: the element's, in shared
  // memory; curved ones: per point, each value loaded where it is used)
  const double* gp = CV ? gfe + lf * kFaceC * NQF + fq : nullptr;
  T nbuf[3];
  if constexpr (CV) {
#pragma unroll
    for (int c = 0; c < 3; ++c) nbuf[c] = T(gp[(kFaceN + c) * NQF]);
  }
  const T* n = CV ? nbuf : sg + kGeoN + 3 * lf;
  const T fJ = CV ? T(gp[kFaceFJ * NQF]) : sg[kGeoFJ + lf];
  const T fw = fJ * w1[q1] * w1[q2];
  if (nb >= 0) {
    {
      // the gradient-flux jump first: Qo and Qn are dead after it
      T qd[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) qd[r] = T(0.5) * (Qo[r] - Qn[r]);
      // Roe flux in one orientation for both sides: the element that sees
      // the face on its high side is "left"; the other side negates it
      T F[5];
      const T sgn = end ? T(1) : T(-1);
      if constexpr (VO) {  // no inviscid flux
      } else if constexpr (!std::is_same<T, double>::value) {  // FP32 and pairs measured better with the copies
        T UL[5], UR[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          UL[r] = end ? Uo[r] : Un[r];
          UR[r] = end ? Un[r] : Uo[r];
        }
        const T nn[3] = {sgn * n[0], sgn * n[1], sgn * n[2]};
        roe_flux(UL, UR, nn, gamma, F);
      } else {
        roe_flux_oriented(Uo, Un, end, n, gamma, F);
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) fa[r * OS] = VO ? -qd[r] : sgn * F[r] - qd[r];
    }
    if (mu != T(0)) {
      T d[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) d[r] = Uo[r] - T(0.5) * (Uo[r] + Un[r]);  // Uo - Uhat
      {
        T Jbuf[9];
        if constexpr (CV) {
#pragma unroll
          for (int c = 0; c < 9; ++c) Jbuf[c] = T(gp[c * NQF]);
        }
        dual_consistency_ref(Uo, d, n, mu, CV ? Jbuf : Ji, fw, fb, OS, kq);
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) d[r] = Uo[r] - Un[r];  // jump
      T ro[5], rn[5];
      visc_jump_n(Uo, d, n, mu, ro, kq);  // BR2 lifting sources of both sides
      visc_jump_n(Un, d, n, mu, rn, kq);
      const T lift = CV ? T(gp[kFaceLift * NQF]) : so[C::oC + end] / detJ;
      const T lo = T(0.5) * eta * T(0.5) * fJ * lift;
      const T ln = T(0.5) * eta * T(0.5) * fJ * lift_n;
#pragma unroll
      for (int r = 1; r < 5; ++r) fa[r * OS] += lo * ro[r] + ln * rn[r];
    }
  } else if constexpr (!is_pair<T>::value) {
    T Ub[5];
    const int bad = boundary_state(nb, Uo, n, prm, Ub);
    if (bad && flag) atomicOr(flag, 2);
    if constexpr (VO) {
#pragma unroll
      for (int r = 0; r < 5; ++r) fa[r * OS] = -Qo[r];
    } else {
      T F[5];
      euler_flux_n(Ub, gamma, n, F);
#pragma unroll
      for (int r = 0; r < 5; ++r) fa[r * OS] = F[r] - Qo[r];
    }
    if (mu != T(0)) {
      T d[5], rb[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) d[r] = Uo[r] - Ub[r];
      {
        T Jbuf[9];
        if constexpr (CV) {
#pragma unroll
          for (int c = 0; c < 9; ++c) Jbuf[c] = T(gp[c * NQF]);
        }
        dual_consistency_ref(Uo, d, n, mu, CV ? Jbuf : Ji, fw, fb, OS, kq);
      }
      visc_jump_n(Ub, d, n, mu, rb, kq);
      const T lb = eta * fJ * (CV ? T(gp[kFaceLift * NQF]) : so[C::oC + end] / detJ);
#pragma unroll
      for (int r = 1; r < 5; ++r) fa[r * OS] += lb * rb[r];
    }
  }
  if (mu == T(0)) {
#pragma unroll
    for (int i = 0; i < 12; ++i) fb[i * OS] = T(0);
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) fa[r * OS] *= fw;
}

// The inputs of face_point_fluxes for face point (lf, fq) of element e from
// the trace buffer Tr[E][6][10][NQF]; returns nb.
template <int P, class T, bool CV>
__device__ __forceinline__ int load_face_point(long e, int lf, int fq, const T* __restrict__ Tr,
                                               const int* __restrict__ nbr, const T* so,
                                               const double* __restrict__ geo, const double* __restrict__ gf,
                                               T* Uo, T* Qo, T* Un, T* Qn, T& lift_n)
{
  using C = Cfg<P>;
  constexpr int NQF = C::NQF;
  const T* To = Tr + ((e * 6 + lf) * 10) * NQF;
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    Uo[r] = To[r * NQF + fq];
    Qo[r] = To[(5 + r) * NQF + fq];
  }
  const int nb = nbr[e * 6 + lf];
  lift_n = T(0);
  if (nb >= 0) {
    const T* Tn = Tr + (((long)nb * 6 + (lf ^ 1)) * 10) * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      Un[r] = Tn[r * NQF + fq];
      Qn[r] = Tn[(5 + r) * NQF + fq];
    }
    if constexpr (CV)  // the neighbour's lifting scale at this face point
      lift_n = T(gf[(((long)nb * 6 + (lf ^ 1)) * kFaceC + kFaceLift) * NQF + fq]);
    else
      lift_n = so[C::oC + ((lf & 1) ^ 1)] / T(geo[(long)nb * kGeoStride + kGeoDetJ]);
  }
  return nb;
}

// The global operands of one entry's RK stage value: the step's base state
// and either the RK4 accumulator (stages 2-4) or the stage input (TVD-RK3
// stages 2-3), never both.  A kernel loads those of all its thread's entries
// before it stores any result: the stores may alias the loads as far as the
// compiler knows, so loads interleaved with stores would each wait a full
// memory round trip.
struct RkOperands {
  double ub, x;
};

__device__ __forceinline__ RkOperands rk_stage_load(const StageArgs& sa, long i, const double* ue)
{
  RkOperands q;
  q.ub = sa.Ubase[i];
  if (sa.mode >= MODE_RK4_1 && sa.mode <= MODE_RK4_3)
    q.x = sa.acc ? sa.acc[i] : 0.;
  else
    q.x = sa.mode == MODE_TVD_1 || sa.mode == MODE_TVD_2 ? *ue : 0.;
  return q;
}

// The RK stage value of one entry (time_distributed.cpp:46-102, stage 3 of
// RK4 with dt as the reference's CPU solver) from its loaded operands:
// updates the accumulator and returns the new stage state.  The products
// and sums are written as explicit fused multiply-adds, so every stage
// kernel (FP64, mixed, paired, nodal) rounds the update the same way
// whatever the compiler would contract on its own.
__device__ __forceinline__ double rk_stage_apply(const StageArgs& sa, long i, double fr, const RkOperands& q)
{
  const double dt = sa.dt;
  double un = 0.;
  switch (sa.mode) {
    case MODE_RK4_0:  // (a null accumulator: a stage state recomputed for a reverse step, which needs none)
      if (sa.acc) sa.acc[i] = fr;
      un = fma(dt * fr, 0.5, q.ub);
      break;
    case MODE_RK4_1:
      if (sa.acc) sa.acc[i] = fma(2., fr, q.x);
      un = fma(dt * fr, 0.5, q.ub);
      break;
    case MODE_RK4_2:
      if (sa.acc) sa.acc[i] = fma(2., fr, q.x);
      un = fma(dt, fr, q.ub);
      break;
    case MODE_RK4_3:  // (an explicit add: fr is a product the compiler could otherwise fuse into it)
      un = fma((1. / 6.) * __dadd_rn(q.x, fr), dt, q.ub);
      break;
    case MODE_TVD_0:
      un = fma(dt, fr, q.ub);
      break;
    case MODE_TVD_1:
      un = fma(0.25 * dt, fr, fma(0.25, q.x, 0.75 * q.ub));
      break;
    case MODE_TVD_2:
      un = fma((2. / 3.) * dt, fr, fma(2. / 3., q.x, (1. / 3.) * q.ub));
      break;
  }
  return un;
}

// ------------------------------------------------------------- stage kernel
//
// Shared memory: [operators (T) | inverse 1D mass matrix (FP64) | element
// geometry (T) | misc] followed by one scratch region reused by the phases:
//   volume  V0[5NB] V1[5NB] G[3][5][NB]                               (T)
//   faces   (three faces at a time)                                    (T)
//           Fa[3][5][NQF]   face flux coefficient of phi, times fJ w
//           Fb[3][12][NQF]  reference-space coefficient of grad phi, vars 1..4
//           Su[3][13][NQF]  test functions after the first tangential direction
//           Sc[3][9][NQF]   after the second (aliases Fb)
//   minv    M0[5NB] M1[5NB]                                            (FP64)
//   traces  sN[3][10][NQF] sY[3][15][NQF] of the new state, which sits at oTrU (T)
// The residual of the thread's own node stays in registers until the inverse
// mass matrix is applied.
template <int P, class T>
struct StageSmem {
  using C = Cfg<P>;
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int ST = (int)sizeof(T), SD = (int)sizeof(double);
  static constexpr int oOps = 0;
  static constexpr int oMi = align16(C::OPS * ST);
  static constexpr int oGeo = oMi + align16(P * P * SD);
  static constexpr int oMisc = oGeo + align16(kGeoStride * ST);
  static constexpr int oX = oMisc + align16(8 * ST);
  static constexpr int VOL = 25 * NB * ST;
  static constexpr int FACE = C::FPP * (5 + 12 + 13) * NQF * ST;
  static constexpr int MINV = 10 * NB * SD;
  static constexpr int RED = C::NTS * SD;
  // byte offset of the new state inside the scratch: after the trace buffers
  // and clear of M0/M1, which are still being read when it is written
  static constexpr int oTrU = align16(25 * C::FPP * NQF * ST) > MINV ? align16(25 * C::FPP * NQF * ST) : MINV;
  static constexpr int TRACE = oTrU + 5 * NB * ST;
  static constexpr int X0 = VOL > FACE ? VOL : FACE;
  static constexpr int X1 = MINV > RED ? MINV : RED;
  static constexpr int X2 = X0 > X1 ? X0 : X1;
  static constexpr int X = X2 > TRACE ? X2 : TRACE;
  static constexpr int TOTAL = oX + align16(X);
  static_assert(oTrU >= MINV, "epilogue state must not overlap the inverse-mass buffers");
  static_assert(oX % 16 == 0 && oMi % 16 == 0 && (5 * NB * ST) % 16 == 0 || P % 2 == 1,
                "contraction tiles start on 16-byte boundaries");
};

// CV (curved elements): geometry per point from gv [E][kVolC][P^3] and
// gf [E][6][kFaceC][P^2]; the inverse mass matrix of such an element is
// B3^-1 diag(1/(w detJ)) B3^-T (its mass matrix is B3^T diag(w detJ) B3 with
// B3 = B x B x B square), applied as six 1D contractions and a scaling.
// HT: with the heat flux kq = mu gamma / Pr (prm.kq), an extension the
// reference does not have; the HT = false kernels carry no trace of it.
template <int P, class T, bool CV, bool HT>
__global__ void __launch_bounds__(Cfg<P>::NTS, (MinBlocks<P, T>::value))
stage_kernel(long E, const double* Us, const T* __restrict__ Tr, const T* __restrict__ opsg,
             const double* __restrict__ opsd, const double* __restrict__ geo, const double* __restrict__ gv,
             const double* __restrict__ gf, const int* __restrict__ nbr, DevParams prm, StageArgs sa)
{
  using C = Cfg<P>;
  using L = StageSmem<P, T>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NF, FPP = C::FPP;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw + L::oOps);
  double* sMi = reinterpret_cast<double*>(smraw + L::oMi);
  T* sg = reinterpret_cast<T*>(smraw + L::oGeo);
  unsigned char* sXb = smraw + L::oX;
  T* sX = reinterpret_cast<T*>(sXb);
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  const bool node = tid < NB;  // thread owns node / volume point `tid`

  T* V0 = sX;
  T* V1 = sX + 5 * NB;
  T* G = sX + 10 * NB;
  if (DGB_PREFETCH_L2 && sizeof(T) == 8) {  // data of the face phase and the RK update, read much later
    // (FP64 only: measured 3.4% faster stage there, 0.4% slower in FP32)
    const int nt = blockDim.x;
    prefetch_range(Tr + e * 60 * NQF, 60L * NQF * sizeof(T), tid, nt);
    if (tid < 6) {
      const int nb = nbr[e * 6 + tid];
      if (nb >= 0) prefetch_range(Tr + ((long)nb * 6 + (tid ^ 1)) * 10 * NQF, 10L * NQF * sizeof(T), 0, 1);
    }
    if (sa.Ubase) prefetch_range(sa.Ubase + e * 5 * NB, 40L * NB, tid, nt);
    if (sa.acc && sa.mode >= MODE_RK4_1 && sa.mode <= MODE_RK4_3)
      prefetch_range(sa.acc + e * 5 * NB, 40L * NB, tid, nt);
  }
  for (int i = tid; i < C::OPS; i += blockDim.x) so[i] = opsg[i];
  for (int i = tid; i < P * P; i += blockDim.x) sMi[i] = opsd[(CV ? C::oBi : C::oMi) + i];
  for (int i = tid; i < kGeoStride; i += blockDim.x) sg[i] = T(geo[e * kGeoStride + i]);
  const double* Ue = Us + e * 5 * NB;
  for (int i = tid; i < 5 * NB; i += blockDim.x) V0[i] = T(Ue[i]);
  __syncthreads();

  const T* B = so + C::oB;
  const T* Bd = so + C::oBd;
  const T* Dq = so + C::oDq;
  const double detJd = geo[e * kGeoStride + kGeoDetJ];
  const T detJ = sg[kGeoDetJ];
  const T* Ji = sg + kGeoJinv;
  const T gamma = T(prm.gamma), mu = T(prm.mu), kq = HT ? T(prm.kq) : T(0);
  T Rv[5] = {T(0), T(0), T(0), T(0), T(0)};  // residual of node tid
  const double* gve = CV ? gv + e * kVolC * NB : nullptr;
  const double* gfe = CV ? gf + e * 6 * kFaceC * NQF : nullptr;
  T wJq = T(0);  // w detJ at quadrature point tid (curved elements: for the source)

  // ---------------- volume integral (solve.cpp:276-341) + source (345-360)
  if (node) contract<P, 0, false, false>(B, V0, V1, tid);
  __syncthreads();
  if (node) contract<P, 1, false, false>(B, V1, V0, tid);
  __syncthreads();
  if (node) contract<P, 2, false, false>(B, V0, V1, tid);  // V1: values at quadrature points
  __syncthreads();
  if (node) {
    contract<P, 0, false, false>(Dq, V1, G, tid);
    contract<P, 1, false, false>(Dq, V1, G + 5 * NB, tid);
    contract<P, 2, false, false>(Dq, V1, G + 10 * NB, tid);
  }
  __syncthreads();
  if (node) {  // pointwise flux at quadrature point tid
    const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);
    const T* w = so + C::oW;
    T Jbuf[9];
    T wJ;
    if constexpr (CV) {
#pragma unroll
      for (int c = 0; c < 9; ++c) Jbuf[c] = T(gve[c * NB + tid]);
      wJ = w[qx] * w[qy] * w[qz] * T(gve[kVolDetJ * NB + tid]);
      wJq = wJ;
    } else {
      wJ = w[qx] * w[qy] * w[qz] * detJ;
    }
    const T* Jq = CV ? Jbuf : Ji;  // inverse Jacobian at this point
    T S[5], Gp[3][5], H[3][5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      S[r] = V1[r * NB + tid];
      const T g0 = G[r * NB + tid], g1 = G[5 * NB + r * NB + tid], g2 = G[10 * NB + r * NB + tid];
#pragma unroll
      for (int c = 0; c < 3; ++c) Gp[c][r] = Jq[c] * g0 + Jq[3 + c] * g1 + Jq[6 + c] * g2;
    }
    euler_flux(S, gamma, H);
    if (mu != T(0)) {
      T Q[3][5];
      visc_flux(S, Gp, mu, Q, kq);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 5; ++r) H[c][r] = Q[c][r] - H[c][r];
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 5; ++r) H[c][r] = -H[c][r];
    }
    // contravariant components scaled by the quadrature weight
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int r = 0; r < 5; ++r)
        G[i * 5 * NB + r * NB + tid] = wJ * (Jq[3 * i] * H[0][r] + Jq[3 * i + 1] * H[1][r] + Jq[3 * i + 2] * H[2][r]);
  }
  __syncthreads();
  if (node) {  // sum_i Dq_i^T Ghat_i
    contract<P, 0, true, false>(Dq, G, V0, tid);
    contract<P, 1, true, true>(Dq, G + 5 * NB, V0, tid);
    contract<P, 2, true, true>(Dq, G + 10 * NB, V0, tid);
    if constexpr (CV) {  // source, tested at the quadrature points with w detJ
#pragma unroll
      for (int r = 0; r < 5; ++r) V0[r * NB + tid] -= T(prm.src[r]) * wJq;
    }
  }
  __syncthreads();
  if (node) contract<P, 0, true, false>(B, V0, V1, tid);
  __syncthreads();
  if (node) contract<P, 1, true, false>(B, V1, V0, tid);
  __syncthreads();
  if (node) {
    contract_reg<P, 2, true>(B, V0, tid, Rv);
    if constexpr (!CV) {
      const T* Wb = so + C::oWb;
      const int ix = tid % P, iy = (tid / P) % P, iz = tid / (P * P);
      const T ws = Wb[ix] * Wb[iy] * Wb[iz] * detJ;
#pragma unroll
      for (int r = 0; r < 5; ++r) Rv[r] -= T(prm.src[r]) * ws;
    }
  }
  __syncthreads();

  // ---------------- faces (solve.cpp:393-794), three at a time
  // BR2 lifting: the face-restricted lifting operator E_f Minv E_f^T of an
  // affine element is (cend / detJ) (K x K) with K = B M1^-1 B^T; since
  // M1 = B^T diag(w) B with B square, K = diag(1/w) and the lifted jump at a
  // face point is (cend / detJ) fJ times the pointwise source (solve.cpp:402-480)
  T* Fa = sX;                // [FPP][5][NQF]
  T* Fb = Fa + FPP * 5 * NQF;  // [FPP][12][NQF]
  T* Su = Fb + FPP * 12 * NQF; // [FPP][13][NQF]
  T* Sc = Fb;                // [FPP][9][NQF]
#pragma unroll 1
  for (int half = 0; half < 6 / FPP; ++half) {
    if (tid < NH) {
      const int j = tid / NQF, lf = FPP * half + j, fq = tid % NQF;
      T Uo[5], Qo[5], Un[5], Qn[5], lift_n;
      const int nb = load_face_point<P, T, CV>(e, lf, fq, Tr, nbr, so, geo, gf, Uo, Qo, Un, Qn, lift_n);
      face_point_fluxes<P, T, CV>(lf, fq, nb, Uo, Qo, Un, Qn, lift_n, so, sg, gfe, prm, gamma, mu, kq, detJ, Ji,
                                  sa.flag, Fa + j * 5 * NQF + fq, Fb + j * 12 * NQF + fq);
    }
    __syncthreads();
    if (tid < NH) {  // test functions, first tangential direction: items (j, t1, q2)
      const int j = tid / NQF, lf = FPP * half + j, fq = tid % NQF, t1 = fq % P, q2 = fq / P, a = lf >> 1;
      const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
      const T* fa = Fa + j * 5 * NQF;
      const T* fb = Fb + j * 12 * NQF;
      T u1[5], u2[4], un[4];
#pragma unroll
      for (int r = 0; r < 5; ++r) u1[r] = T(0);
#pragma unroll
      for (int r = 0; r < 4; ++r) u2[r] = un[r] = T(0);
#pragma unroll
      for (int q1 = 0; q1 < P; ++q1) {
        const int q = q1 + P * q2;
        const T b = B[q1 * P + t1], bd = Bd[q1 * P + t1];
        u1[0] = fma(b, fa[q], u1[0]);
#pragma unroll
        for (int r = 1; r < 5; ++r) {
          u1[r] = fma(b, fa[r * NQF + q], u1[r]);
          u1[r] = fma(bd, fb[(ax1 * 4 + r - 1) * NQF + q], u1[r]);
          u2[r - 1] = fma(b, fb[(ax2 * 4 + r - 1) * NQF + q], u2[r - 1]);
          un[r - 1] = fma(b, fb[(a * 4 + r - 1) * NQF + q], un[r - 1]);
        }
      }
      T* su = Su + j * 13 * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) su[r * NQF + fq] = u1[r];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        su[(5 + r) * NQF + fq] = u2[r];
        su[(9 + r) * NQF + fq] = un[r];
      }
    }
    __syncthreads();
    if (tid < NH) {  // second tangential direction: items (j, t1, t2)
      const int j = tid / NQF, fq = tid % NQF, t1 = fq % P, t2 = fq / P;
      const T* su = Su + j * 13 * NQF;
      T c0[5], cn[4];
#pragma unroll
      for (int r = 0; r < 5; ++r) c0[r] = T(0);
#pragma unroll
      for (int r = 0; r < 4; ++r) cn[r] = T(0);
#pragma unroll
      for (int q2 = 0; q2 < P; ++q2) {
        const int q = t1 + P * q2;
        const T b = B[q2 * P + t2], bd = Bd[q2 * P + t2];
        c0[0] = fma(b, su[q], c0[0]);
#pragma unroll
        for (int r = 1; r < 5; ++r) {
          c0[r] = fma(b, su[r * NQF + q], c0[r]);
          c0[r] = fma(bd, su[(4 + r) * NQF + q], c0[r]);
          cn[r - 1] = fma(b, su[(8 + r) * NQF + q], cn[r - 1]);
        }
      }
      T* sc = Sc + j * 9 * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) sc[r * NQF + fq] = c0[r];
#pragma unroll
      for (int r = 0; r < 4; ++r) sc[(5 + r) * NQF + fq] = cn[r];
    }
    __syncthreads();
    if (node) {  // scatter to the node through the normal-direction factors
      const int ix = tid % P, iy = (tid / P) % P, iz = tid / (P * P);
      const T* Ev = so + C::oE;
      const T* Dv = so + C::oD;
#pragma unroll
      for (int j = 0; j < FPP; ++j) {
        const int lf = FPP * half + j, a = lf >> 1, end = lf & 1;
        const int ia = a == 0 ? ix : a == 1 ? iy : iz;
        const int t1 = a == 0 ? iy : ix, t2 = a == 2 ? iy : iz;
        const T ev = Ev[end * P + ia], dv = Dv[end * P + ia];
        const T* sc = Sc + j * 9 * NQF + t1 + P * t2;
        Rv[0] += ev * sc[0];
#pragma unroll
        for (int r = 1; r < 5; ++r) Rv[r] += ev * sc[r * NQF] + dv * sc[(4 + r) * NQF];
      }
    }
    __syncthreads();
  }

  // ---------------- norm partial, f = -Minv R (solve.cpp:800-804) in FP64, RK update
  if (sa.part) {  // sum of R^2 over the element, fixed order
    double s = 0.;
    if (node) {
#pragma unroll
      for (int r = 0; r < 5; ++r) s += double(Rv[r]) * double(Rv[r]);
    }
    double* red = reinterpret_cast<double*>(sXb);
    red[tid] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.;
      for (int i = 0; i < C::NTS; ++i) t += red[i];
      sa.part[e] = t;
    }
    __syncthreads();
  }
  double* M0 = reinterpret_cast<double*>(sXb);
  double* M1 = M0 + 5 * NB;
  if (node) {
#pragma unroll
    for (int r = 0; r < 5; ++r) M0[r * NB + tid] = double(Rv[r]);
  }
  __syncthreads();
  if constexpr (CV) {  // B3^-T, 1/(w detJ), then B3^-1 (the last direction below)
    if (node) contract<P, 0, true, false>(sMi, M0, M1, tid);
    __syncthreads();
    if (node) contract<P, 1, true, false>(sMi, M1, M0, tid);
    __syncthreads();
    if (node) {
      contract<P, 2, true, false>(sMi, M0, M1, tid);
      const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);
      const double iw = 1.0 / (opsd[C::oW + qx] * opsd[C::oW + qy] * opsd[C::oW + qz] * gve[kVolDetJ * NB + tid]);
#pragma unroll
      for (int r = 0; r < 5; ++r) M1[r * NB + tid] *= iw;
    }
    __syncthreads();
    if (node) contract<P, 0, false, false>(sMi, M1, M0, tid);
    __syncthreads();
  }
  if (node) contract<P, CV ? 1 : 0, false, false>(sMi, M0, M1, tid);
  __syncthreads();
  if (node) contract<P, CV ? 2 : 1, false, false>(sMi, M1, M0, tid);
  __syncthreads();
  T* sUn = reinterpret_cast<T*>(sXb + L::oTrU);  // new state for the epilogue traces
  if (node) {
    double f[5];
    if constexpr (CV) {
      // all three directions of B3^-1 are done; copy out
#pragma unroll
      for (int r = 0; r < 5; ++r) f[r] = M0[r * NB + tid];
    } else {
      contract_reg<P, 2, false>(sMi, M0, tid, f);
    }
    const double sc = CV ? -1.0 : -1.0 / detJd;
    const long base = e * 5 * NB;
    if (sa.mode == MODE_RESIDUAL) {
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const long i = base + r * NB + tid;
        sa.fout[i] = f[r] * sc;
        if (sa.Rout) sa.Rout[i] = double(Rv[r]);
      }
    } else {
      RkOperands q[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) q[r] = rk_stage_load(sa, base + r * NB + tid, Ue + r * NB + tid);
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const double un = rk_stage_apply(sa, base + r * NB + tid, f[r] * sc, q[r]);
        sa.Uout[base + r * NB + tid] = un;
        sUn[r * NB + tid] = T(un);
      }
    }
  }
  // ---------------- face traces of the new state for the next stage
  if (sa.Tnext) {
    __syncthreads();
    T* Te = reinterpret_cast<T*>(sa.Tnext) + e * 60 * NQF;
#pragma unroll 1
    for (int half = 0; half < 6 / FPP; ++half) {
      if (half) __syncthreads();
      trace_half<P, T, CV>(half, sUn, sX, sX + 10 * FPP * NQF, so, sg, mu, kq, Te, gfe);
    }
  }
}

// ------------------------------------------------------------ host launchers
// Instantiated per compute type T and heat flag HT, one translation unit each
// (kernels_fp64.cu, kernels_fp32.cu, kernels_heat_fp64.cu, kernels_heat_fp32.cu).

template <int P, class T, bool HT>
cudaError_t prepare_p()
{
  cudaError_t e = cudaFuncSetAttribute(trace_kernel<P, T, false, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TraceSmem<P, T>::TOTAL);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(trace_kernel<P, T, true, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TraceSmem<P, T>::TOTAL);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(stage_kernel<P, T, false, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             StageSmem<P, T>::TOTAL);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(stage_kernel<P, T, true, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             StageSmem<P, T>::TOTAL);
  return e;
}

template <int P, class T, bool HT>
cudaError_t launch_trace_p(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  if (L.gf)
    trace_kernel<P, T, true, HT><<<(unsigned)L.E, Cfg<P>::NTS, TraceSmem<P, T>::TOTAL, st>>>(
        L.E, U, reinterpret_cast<const T*>(L.ops), L.geo, L.gf, reinterpret_cast<T*>(Tout), L.prm);
  else
    trace_kernel<P, T, false, HT><<<(unsigned)L.E, Cfg<P>::NTS, TraceSmem<P, T>::TOTAL, st>>>(
        L.E, U, reinterpret_cast<const T*>(L.ops), L.geo, nullptr, reinterpret_cast<T*>(Tout), L.prm);
  return cudaGetLastError();
}

template <int P, class T, bool HT>
cudaError_t launch_stage_p(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                           cudaStream_t st)
{
  if (L.gv)
    stage_kernel<P, T, true, HT><<<(unsigned)L.E, Cfg<P>::NTS, StageSmem<P, T>::TOTAL, st>>>(
        L.E, Us, reinterpret_cast<const T*>(Tin), reinterpret_cast<const T*>(L.ops), L.opsd, L.geo, L.gv, L.gf,
        L.nbr, L.prm, sa);
  else
    stage_kernel<P, T, false, HT><<<(unsigned)L.E, Cfg<P>::NTS, StageSmem<P, T>::TOTAL, st>>>(
        L.E, Us, reinterpret_cast<const T*>(Tin), reinterpret_cast<const T*>(L.ops), L.opsd, L.geo, nullptr,
        nullptr, L.nbr, L.prm, sa);
  return cudaGetLastError();
}

// the dispatch on the order, for one (T, HT)
template <class T, bool HT>
cudaError_t prepare_t(int P)
{
  switch (P) {
    case 1: return prepare_p<1, T, HT>();
    case 2: return prepare_p<2, T, HT>();
    case 3: return prepare_p<3, T, HT>();
    case 4: return prepare_p<4, T, HT>();
    case 5: return prepare_p<5, T, HT>();
    case 6: return prepare_p<6, T, HT>();
    case 7: return prepare_p<7, T, HT>();
  }
  return cudaErrorInvalidValue;
}

template <class T, bool HT>
cudaError_t launch_trace_t(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_trace_p<1, T, HT>(L, U, Tout, st);
    case 2: return launch_trace_p<2, T, HT>(L, U, Tout, st);
    case 3: return launch_trace_p<3, T, HT>(L, U, Tout, st);
    case 4: return launch_trace_p<4, T, HT>(L, U, Tout, st);
    case 5: return launch_trace_p<5, T, HT>(L, U, Tout, st);
    case 6: return launch_trace_p<6, T, HT>(L, U, Tout, st);
    case 7: return launch_trace_p<7, T, HT>(L, U, Tout, st);
  }
  return cudaErrorInvalidValue;
}

template <class T, bool HT>
cudaError_t launch_stage_t(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                           cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_stage_p<1, T, HT>(L, Us, Tin, sa, st);
    case 2: return launch_stage_p<2, T, HT>(L, Us, Tin, sa, st);
    case 3: return launch_stage_p<3, T, HT>(L, Us, Tin, sa, st);
    case 4: return launch_stage_p<4, T, HT>(L, Us, Tin, sa, st);
    case 5: return launch_stage_p<5, T, HT>(L, Us, Tin, sa, st);
    case 6: return launch_stage_p<6, T, HT>(L, Us, Tin, sa, st);
    case 7: return launch_stage_p<7, T, HT>(L, Us, Tin, sa, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dgb
