// Discrete adjoint (vector-Jacobian product) of the FP64 residual, hand-written.
//
// For f(U) = -Minv R(U) and an adjoint vector lam (same layout as U) it
// computes Ubar = (df/dU)^T lam = (dR/dU)^T mu with mu = -Minv^T lam.  R is the
// sum of the volume integral and the face terms (solve.cpp:276-794); its
// transpose is applied by three launches:
//   trace_kernel<P,double>  forward face traces of U (values, viscous normal flux)
//   adjA_kernel             per element: mu, the volume term's transpose into
//                           Ubar_part, and for each face point the adjoint of
//                           this element's trace and of the neighbour's trace
//                           (TA[e][lf][20][NQF]: own 10, neighbour 10)
//   adjB_kernel             per element: gathers its neighbours' contributions to
//                           its traces, applies the transpose of the trace map
//                           (face value and gradient of U) and adds Ubar_part
// Every pointwise function is differentiated by hand in physics_vjp.cuh.
// HT: with the heat flux (prm.kq); the HT = false kernels carry no trace of it.
// Instantiated by adjoint.cu (HT = false) and adjoint_heat.cu (HT = true).
#pragma once
#include <cuda_runtime.h>

#include "../../include/dgb200.h"
#include "adjoint.hpp"
#include "kernels.cuh"
#include "physics_vjp.cuh"

// 8 resident CTAs per SM (128 registers a thread at P <= 4): the spills this
// costs are cheaper than the latency exposed at 4 CTAs per SM (measured on
// the reverse RK4 step at 32^3 and 16^3, p = 3)
#ifndef DGB_ADJA_MINB
#define DGB_ADJA_MINB 8
#endif
#ifndef DGB_ADJB_MINB
#define DGB_ADJB_MINB 8
#endif

namespace dgb {

// resident CTAs per SM the adjoint kernels are compiled for (register cap);
// applied to the small element sizes, where one CTA has few threads
template <int P, int M>
struct AdjMinB {
  static constexpr int value = Cfg<P>::NT <= 64 ? M : 1;
};

// Face value S and reference gradient g of a nodal field sUx[5][NB] at the face
// points of faces lf = 3*half + j (threads tid < 3*NQF), returned in
// registers; scratch sN[3][10][NQF], sY[3][15][NQF]; contains two barriers.
template <int P>
__device__ __forceinline__ void face_value_grad(int half, const double* sUx, double* sN, double* sY,
                                                const double* so, double S[5], double g[3][5])
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  const int tid = threadIdx.x;
  const double* B = so + C::oB;
  const double* Bd = so + C::oBd;
  if (tid < NH) {
    const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, t1 = fq % P, t2 = fq / P;
    const int a = lf >> 1, end = lf & 1;
    const double* Ev = so + C::oE + end * P;
    const double* Dv = so + C::oD + end * P;
    double* out = sN + j * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double v = 0., dn = 0.;
#pragma unroll
      for (int ia = 0; ia < P; ++ia) {
        const double u = sUx[r * NB + face_node<P>(a, ia, t1, t2)];
        v = fma(Ev[ia], u, v);
        dn = fma(Dv[ia], u, dn);
      }
      out[r * NQF + fq] = v;
      out[(5 + r) * NQF + fq] = dn;
    }
  }
  __syncthreads();
  if (tid < NH) {
    const int j = tid / NQF, fq = tid % NQF, q1 = fq % P, t2 = fq / P;
    const double* in = sN + j * 10 * NQF;
    double* out = sY + j * 15 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double yv = 0., yd = 0., yn = 0.;
#pragma unroll
      for (int t1 = 0; t1 < P; ++t1) {
        const double v = in[r * NQF + t1 + P * t2];
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
  if (tid < NH) {
    const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, q1 = fq % P, q2 = fq / P, a = lf >> 1;
    const double* in = sY + j * 15 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double v = 0., d1 = 0., d2 = 0., dn = 0.;
#pragma unroll
      for (int t2 = 0; t2 < P; ++t2) {
        const double bv = B[q2 * P + t2], bd = Bd[q2 * P + t2];
        const double yv = in[r * NQF + q1 + P * t2];
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
  }
}

// Transpose of face_value_grad for faces 3*half + j: accumulates into Racc
// (the thread's node, tid < NB) sum_q phi(q) sv(q) + grad_ref phi(q) . sg(q),
// with sv[3][5][NQF], sg[3][15][NQF] (component i*5 + r) in shared memory.
// Scratch su[3][15][NQF], sc[3][10][NQF]; contains three barriers.
template <int P>
__device__ __forceinline__ void face_test_transpose(int half, const double* sv, const double* sgr, double* su,
                                                    double* sc, const double* so, double Racc[5])
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  const int tid = threadIdx.x;
  const double* B = so + C::oB;
  const double* Bd = so + C::oBd;
  if (tid < NH) {  // first tangential direction: items (j, t1, q2)
    const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, t1 = fq % P, q2 = fq / P, a = lf >> 1;
    const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
    const double* fv = sv + j * 5 * NQF;
    const double* fg = sgr + j * 15 * NQF;
    double u1[5] = {0., 0., 0., 0., 0.}, u2[5] = {0., 0., 0., 0., 0.}, un[5] = {0., 0., 0., 0., 0.};
#pragma unroll
    for (int q1 = 0; q1 < P; ++q1) {
      const int q = q1 + P * q2;
      const double b = B[q1 * P + t1], bd = Bd[q1 * P + t1];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        u1[r] = fma(b, fv[r * NQF + q], u1[r]);
        u1[r] = fma(bd, fg[(ax1 * 5 + r) * NQF + q], u1[r]);
        u2[r] = fma(b, fg[(ax2 * 5 + r) * NQF + q], u2[r]);
        un[r] = fma(b, fg[(a * 5 + r) * NQF + q], un[r]);
      }
    }
    double* o = su + j * 15 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      o[r * NQF + fq] = u1[r];
      o[(5 + r) * NQF + fq] = u2[r];
      o[(10 + r) * NQF + fq] = un[r];
    }
  }
  __syncthreads();
  if (tid < NH) {  // second tangential direction: items (j, t1, t2)
    const int j = tid / NQF, fq = tid % NQF, t1 = fq % P, t2 = fq / P;
    const double* i1 = su + j * 15 * NQF;
    double c0[5] = {0., 0., 0., 0., 0.}, cn[5] = {0., 0., 0., 0., 0.};
#pragma unroll
    for (int q2 = 0; q2 < P; ++q2) {
      const int q = t1 + P * q2;
      const double b = B[q2 * P + t2], bd = Bd[q2 * P + t2];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        c0[r] = fma(b, i1[r * NQF + q], c0[r]);
        c0[r] = fma(bd, i1[(5 + r) * NQF + q], c0[r]);
        cn[r] = fma(b, i1[(10 + r) * NQF + q], cn[r]);
      }
    }
    double* o = sc + j * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      o[r * NQF + fq] = c0[r];
      o[(5 + r) * NQF + fq] = cn[r];
    }
  }
  __syncthreads();
  if (tid < NB) {
    const int ix = tid % P, iy = (tid / P) % P, iz = tid / (P * P);
    const double* Ev = so + C::oE;
    const double* Dv = so + C::oD;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int lf = 3 * half + j, a = lf >> 1, end = lf & 1;
      const int ia = a == 0 ? ix : a == 1 ? iy : iz;
      const int t1 = a == 0 ? iy : ix, t2 = a == 2 ? iy : iz;
      const double ev = Ev[end * P + ia], dv = Dv[end * P + ia];
      const double* c = sc + j * 10 * NQF + t1 + P * t2;
#pragma unroll
      for (int r = 0; r < 5; ++r) Racc[r] += ev * c[r * NQF] + dv * c[(5 + r) * NQF];
    }
  }
  __syncthreads();
}

// Gauss-point form of face_value_grad: the field sVx[5][NB] holds values at
// the Gauss points (vspace.cuh); the face value and normal derivative come
// from the normal line through EL / DL, the tangential derivatives from Dq
// on the face.  Scratch sN[3][10][NQF]; contains one barrier.  With WG
// false only S is returned; gface_grad_point reads g from sN afterwards.
template <int P>
__device__ __forceinline__ void gface_grad_point(int half, const double* sN, const double* so, double g[3][5])
{
  using C = Cfg<P>;
  constexpr int NQF = C::NQF;
  const int tid = threadIdx.x;
  const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, q1 = fq % P, q2 = fq / P, a = lf >> 1;
  const double* in = sN + j * 10 * NQF;
  const double* Dq = so + C::oDq;
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double d1 = 0., d2 = 0.;
#pragma unroll
    for (int k = 0; k < P; ++k) {
      d1 = fma(Dq[q1 * P + k], in[r * NQF + k + P * q2], d1);
      d2 = fma(Dq[q2 * P + k], in[r * NQF + q1 + P * k], d2);
    }
    const double dn = in[(5 + r) * NQF + fq];
    g[0][r] = a == 0 ? dn : d1;
    g[1][r] = a == 0 ? d1 : (a == 1 ? dn : d2);
    g[2][r] = a == 2 ? dn : d2;
  }
}

template <int P, bool WG = true>
__device__ __forceinline__ void gface_value_grad(int half, const double* sVx, double* sN, const double* so,
                                                 double S[5], double g[3][5])
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  const int tid = threadIdx.x;
  if (tid < NH) {
    const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, t1 = fq % P, t2 = fq / P;
    const int a = lf >> 1, end = lf & 1;
    const double* Ev = so + C::oEh + end * P;
    const double* Dv = so + C::oDh + end * P;
    double* out = sN + j * 10 * NQF;
    // each face point walks its normal line from a different start, so the
    // 16 face points a half-warp reads at once fall in distinct banks (in
    // order along an x- or y-line they are 32 or 128 bytes apart)
    const int q0 = t1 + t2;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double v = 0., dn = 0.;
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const int qa = (q0 + k) % P;
        const double u = sVx[r * NB + face_node<P>(a, qa, t1, t2)];
        v = fma(Ev[qa], u, v);
        dn = fma(Dv[qa], u, dn);
      }
      out[r * NQF + fq] = v;
      out[(5 + r) * NQF + fq] = dn;
    }
  }
  __syncthreads();
  if (tid < NH) {
    const int j = tid / NQF, fq = tid % NQF;
    const double* in = sN + j * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) S[r] = in[r * NQF + fq];
    if (WG) gface_grad_point<P>(half, sN, so, g);
  }
}

// Transpose of gface_value_grad for faces 3*half + j: accumulates into Racc
// (the thread's Gauss point, tid < NB) the adjoints sv[3][5][NQF] of the face
// values and sgr[3][15][NQF] of the reference gradients (component i*5 + r).
// Scratch sc[3][10][NQF]; contains two barriers.
template <int P>
__device__ __forceinline__ void gface_test_transpose(int half, const double* sv, const double* sgr, double* sc,
                                                     const double* so, double Racc[5])
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  const int tid = threadIdx.x;
  const double* Dq = so + C::oDq;
  if (tid < NH) {  // value adjoint through the tangential derivatives; normal derivative adjoint
    const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, t1 = fq % P, t2 = fq / P, a = lf >> 1;
    const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
    const double* fv = sv + j * 5 * NQF;
    const double* fg = sgr + j * 15 * NQF;
    double* o = sc + j * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double s = fv[r * NQF + fq];
#pragma unroll
      for (int k = 0; k < P; ++k) {
        s = fma(Dq[k * P + t1], fg[(ax1 * 5 + r) * NQF + k + P * t2], s);
        s = fma(Dq[k * P + t2], fg[(ax2 * 5 + r) * NQF + t1 + P * k], s);
      }
      o[r * NQF + fq] = s;
      o[(5 + r) * NQF + fq] = fg[(a * 5 + r) * NQF + fq];
    }
  }
  __syncthreads();
  if (tid < NB) {  // each Gauss point gathers from the face points on its normal lines
    const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);
    const double* Ev = so + C::oEh;
    const double* Dv = so + C::oDh;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int lf = 3 * half + j, a = lf >> 1, end = lf & 1;
      const int qa = a == 0 ? qx : a == 1 ? qy : qz;
      const int t1 = a == 0 ? qy : qx, t2 = a == 2 ? qy : qz;
      const double ev = Ev[end * P + qa], dv = Dv[end * P + qa];
      const double* c = sc + j * 10 * NQF + t1 + P * t2;
#pragma unroll
      for (int r = 0; r < 5; ++r) Racc[r] += ev * c[r * NQF] + dv * c[(5 + r) * NQF];
    }
  }
  __syncthreads();
}

// Inputs of one boundary face point of adjA (passed by value to a function
// that is not inlined).
struct AdjWallIn {
  double Uo[5], n[3], ab[5], zb[5], dcb[3][5], fw, lift;
};

// The adjoint of a boundary face point's fluxes (ghost state, its Euler flux,
// dual consistency, BR2 lifting, the ghost state's own VJP), written to the
// point's slots of TA: T[c * NQF] for c < 20.  Not inlined: boundary points
// are rare, and inlined their registers would count on every path.
static __device__ __noinline__ void adj_boundary_face_point(const AdjWallIn in, int nb, const DevParams prm, double gamma,
                                                     double mu, double kq, int* flag, double* T, int NQF)
{
  double Uob[5] = {0., 0., 0., 0., 0.}, Qob[5];
  double Ubd[5], Ubb[5] = {0., 0., 0., 0., 0.};
  boundary_state(nb, in.Uo, in.n, prm, Ubd);
  {
    double fb[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) fb[r] = in.fw * in.ab[r];
    euler_flux_n_vjp(Ubd, gamma, in.n, fb, Ubb);
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) Qob[r] = -in.fw * in.ab[r];
  if (mu != 0.) {
    double d[5], dbar[5] = {0., 0., 0., 0., 0.};
#pragma unroll
    for (int r = 0; r < 5; ++r) d[r] = in.Uo[r] - Ubd[r];
    visc_rank1_vjp(in.Uo, d, in.n, mu, in.dcb, Uob, dbar, kq);
    const double co = in.fw * in.lift;
    double rbb[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) rbb[r] = co * in.zb[r];
    visc_jump_n_vjp(Ubd, d, in.n, mu, rbb, Ubb, dbar, kq);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      Uob[r] += dbar[r];
      Ubb[r] -= dbar[r];
    }
  }
  // an isothermal wall point leaves its dJ/dTw term (Ub[4] = r R Tw / (gamma - 1)) in the
  // first slot of the neighbour half of TA, which no element reads for a boundary face
  const double wall_term = nb == -8 ? Ubb[4] * in.Uo[0] * (prm.R / (prm.gamma - 1.)) : 0.;
  if (boundary_state_vjp(nb, in.Uo, in.n, prm, Ubb, Uob) && flag) atomicOr(flag, 8);
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    T[r * NQF] = Uob[r];
    T[(5 + r) * NQF] = Qob[r];
    T[(10 + r) * NQF] = r == 0 ? wall_term : 0.;
    T[(15 + r) * NQF] = 0.;
  }
}

template <int P>
struct AdjASmem {
  using C = Cfg<P>;
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int oOps = 0;
  static constexpr int oGeo = (C::OPS + 1) & ~1;
  static constexpr int oNb = oGeo + kGeoStride;   // the neighbours across the six faces (int)
  static constexpr int oMu = oNb + 4;              // mu [5][NB], alive through the face phase
  static constexpr int oX = oMu + 5 * NB;          // scratch
  // volume: V0 V1 Sq [5NB each], G [15NB], N [15NB]
  static constexpr int VOL = 45 * NB;
  // faces: sN[3][10] sY[3][15] (x NQF)
  static constexpr int FACE = 75 * NQF;
  static constexpr int TOTAL = oX + (VOL > FACE ? VOL : FACE);
  // contractions read lines of even P with 16-byte loads: tiles must start on
  // even double offsets
  static_assert(P % 2 == 1 || (oMu % 2 == 0 && oX % 2 == 0 && NB % 2 == 0), "16-byte aligned tiles");
};

// CV (curved elements): per-point geometry from gv / gf as in the stage
// kernel; the inverse mass matrix B3^-1 diag(1/(w detJ)) B3^-T is symmetric,
// so mu takes the same operator.
// GS: the Gauss-point form (vspace.cuh): U, lam and the result hold values at
// the Gauss points, the VJP of f_V = -Y(V) / (w detJ); mu = -lam / (w detJ)
// pointwise, no interpolation to or from the Gauss points, and the face
// values / gradients of mu through the normal lines.
template <int P, bool CV, bool HT, bool GS>
__global__ void __launch_bounds__(Cfg<P>::NT, (AdjMinB<P, DGB_ADJA_MINB>::value))
adjA_kernel(long E, const double* __restrict__ U, const double* __restrict__ Tr, VjpArgs v,
            const double* __restrict__ opsg, const double* __restrict__ geo, const double* __restrict__ gv,
            const double* __restrict__ gf, const int* __restrict__ nbr, DevParams prm,
            double* __restrict__ Ubar_part, double* __restrict__ TA, int* flag)
{
  using C = Cfg<P>;
  using L = AdjASmem<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  extern __shared__ __align__(16) double sm[];
  double* so = sm + L::oOps;
  double* sg = sm + L::oGeo;
  double* Mu = sm + L::oMu;
  double* sX = sm + L::oX;
  double* V0 = sX;
  double* V1 = sX + 5 * NB;
  double* Sq = sX + 10 * NB;
  double* G = sX + 15 * NB;
  double* N = sX + 30 * NB;
  int* sNb = reinterpret_cast<int*>(sm + L::oNb);
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  const bool node = tid < NB;
  // the element's entries of lam's terms and of the state, per thread, with
  // all their loads in flight together (the launch has Cfg<P>::NT threads)
  constexpr int NT = C::NT, NL = (5 * NB + NT - 1) / NT;
  double ul[NL];
  {
    double xl[NL], yl[NL], zl[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      const int i = tid + k * NT;
      const long g = e * 5 * NB + i;
      if (i < 5 * NB) {
        xl[k] = v.X[g];
        yl[k] = v.Y ? v.Y[g] : 0.;
        zl[k] = v.Z ? v.Z[g] : 0.;
        ul[k] = U[g];
      }
    }
    if (tid < 6) sNb[tid] = nbr[e * 6 + tid];
    for (int i = tid; i < C::OPS; i += NT) so[i] = opsg[i];
    for (int i = tid; i < kGeoStride; i += NT) sg[i] = geo[e * kGeoStride + i];
#pragma unroll
    for (int k = 0; k < NL; ++k) {  // lam = cx X + cy Y + cz Z
      const int i = tid + k * NT;
      if (i < 5 * NB) {
        double l = v.cx * xl[k];
        if (v.Y) l = fma(v.cy, yl[k], l);
        if (v.Z) l = fma(v.cz, zl[k], l);
        V0[i] = l;
      }
    }
  }
  __syncthreads();
  const double* B = so + C::oB;
  const double* Dq = so + C::oDq;
  const double* Mi = so + (CV ? C::oBi : C::oMi);
  const double detJ = sg[kGeoDetJ];
  const double gamma = prm.gamma, mu = prm.mu, kq = HT ? prm.kq : 0.;
  const double* gve = CV ? gv + e * kVolC * NB : nullptr;
  const double* gfe = CV ? gf + e * 6 * kFaceC * NQF : nullptr;

  // mu = -Minv^T lam  (f = -Minv R)
  if constexpr (GS) {  // diagonal: -lam / (w detJ) at each Gauss point
    if (node) {
      const double* w = so + C::oW;
      const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);
      const double iw = -1.0 / (w[qx] * w[qy] * w[qz] * (CV ? gve[kVolDetJ * NB + tid] : detJ));
#pragma unroll
      for (int r = 0; r < 5; ++r) Mu[r * NB + tid] = V0[r * NB + tid] * iw;
    }
  } else if constexpr (CV) {  // B3^-T, 1/(w detJ), B3^-1
    if (node) contract<P, 0, true, false>(Mi, V0, V1, tid);
    __syncthreads();
    if (node) contract<P, 1, true, false>(Mi, V1, V0, tid);
    __syncthreads();
    if (node) {
      contract<P, 2, true, false>(Mi, V0, V1, tid);
      const double* w = so + C::oW;
      const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);
      const double iw = -1.0 / (w[qx] * w[qy] * w[qz] * gve[kVolDetJ * NB + tid]);
#pragma unroll
      for (int r = 0; r < 5; ++r) V1[r * NB + tid] *= iw;
    }
    __syncthreads();
    if (node) contract<P, 0, false, false>(Mi, V1, V0, tid);
    __syncthreads();
    if (node) contract<P, 1, false, false>(Mi, V0, V1, tid);
    __syncthreads();
    if (node) contract<P, 2, false, false>(Mi, V1, Mu, tid);
  } else {
    if (node) contract<P, 0, true, false>(Mi, V0, V1, tid);
    __syncthreads();
    if (node) contract<P, 1, true, false>(Mi, V1, V0, tid);
    __syncthreads();
    if (node) contract<P, 2, true, false>(Mi, V0, Mu, tid, -1.0 / detJ);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NL; ++k) {  // the state (at the Gauss points already in GS)
    const int i = tid + k * NT;
    if (i < 5 * NB) (GS ? Sq : V0)[i] = ul[k];
  }
  __syncthreads();

  // ---- volume: recompute S, grad S at the quadrature points; mu and its
  // gradient there; reverse the pointwise flux; transposed projections
  if constexpr (!GS) {
    if (node) contract<P, 0, false, false>(B, V0, V1, tid);
    __syncthreads();
    if (node) contract<P, 1, false, false>(B, V1, V0, tid);
    __syncthreads();
    if (node) contract<P, 2, false, false>(B, V0, Sq, tid);
    __syncthreads();
  }
  if (node) {
    contract<P, 0, false, false>(Dq, Sq, G, tid);
    contract<P, 1, false, false>(Dq, Sq, G + 5 * NB, tid);
    contract<P, 2, false, false>(Dq, Sq, G + 10 * NB, tid);
    if constexpr (!GS) contract<P, 0, false, false>(B, Mu, V0, tid);
  }
  __syncthreads();
  if constexpr (!GS) {
    if (node) contract<P, 1, false, false>(B, V0, V1, tid);
    __syncthreads();
    if (node) contract<P, 2, false, false>(B, V1, V0, tid);  // V0: mu at quadrature points
    __syncthreads();
  }
  if (node) {
    const double* Mq = GS ? Mu : V0;  // mu at the quadrature points
    contract<P, 0, false, false>(Dq, Mq, N, tid);
    contract<P, 1, false, false>(Dq, Mq, N + 5 * NB, tid);
    contract<P, 2, false, false>(Dq, Mq, N + 10 * NB, tid);
  }
  __syncthreads();
  if (node) {  // pointwise reverse at quadrature point tid
    const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);
    const double* w = so + C::oW;
    double Jbuf[9];
    if constexpr (CV) {
#pragma unroll
      for (int c = 0; c < 9; ++c) Jbuf[c] = gve[c * NB + tid];
    }
    const double* Ji = CV ? Jbuf : sg + kGeoJinv;  // inverse Jacobian at this point
    const double wJ = w[qx] * w[qy] * w[qz] * (CV ? gve[kVolDetJ * NB + tid] : detJ);
    double S[5], Hb[3][5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      S[r] = Sq[r * NB + tid];
      const double n0 = N[r * NB + tid], n1 = N[5 * NB + r * NB + tid], n2 = N[10 * NB + r * NB + tid];
#pragma unroll
      for (int c = 0; c < 3; ++c) Hb[c][r] = wJ * (n0 * Ji[c] + n1 * Ji[3 + c] + n2 * Ji[6 + c]);  // adjoint of H = Q - F
    }
    double Sb[5] = {0., 0., 0., 0., 0.}, Gb[3][5];
    // F enters H with a minus sign; the Euler VJP is linear in its cotangent
    euler_flux_vjp(S, gamma, Hb, Sb);
#pragma unroll
    for (int r = 0; r < 5; ++r) Sb[r] = -Sb[r];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 5; ++r) Gb[c][r] = 0.;
    if (mu != 0.) {  // the physical gradients only now: they are dead outside the viscous VJP
      double Gp[3][5];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const double g0 = G[r * NB + tid], g1 = G[5 * NB + r * NB + tid], g2 = G[10 * NB + r * NB + tid];
#pragma unroll
        for (int c = 0; c < 3; ++c) Gp[c][r] = Ji[c] * g0 + Ji[3 + c] * g1 + Ji[6 + c] * g2;
      }
      visc_flux_vjp(S, Gp, mu, Hb, Sb, Gb, kq);
    }
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      Sq[r * NB + tid] = Sb[r];
#pragma unroll
      for (int i = 0; i < 3; ++i)
        N[i * 5 * NB + r * NB + tid] = Ji[3 * i] * Gb[0][r] + Ji[3 * i + 1] * Gb[1][r] + Ji[3 * i + 2] * Gb[2][r];
    }
  }
  __syncthreads();
  double Ub[5] = {0., 0., 0., 0., 0.};
  if constexpr (GS) {  // S-bar + sum_i Dq_i^T g-bar_i at the Gauss point
    if (node) {
      contract<P, 0, true, false>(Dq, N, V0, tid);
      contract<P, 1, true, true>(Dq, N + 5 * NB, V0, tid);
      contract<P, 2, true, true>(Dq, N + 10 * NB, V0, tid);
#pragma unroll
      for (int r = 0; r < 5; ++r) Ub[r] = V0[r * NB + tid] + Sq[r * NB + tid];
    }
    __syncthreads();
  } else {
    if (node) {  // S-bar + sum_i Dq_i^T g-bar_i, then B^T in three directions
      contract<P, 0, true, false>(Dq, N, V0, tid);
      contract<P, 1, true, true>(Dq, N + 5 * NB, V0, tid);
      contract<P, 2, true, true>(Dq, N + 10 * NB, V0, tid);
#pragma unroll
      for (int r = 0; r < 5; ++r) V0[r * NB + tid] += Sq[r * NB + tid];
    }
    __syncthreads();
    if (node) contract<P, 0, true, false>(B, V0, V1, tid);
    __syncthreads();
    if (node) contract<P, 1, true, false>(B, V1, V0, tid);
    __syncthreads();
    if (node) contract_reg<P, 2, true>(B, V0, tid, Ub);
    __syncthreads();
  }

  if (node) {  // the volume part is final: out now, so it holds no registers through the faces
#pragma unroll
    for (int r = 0; r < 5; ++r) Ubar_part[e * 5 * NB + r * NB + tid] = Ub[r];
  }

  // ---- faces.  The lifting's transpose is pointwise like the lifting
  // (K = diag(1/w), see the stage kernel): zb = (K x K)^T (ef fw mu) = ef fJ mu.
  double* sN = sX;
  double* sY = sN + 30 * NQF;
  const double* w1 = so + C::oW;
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, q1 = fq % P, q2 = fq / P, end = lf & 1;
    // this face point's traces, the neighbour and its lifting scale, loaded
    // before the face values of mu are formed
    int nb = -1;
    double Uo[5], Un[5], lift_nb = 0.;
    if (tid < NH) {
      nb = sNb[lf];
      const double* To = Tr + ((e * 6 + lf) * 10) * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) Uo[r] = To[r * NQF + fq];
      if (nb >= 0) {
        const double* Tn = Tr + (((long)nb * 6 + (lf ^ 1)) * 10) * NQF;
#pragma unroll
        for (int r = 0; r < 5; ++r) Un[r] = Tn[r * NQF + fq];
        lift_nb = CV ? gf[(((long)nb * 6 + (lf ^ 1)) * kFaceC + kFaceLift) * NQF + fq]
                     : so[C::oC + (end ^ 1)] / geo[(long)nb * kGeoStride + kGeoDetJ];
      }
    }
    double Sm[5], gm[3][5];
    if constexpr (GS)  // the gradient of mu is read from sN where the viscous terms need it
      gface_value_grad<P, false>(half, Mu, sN, so, Sm, gm);
    else
      face_value_grad<P>(half, Mu, sN, sY, so, Sm, gm);
    if (tid < NH) {
      const double* gp = CV ? gfe + lf * kFaceC * NQF + fq : nullptr;  // this face point's geometry
      const double fJ = CV ? gp[kFaceFJ * NQF] : sg[kGeoFJ + lf];
      const double fw = fJ * w1[q1] * w1[q2];
      const double ef = prm.eta * (nb >= 0 ? 0.5 : 1.0);
      const double lift = CV ? gp[kFaceLift * NQF] : so[C::oC + end] / detJ;  // own lifting scale
      double zb[5];
      zb[0] = 0.;  // the lifting has no mass component
#pragma unroll
      for (int r = 1; r < 5; ++r) zb[r] = ef * fJ * Sm[r];
      double nbuf[3], Jbuf[9];
      if constexpr (CV) {
#pragma unroll
        for (int c = 0; c < 3; ++c) nbuf[c] = gp[(kFaceN + c) * NQF];
#pragma unroll
        for (int c = 0; c < 9; ++c) Jbuf[c] = gp[c * NQF];
      }
      const double* n = CV ? nbuf : sg + kGeoN + 3 * lf;
      const double* Ji = CV ? Jbuf : sg + kGeoJinv;
      double ab[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) ab[r] = Sm[r];
      // adjoint of the dual-consistency tensor: dc_bar[c] = -fw sum_i Jinv[i][c] grad_i(mu),
      // made where the viscous terms use it
      auto dual_bar = [&](double dcb[3][5]) {
        if constexpr (GS) gface_grad_point<P>(half, sN, so, gm);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          dcb[c][0] = 0.;
#pragma unroll
          for (int r = 1; r < 5; ++r)
            dcb[c][r] = -fw * (Ji[c] * gm[0][r] + Ji[3 + c] * gm[1][r] + Ji[6 + c] * gm[2][r]);
        }
      };
      double Uob[5] = {0., 0., 0., 0., 0.}, Qob[5];
      double* TAe = TA + ((e * 6 + lf) * 20) * NQF;
      if (nb >= 0) {
        double Unb[5] = {0., 0., 0., 0., 0.};
        const double iro = 1. / Uo[0], irn = 1. / Un[0];  // once per side for all its VJPs
        {  // Roe flux.  The forward orients it (the high side is left) so that
           // both elements compute the same bits; as a function it is
           // f(Uo, Un, n_out) either way (antisymmetric under swapping the
           // sides and flipping n), so its VJP is taken in this element's
           // orientation, without the side copies
          double fb[5];
#pragma unroll
          for (int r = 0; r < 5; ++r) fb[r] = fw * ab[r];
          roe_flux_vjp_r(Uo, Un, iro, irn, n, gamma, fb, Uob, Unb);
        }
#pragma unroll
        for (int r = 0; r < 5; ++r) Qob[r] = -0.5 * fw * ab[r];
        if (mu != 0.) {
          double d[5], dbar[5] = {0., 0., 0., 0., 0.};
#pragma unroll
          for (int r = 0; r < 5; ++r) d[r] = Uo[r] - 0.5 * (Uo[r] + Un[r]);
          {
            double dcb[3][5];
            dual_bar(dcb);
            visc_rank1_vjp_r(Uo, iro, d, n, mu, dcb, Uob, dbar, kq);
          }
#pragma unroll
          for (int r = 0; r < 5; ++r) {
            Uob[r] += 0.5 * dbar[r];
            Unb[r] -= 0.5 * dbar[r];
            d[r] = Uo[r] - Un[r];
            dbar[r] = 0.;
          }
          const double co = 0.5 * fw * lift;
          const double cn = 0.5 * fw * lift_nb;
          double rob[5], rnb[5];
#pragma unroll
          for (int r = 0; r < 5; ++r) {
            rob[r] = co * zb[r];
            rnb[r] = cn * zb[r];
          }
          visc_jump_n_vjp_r(Uo, iro, d, n, mu, rob, Uob, dbar, kq);
          visc_jump_n_vjp_r(Un, irn, d, n, mu, rnb, Unb, dbar, kq);
#pragma unroll
          for (int r = 0; r < 5; ++r) {
            Uob[r] += dbar[r];
            Unb[r] -= dbar[r];
          }
        }
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          TAe[r * NQF + fq] = Uob[r];
          TAe[(5 + r) * NQF + fq] = Qob[r];
          TAe[(10 + r) * NQF + fq] = Unb[r];
          TAe[(15 + r) * NQF + fq] = -Qob[r];
        }
      } else {  // boundary face point: a call, so its registers stay out of the interior path
        AdjWallIn in;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          in.Uo[r] = Uo[r];
          in.ab[r] = ab[r];
          in.zb[r] = zb[r];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) in.n[c] = n[c];
        if (mu != 0.) {
          dual_bar(in.dcb);
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 5; ++r) in.dcb[c][r] = 0.;
        }
        in.fw = fw;
        in.lift = lift;
        adj_boundary_face_point(in, nb, prm, gamma, mu, kq, flag, TAe + fq, NQF);
      }
    }
    __syncthreads();
  }
}

template <int P>
struct AdjBSmem {
  using C = Cfg<P>;
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int oOps = 0;
  static constexpr int oGeo = (C::OPS + 1) & ~1;
  static constexpr int oNb = oGeo + kGeoStride;  // the neighbours across the six faces (int)
  static constexpr int oU = oNb + 4;
  static constexpr int oX = oU + 5 * NB;
  // sN[3][10] sY[3][15] (then su[3][15] sc[3][10] in their place), sv[3][5], sgr[3][15]  (x NQF)
  static constexpr int TOTAL = oX + 75 * NQF + 60 * NQF;
};

// GS: the Gauss-point form (U and the result at the Gauss points), as adjA.
template <int P, bool CV, bool HT, bool GS>
__global__ void __launch_bounds__(Cfg<P>::NT, (AdjMinB<P, DGB_ADJB_MINB>::value))
adjB_kernel(long E, const double* __restrict__ U, const double* __restrict__ TA, const double* __restrict__ opsg,
            const double* __restrict__ geo, const double* __restrict__ gf, const int* __restrict__ nbr,
            DevParams prm, const double* __restrict__ Ubar_part, VjpArgs v)
{
  using C = Cfg<P>;
  using L = AdjBSmem<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  extern __shared__ __align__(16) double sm[];
  double* so = sm + L::oOps;
  double* sg = sm + L::oGeo;
  double* sU = sm + L::oU;
  double* sX = sm + L::oX;
  double* sN = sX;
  double* sY = sX + 30 * NQF;
  double* su = sX;              // reuses sN / sY after the face values are in registers
  double* sc = sX + 45 * NQF;
  double* sv = sX + 75 * NQF;
  double* sgr = sv + 15 * NQF;
  int* sNb = reinterpret_cast<int*>(sm + L::oNb);
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  constexpr int NT = C::NT, NL = (5 * NB + NT - 1) / NT;  // the launch has NT threads
  double ul[NL];
#pragma unroll
  for (int k = 0; k < NL; ++k) {  // all loads in flight together
    const int i = tid + k * NT;
    if (i < 5 * NB) ul[k] = U[e * 5 * NB + i];
  }
  double Racc[5] = {0., 0., 0., 0., 0.};
  if (tid < NB) {
#pragma unroll
    for (int r = 0; r < 5; ++r) Racc[r] = Ubar_part[e * 5 * NB + r * NB + tid];
  }
  if (tid < 6) sNb[tid] = nbr[e * 6 + tid];
  for (int i = tid; i < C::OPS; i += NT) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += NT) sg[i] = geo[e * kGeoStride + i];
#pragma unroll
  for (int k = 0; k < NL; ++k) {
    const int i = tid + k * NT;
    if (i < 5 * NB) sU[i] = ul[k];
  }
  __syncthreads();
  const double mu = prm.mu, kq = HT ? prm.kq : 0.;
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    // this face point's trace adjoints (its own and the neighbour's side),
    // loaded before the face values are formed
    double vb[5], qb[5];
    if (tid < NH) {
      const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF;
      const int nb = sNb[lf];
      const double* TAo = TA + ((e * 6 + lf) * 20) * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        vb[r] = TAo[r * NQF + fq];
        qb[r] = TAo[(5 + r) * NQF + fq];
      }
      if (nb >= 0) {
        const double* TAn = TA + (((long)nb * 6 + (lf ^ 1)) * 20) * NQF;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          vb[r] += TAn[(10 + r) * NQF + fq];
          qb[r] += TAn[(15 + r) * NQF + fq];
        }
      }
    }
    double S[5], g[3][5];
    if constexpr (GS)
      gface_value_grad<P>(half, sU, sN, so, S, g);
    else
      face_value_grad<P>(half, sU, sN, sY, so, S, g);
    if (tid < NH) {
      const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF;
      double gb[3][5];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 5; ++r) gb[c][r] = 0.;
      if (mu != 0.) {  // trace Qn = A(S, Gp) . n
        double nbuf[3], Jbuf[9];
        if constexpr (CV) {
          const double* gp = gf + ((e * 6 + lf) * kFaceC) * NQF + fq;
#pragma unroll
          for (int c = 0; c < 3; ++c) nbuf[c] = gp[(kFaceN + c) * NQF];
#pragma unroll
          for (int c = 0; c < 9; ++c) Jbuf[c] = gp[c * NQF];
        }
        const double* n = CV ? nbuf : sg + kGeoN + 3 * lf;
        const double* Ji = CV ? Jbuf : sg + kGeoJinv;
        double Gp[3][5], Qb[3][5], Gpb[3][5];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int r = 0; r < 5; ++r) {
            Gp[c][r] = Ji[c] * g[0][r] + Ji[3 + c] * g[1][r] + Ji[6 + c] * g[2][r];
            Qb[c][r] = qb[r] * n[c];
            Gpb[c][r] = 0.;
          }
        visc_flux_vjp(S, Gp, mu, Qb, vb, Gpb, kq);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int r = 0; r < 5; ++r) gb[i][r] = Ji[3 * i] * Gpb[0][r] + Ji[3 * i + 1] * Gpb[1][r] + Ji[3 * i + 2] * Gpb[2][r];
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        sv[(j * 5 + r) * NQF + fq] = vb[r];
#pragma unroll
        for (int i = 0; i < 3; ++i) sgr[(j * 15 + i * 5 + r) * NQF + fq] = gb[i][r];
      }
    }
    __syncthreads();
    if constexpr (GS)
      gface_test_transpose<P>(half, sv, sgr, sc, so, Racc);
    else
      face_test_transpose<P>(half, sv, sgr, su, sc, so, Racc);
  }
  if (tid < NB) {
    double ai[5];  // the running sum's entries, loaded before any store (acc_out may be acc_in)
#pragma unroll
    for (int r = 0; r < 5; ++r) ai[r] = v.acc_out && v.acc_in ? v.acc_in[e * 5 * NB + r * NB + tid] : 0.;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const long g = e * 5 * NB + r * NB + tid;
      if (v.a_out) v.a_out[g] = Racc[r];
      if (v.acc_out) v.acc_out[g] = ai[r] + Racc[r];
    }
  }
}

// ------------------------------------------------------------ host launchers
// GS: the Gauss-point form (the reverse steps of recorded runs in that form)

template <int P, bool CV, bool HT, bool GS>
cudaError_t prepare_pc()
{
  static_assert(AdjASmem<P>::TOTAL * 8 <= 227 * 1024, "adjoint shared memory");
  cudaError_t e = cudaFuncSetAttribute(adjA_kernel<P, CV, HT, GS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(AdjASmem<P>::TOTAL * sizeof(double)));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(adjB_kernel<P, CV, HT, GS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(AdjBSmem<P>::TOTAL * sizeof(double)));
}

template <int P, bool HT, bool GS>
cudaError_t prepare_adj_p()
{
  cudaError_t e = prepare_pc<P, false, HT, GS>();
  return e == cudaSuccess ? prepare_pc<P, true, HT, GS>() : e;
}

template <int P, bool CV, bool HT, bool GS>
cudaError_t vjp_pc(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, const double* Tr, cudaStream_t st)
{
  adjA_kernel<P, CV, HT, GS><<<(unsigned)L.E, Cfg<P>::NT, AdjASmem<P>::TOTAL * sizeof(double), st>>>(
      L.E, v.U, Tr, v, L.opsd, L.geo, L.gv, L.gf, L.nbr, L.prm, s.part, s.ta, s.flag);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  adjB_kernel<P, CV, HT, GS><<<(unsigned)L.E, Cfg<P>::NT, AdjBSmem<P>::TOTAL * sizeof(double), st>>>(
      L.E, v.U, s.ta, L.opsd, L.geo, L.gf, L.nbr, L.prm, s.part, v);
  return cudaGetLastError();
}

template <int P, bool HT, bool GS>
cudaError_t vjp_p(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st)
{
  cudaError_t e;
  const double* Tr = v.Tr;
  if (!Tr) {  // FP64 face traces of v.U (a mixed-precision handle's stages have FP32 ones)
    KLaunch L64 = L;
    L64.precision = DGB_FP64;
    L64.ops = L.opsd;
    e = GS ? launch_vtrace(L64, v.U, s.trace, st) : launch_trace(L64, v.U, s.trace, st);
    if (e != cudaSuccess) return e;
    Tr = s.trace;
  }
  return L.gv ? vjp_pc<P, true, HT, GS>(L, v, s, Tr, st) : vjp_pc<P, false, HT, GS>(L, v, s, Tr, st);
}

// the dispatch on the order, for one (HT, GS)
template <bool HT, bool GS>
cudaError_t prepare_adj_t(int P)
{
  switch (P) {
    case 1: return prepare_adj_p<1, HT, GS>();
    case 2: return prepare_adj_p<2, HT, GS>();
    case 3: return prepare_adj_p<3, HT, GS>();
    case 4: return prepare_adj_p<4, HT, GS>();
    case 5: return prepare_adj_p<5, HT, GS>();
    case 6: return prepare_adj_p<6, HT, GS>();
    case 7: return prepare_adj_p<7, HT, GS>();
  }
  return cudaErrorInvalidValue;
}

template <bool HT, bool GS>
cudaError_t launch_vjp_t(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st)
{
  switch (L.P) {
    case 1: return vjp_p<1, HT, GS>(L, v, s, st);
    case 2: return vjp_p<2, HT, GS>(L, v, s, st);
    case 3: return vjp_p<3, HT, GS>(L, v, s, st);
    case 4: return vjp_p<4, HT, GS>(L, v, s, st);
    case 5: return vjp_p<5, HT, GS>(L, v, s, st);
    case 6: return vjp_p<6, HT, GS>(L, v, s, st);
    case 7: return vjp_p<7, HT, GS>(L, v, s, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dgb
