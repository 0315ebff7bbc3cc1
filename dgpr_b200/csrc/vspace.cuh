// Gauss-point form of the RK stage, used by dgb_step.
//
// The nodal state U (equispaced Lagrange coefficients, the reference's
// layout, basis.cpp:91-148) and its values at the P^3 Gauss points,
// V = (B x B x B) U, describe the same polynomial: B is square and
// invertible.  Written in V, the discretisation of solve.cpp:150-807 keeps
// every integral and changes only the algebra around them:
//   mass matrix     M = B3^T diag(w detJ) B3  ->  f_V = -Y / (w detJ), Y = B3^-T R
//                   (diagonal: the Gauss points integrate the mass exactly)
//   volume term     R_vol = B3^T sum_i Dq_i^T Ghat_i  ->  Y_vol = sum_i Dq_i^T Ghat_i
//   face terms      phi_node(face point) = (E_end x B x B) -> (EL_end x I x I):
//                   a face point's coefficient reaches the P Gauss points on
//                   its normal line through EL = E B^-1 (values) and
//                   DL = D B^-1 (normal derivatives); the tangential
//                   derivative terms become Dq^T along the face
//   face traces     value / normal derivative at a face point from the normal
//                   line through EL / DL, tangential derivatives by Dq on the
//                   face; no tangential interpolation
// Against the nodal stage kernel this drops the interpolation to the Gauss
// points, the B^T and M1^-1 contractions and one of the two tangential
// passes of the face test functions.  dgb_step converts U -> V before its
// steps and V -> U after them (gauss_basis_kernel); the
// state, stage states and RK accumulator in between are Gauss-point values.
// The face-point fluxes (face_point_fluxes) and the pointwise physics are
// the nodal kernel's own functions.
#pragma once

#include "kernels.cuh"

// L2 prefetch at the start of the FP32 Gauss-point stage as in FP64
// (measured 0.8% faster there; it was slower for the nodal FP32 kernel)
#ifndef DGB_PREFETCH_L2_F32
#define DGB_PREFETCH_L2_F32 1
#endif

// Faces per pass of the Gauss-point kernels' face phase and trace epilogue:
// 6 is one pass over all 6 P^2 face points, each thread striding over them;
// 0 takes the nodal kernels' DGB_FACES_PER_PASS (3: two passes, the threads
// past 3 P^2 idle).  One pass leaves fewer half-empty warps and barriers for
// more shared memory (still 10 CTAs per SM at p = 3); measured on the B200
// against two passes, same bits: FP64 stage -4.5% (32^3, p = 3) and -3%
// (24^3, p = 4), mixed -1.4% and -6.5%.
#ifndef DGB_VFACES_PER_PASS
#define DGB_VFACES_PER_PASS 6
#endif

namespace dgb {

// Synchronizes the threads that own an element: the CTA (GT = 0), a warp
// (GT = 32), or a group of GT threads on named barrier id.
template <int GT>
__device__ __forceinline__ void group_sync(int id)
{
  if constexpr (GT == 0)
    __syncthreads();
  else if constexpr (GT == 32)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(GT) : "memory");
}

template <int P>
struct VF {
  static constexpr int FN = DGB_VFACES_PER_PASS ? DGB_VFACES_PER_PASS : Cfg<P>::FPP;
  static_assert(6 % FN == 0, "faces per pass must divide 6");
};

// Shared memory: [operators (T) | element geometry (T)] followed by one
// scratch region reused by the phases:
//   volume  V1[5NB] values, G[3][5][NB] gradients then contravariant fluxes
//   faces   Fa[FN][5][NQF] Fb[FN][12][NQF] Gt[FN][9][NQF]
//   norm    Y0[5NB] Y1[5NB] (nodal residual for the printed norm), red[NTS] (FP64)
//   traces  sN[FN][10][NQF], then the new state at oTrU
template <int P, class T, int NTHREADS = Cfg<P>::NTS>
struct VStageSmem {
  using C = Cfg<P>;
  static constexpr int NT = NTHREADS;  // threads of the CTA (the norm reduction buffer)
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int ST = (int)sizeof(T);
  static constexpr int oOps = 0;
  static constexpr int oGeo = align16(C::OPS * ST);
  static constexpr int oX = oGeo + align16(kGeoStride * ST);
  static constexpr int VOL = 20 * NB * ST;
  static constexpr int FACE = VF<P>::FN * (5 + 12 + 9) * NQF * ST;
  static constexpr int oRed = align16(10 * NB * ST);
  static constexpr int NORM = oRed + NT * 8;
  static constexpr int oTrU = align16(10 * VF<P>::FN * NQF * ST);
  static constexpr int TRACE = oTrU + 5 * NB * ST;
  static constexpr int X0 = VOL > FACE ? VOL : FACE;
  static constexpr int X1 = NORM > TRACE ? NORM : TRACE;
  static constexpr int X = X0 > X1 ? X0 : X1;
  static constexpr int TOTAL = oX + align16(X);
};

template <int P, class T>
struct VTraceSmem {
  using C = Cfg<P>;
  static constexpr int ST = (int)sizeof(T);
  static constexpr int oOps = 0;
  static constexpr int oGeo = align16(C::OPS * ST);
  static constexpr int oU = oGeo + align16(kGeoStride * ST);
  static constexpr int oN = oU + align16(5 * C::NB * ST);
  static constexpr int TOTAL = oN + align16(10 * VF<P>::FN * C::NQF * ST);
};

// A Gauss-point tile in shared memory with its x-lines LS >= P entries
// apart: point (x, y, z) of variable r at r * LS P^2 + x + LS (y + P z).
// LS = P is the plain layout; LS = P + 1 at P = 4 spreads the lines over
// the banks, so that the 16 face points of an x- or a y-face, read along
// their normal lines by the lanes of a half-warp, fall in distinct banks
// (plain, they are 32 or 128 bytes apart: 4-way conflicts).
template <int P, int LS>
__device__ __forceinline__ int tile_node(int a, int ia, int t1, int t2)
{
  return a == 0 ? ia + LS * (t1 + P * t2) : a == 1 ? t1 + LS * (ia + P * t2) : t1 + LS * (t2 + P * ia);
}

// Traces of a Gauss-point state sV[5][NB] (shared memory, x-lines LS apart)
// on the FN faces lf = FN*half + j, into Te (this element's slice of the
// trace buffer), in the trace format of trace_half.  Scratch
// sN[FN][10][NQF].  GT: the element belongs to a group of GT threads of the
// CTA (32: a warp, ordered by __syncwarp; more: named barrier gbar), 0: to
// the whole CTA.
template <int P, class T, bool CV, int FN = VF<P>::FN, int GT = 0, int LS = P>
__device__ __forceinline__ void vtrace_half(int half, const T* sV, T* sN, const T* so, const T* sg, T mu, T kq,
                                            T* __restrict__ Te, const double* __restrict__ gfe, int gbar = 0)
{
  using C = Cfg<P>;
  constexpr int NB = LS * P * P, NQF = C::NQF, NH = FN * NQF;  // NB: the tile's variable stride
  const int tid = GT ? (int)(threadIdx.x % GT) : (int)threadIdx.x;
  const int nt = GT ? GT : (int)blockDim.x;
#pragma unroll 1
  for (int i = tid; i < NH; i += nt) {  // along the normal line: value and normal derivative
    const int j = i / NQF, lf = FN * half + j, fq = i % NQF, t1 = fq % P, t2 = fq / P;
    const int a = lf >> 1, end = lf & 1;
    const T* Ev = so + C::oEh + end * P;
    const T* Dv = so + C::oDh + end * P;
    T* out = sN + j * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      T v = T(0), dn = T(0);
#pragma unroll
      for (int qa = 0; qa < P; ++qa) {
        const T u = sV[r * NB + tile_node<P, LS>(a, qa, t1, t2)];
        v = fma(Ev[qa], u, v);
        dn = fma(Dv[qa], u, dn);
      }
      out[r * NQF + fq] = v;
      out[(5 + r) * NQF + fq] = dn;
    }
  }
  group_sync<GT>(gbar);
#pragma unroll 1
  for (int i = tid; i < NH; i += nt) {  // tangential derivatives on the face, then the viscous normal flux
    const int j = i / NQF, lf = FN * half + j, fq = i % NQF, q1 = fq % P, q2 = fq / P, a = lf >> 1;
    const T* in = sN + j * 10 * NQF;
    const T* Dq = so + C::oDq;
    T S[5], g[3][5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      T d1 = T(0), d2 = T(0);
#pragma unroll
      for (int k = 0; k < P; ++k) {
        d1 = fma(Dq[q1 * P + k], in[r * NQF + k + P * q2], d1);
        d2 = fma(Dq[q2 * P + k], in[r * NQF + q1 + P * k], d2);
      }
      const T dn = in[(5 + r) * NQF + fq];
      S[r] = in[r * NQF + fq];
      g[0][r] = a == 0 ? dn : d1;
      g[1][r] = a == 0 ? d1 : (a == 1 ? dn : d2);
      g[2][r] = a == 2 ? dn : d2;
    }
    trace_point_store<P, T, CV>(lf, fq, S, g, sg, gfe, mu, kq, Te);
  }
}

// Face traces of a Gauss-point state V (FP64 in HBM) into Tr[e][lf][10][P*P].
template <int P, class T, bool CV, bool HT>
__global__ void __launch_bounds__(Cfg<P>::NTS)
vtrace_kernel(long E, const double* __restrict__ V, const T* __restrict__ opsg, const double* __restrict__ geo,
              const double* __restrict__ gf, T* __restrict__ Tr, DevParams prm)
{
  using C = Cfg<P>;
  using L = VTraceSmem<P, T>;
  constexpr int NB = C::NB, NQF = C::NQF;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw + L::oOps);
  T* sg = reinterpret_cast<T*>(smraw + L::oGeo);
  T* sV = reinterpret_cast<T*>(smraw + L::oU);
  T* sN = reinterpret_cast<T*>(smraw + L::oN);
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  constexpr int NT = C::NTS, NL = (5 * NB + NT - 1) / NT;  // the launch has NTS threads
  double vl[NL];
  load_spread<5 * NB, NT>(V + e * 5 * NB, tid, vl);
  for (int i = tid; i < C::OPS; i += NT) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += NT) sg[i] = T(geo[e * kGeoStride + i]);
#pragma unroll
  for (int k = 0; k < NL; ++k)
    if (tid + k * NT < 5 * NB) sV[tid + k * NT] = T(vl[k]);
  __syncthreads();
  T* Te = Tr + e * 60 * NQF;
#pragma unroll 1
  for (int half = 0; half < 6 / VF<P>::FN; ++half) {
    if (half) __syncthreads();
    vtrace_half<P, T, CV>(half, sV, sN, so, sg, T(prm.mu), HT ? T(prm.kq) : T(0), Te,
                          CV ? gf + e * 6 * kFaceC * NQF : nullptr);
  }
}


// The volume flux at Gauss point o (solve.cpp:276-341): from the state V1 and
// the reference gradients G[3][5][NB] the contravariant flux
// Ghat_i = w detJ (J^-T)_i . (F_visc - F_inv), passed to out(i, r, value);
// returns w detJ at the point.  Affine elements take Ji / detJ, curved ones
// the per-point record gve.  VO: the viscous flux alone.
template <int P, class T, bool CV, bool VO, class Out>
__device__ __forceinline__ T vpoint_flux(const T* so, const T* V1, const T* G, const T* Ji, T detJ,
                                         const double* gve, T gamma, T mu, T kq, int o, Out out)
{
  using C = Cfg<P>;
  constexpr int NB = C::NB;
  const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
  const T* w = so + C::oW;
  T wJq;
  T Jbuf[9];
  if constexpr (CV) {
#pragma unroll
    for (int c = 0; c < 9; ++c) Jbuf[c] = T(gve[c * NB + o]);
    wJq = w[qx] * w[qy] * w[qz] * T(gve[kVolDetJ * NB + o]);
  } else {
    wJq = w[qx] * w[qy] * w[qz] * detJ;
  }
  const T* Jq = CV ? Jbuf : Ji;
  T S[5], Gp[3][5], H[3][5];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    S[r] = V1[r * NB + o];
    const T g0 = G[r * NB + o], g1 = G[5 * NB + r * NB + o], g2 = G[10 * NB + r * NB + o];
#pragma unroll
    for (int c = 0; c < 3; ++c) Gp[c][r] = Jq[c] * g0 + Jq[3 + c] * g1 + Jq[6 + c] * g2;
  }
  if constexpr (VO) {
    visc_flux(S, Gp, mu, H, kq);
  } else {
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
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int r = 0; r < 5; ++r) out(i, r, wJq * (Jq[3 * i] * H[0][r] + Jq[3 * i + 1] * H[1][r] + Jq[3 * i + 2] * H[2][r]));
  return wJq;
}

// Face phase of the Gauss-point stage (solve.cpp:393-794): adds the face
// terms of element e to Rv (Y = B3^-T R at Gauss point tid, node threads).
// Scratch: sX, [FPP][5 + 12 + 9][NQF].  Any CTA size whose threads cover the
// Gauss points.
template <int P, class T, bool CV, bool VO = false>
__device__ __forceinline__ void vstage_faces(long e, const T* __restrict__ Tr, const int* __restrict__ nbr,
                                             const T* so, const T* sg, T* sX, const double* __restrict__ geo,
                                             const double* __restrict__ gf, const double* gfe, const DevParams& prm,
                                             T gamma, T mu, T kq, T detJ, const T* Ji, int* flag, bool node, int qx,
                                             int qy, int qz, T* Rv)
{
  using C = Cfg<P>;
  constexpr int NQF = C::NQF, FPP = VF<P>::FN, NH = FPP * NQF;
  const int tid = threadIdx.x;
  const T* Dq = so + C::oDq;
  T* Fa = sX;                    // [FPP][5][NQF]
  T* Fb = Fa + FPP * 5 * NQF;    // [FPP][12][NQF]
  T* Gt = Fb + FPP * 12 * NQF;   // [FPP][9][NQF]
#pragma unroll 1
  for (int half = 0; half < 6 / FPP; ++half) {
#pragma unroll 1
    for (int i = tid; i < NH; i += blockDim.x) {
      const int j = i / NQF, lf = FPP * half + j, fq = i % NQF;
      T Uo[5], Qo[5], Un[5], Qn[5], lift_n;
      const int nb = load_face_point<P, T, CV>(e, lf, fq, Tr, nbr, so, geo, gf, Uo, Qo, Un, Qn, lift_n);
      face_point_fluxes<P, T, CV, P * P, VO>(lf, fq, nb, Uo, Qo, Un, Qn, lift_n, so, sg, gfe, prm, gamma, mu, kq,
                                             detJ, Ji, flag, Fa + j * 5 * NQF + fq, Fb + j * 12 * NQF + fq);
    }
    __syncthreads();
#pragma unroll 1
    for (int i = tid; i < NH; i += blockDim.x) {  // tangential test derivatives: g = fa + Dq^T fb_ax1 + Dq^T fb_ax2, h = fb_a
      const int j = i / NQF, lf = FPP * half + j, fq = i % NQF, t1 = fq % P, t2 = fq / P, a = lf >> 1;
      const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
      const T* fa = Fa + j * 5 * NQF;
      const T* fb = Fb + j * 12 * NQF;
      T* gt = Gt + j * 9 * NQF;
      gt[fq] = fa[fq];
#pragma unroll
      for (int r = 1; r < 5; ++r) {
        T s = fa[r * NQF + fq];
#pragma unroll
        for (int k = 0; k < P; ++k) {
          s = fma(Dq[k * P + t1], fb[(ax1 * 4 + r - 1) * NQF + k + P * t2], s);
          s = fma(Dq[k * P + t2], fb[(ax2 * 4 + r - 1) * NQF + t1 + P * k], s);
        }
        gt[r * NQF + fq] = s;
        gt[(4 + r) * NQF + fq] = fb[(a * 4 + r - 1) * NQF + fq];
      }
    }
    __syncthreads();
    if (node) {  // each Gauss point gathers from the face points on its normal lines
      const T* Ev = so + C::oEh;
      const T* Dv = so + C::oDh;
#pragma unroll
      for (int j = 0; j < FPP; ++j) {
        const int lf = FPP * half + j, a = lf >> 1, end = lf & 1;
        const int qa = a == 0 ? qx : a == 1 ? qy : qz;
        const int t1 = a == 0 ? qy : qx, t2 = a == 2 ? qy : qz;
        const T ev = Ev[end * P + qa], dv = Dv[end * P + qa];
        const T* gt = Gt + j * 9 * NQF + t1 + P * t2;
        Rv[0] += ev * gt[0];
#pragma unroll
        for (int r = 1; r < 5; ++r) Rv[r] += ev * gt[r * NQF] + dv * gt[(4 + r) * NQF];
      }
    }
    __syncthreads();
  }
}

// The end of the Gauss-point stage: the norm partial (the nodal residual
// R = B3^T Y), f_V = -Y / (w detJ) in FP64 with the RK update, and the face
// traces of the new state for the next stage.  L: the shared-memory layout
// (VStageSmem), whose reduction buffer holds one FP64 per thread.
template <int P, class T, bool CV, class L>
__device__ __forceinline__ void vstage_finish(long e, const StageArgs& sa, const T* Rv, const double* Ve,
                                              const double* gve, double detJd, unsigned char* sXb, const T* so,
                                              const T* sg, const double* __restrict__ opsd, T mu, T kq,
                                              const double* gfe, bool node, int qx, int qy, int qz)
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, FPP = VF<P>::FN;
  const int tid = threadIdx.x;
  T* sX = reinterpret_cast<T*>(sXb);
  // ---------------- norm partial: the nodal residual R = B3^T Y
  if (sa.part) {
    const T* B = so + C::oB;
    T* Y0 = sX;
    T* Y1 = sX + 5 * NB;
    if (node) {
#pragma unroll
      for (int r = 0; r < 5; ++r) Y0[r * NB + tid] = Rv[r];
    }
    __syncthreads();
    if (node) contract<P, 0, true, false>(B, Y0, Y1, tid);
    __syncthreads();
    if (node) contract<P, 1, true, false>(B, Y1, Y0, tid);
    __syncthreads();
    double s = 0.;
    if (node) {
      T rn[5];
      contract_reg<P, 2, true>(B, Y0, tid, rn);
#pragma unroll
      for (int r = 0; r < 5; ++r) s += double(rn[r]) * double(rn[r]);
    }
    double* red = reinterpret_cast<double*>(sXb + L::oRed);
    red[tid] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.;
      for (int i = 0; i < L::NT; ++i) t += red[i];
      sa.part[e] = t;
    }
    __syncthreads();
  }

  // ---------------- f_V = -Y / (w detJ) in FP64, RK update
  T* sVn = reinterpret_cast<T*>(sXb + L::oTrU);  // new state for the epilogue traces
  if (node) {
    const double* w = opsd + C::oW;
    const double jd = CV ? gve[kVolDetJ * NB + tid] : detJd;
    const double sc = -1.0 / (w[qx] * w[qy] * w[qz] * jd);
    const long base = e * 5 * NB;
    if (sa.mode == MODE_RESIDUAL) {
#pragma unroll
      for (int r = 0; r < 5; ++r) sa.fout[base + r * NB + tid] = double(Rv[r]) * sc;
    } else {
      RkOperands q[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) q[r] = rk_stage_load(sa, base + r * NB + tid, Ve + r * NB + tid);
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const double un = rk_stage_apply(sa, base + r * NB + tid, double(Rv[r]) * sc, q[r]);
        sa.Uout[base + r * NB + tid] = un;
        sVn[r * NB + tid] = T(un);
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
      vtrace_half<P, T, CV>(half, sVn, sX, so, sg, mu, kq, Te, gfe);
    }
  }
}

// One RK stage on Gauss-point states: Vs (stage input), sa.Ubase / sa.acc /
// sa.Uout are Gauss-point arrays, Tr the traces of Vs; sa.mode is an RK mode
// (MODE_RESIDUAL writes f_V to sa.fout).  sa.part gets the element's sum of
// the squared nodal residual, the reference's printed norm.  VO: the viscous
// terms alone (MODE_RESIDUAL with the source zeroed: df_V/dmu times mu, the
// residual being linear in mu), for the parameter gradients.
template <int P, class T, bool CV, bool HT, bool VO = false>
__global__ void __launch_bounds__(Cfg<P>::NTS, (MinBlocks<P, T>::value))
vstage_kernel(long E, const double* Vs, const T* __restrict__ Tr, const T* __restrict__ opsg,
              const double* __restrict__ opsd, const double* __restrict__ geo, const double* __restrict__ gv,
              const double* __restrict__ gf, const int* __restrict__ nbr, DevParams prm, StageArgs sa)
{
  using C = Cfg<P>;
  using L = VStageSmem<P, T>;
  constexpr int NB = C::NB, NQF = C::NQF;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw + L::oOps);
  T* sg = reinterpret_cast<T*>(smraw + L::oGeo);
  unsigned char* sXb = smraw + L::oX;
  T* sX = reinterpret_cast<T*>(sXb);
  const long e = sa.ebase + sa.estep * (long)blockIdx.x;
  const int tid = threadIdx.x;
  const bool node = tid < NB;  // thread owns Gauss point `tid`
  const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);

  T* V1 = sX;
  T* G = sX + 5 * NB;
  if (DGB_PREFETCH_L2 && (sizeof(T) == 8 || DGB_PREFETCH_L2_F32)) {  // data read much later
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
  const double* Ve = Vs + e * 5 * NB;
  constexpr int NT = C::NTS, NL = (5 * NB + NT - 1) / NT;  // the launch has NTS threads
  double vl[NL];
  load_spread<5 * NB, NT>(Ve, tid, vl);
  for (int i = tid; i < C::OPS; i += NT) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += NT) sg[i] = T(geo[e * kGeoStride + i]);
#pragma unroll
  for (int k = 0; k < NL; ++k)
    if (tid + k * NT < 5 * NB) V1[tid + k * NT] = T(vl[k]);
  __syncthreads();

  const T* Dq = so + C::oDq;
  const double detJd = geo[e * kGeoStride + kGeoDetJ];
  const T detJ = sg[kGeoDetJ];
  const T* Ji = sg + kGeoJinv;
  const T gamma = T(prm.gamma), mu = T(prm.mu), kq = HT ? T(prm.kq) : T(0);
  T Rv[5] = {T(0), T(0), T(0), T(0), T(0)};  // Y = B3^-T R at Gauss point tid
  const double* gve = CV ? gv + e * kVolC * NB : nullptr;
  const double* gfe = CV ? gf + e * 6 * kFaceC * NQF : nullptr;

  // ---------------- volume integral (solve.cpp:276-341) + source (345-360)
  if (node) {  // reference gradients at the Gauss points
    contract<P, 0, false, false>(Dq, V1, G, tid);
    contract<P, 1, false, false>(Dq, V1, G + 5 * NB, tid);
    contract<P, 2, false, false>(Dq, V1, G + 10 * NB, tid);
  }
  __syncthreads();
  T wJq = T(0);
  if (node)  // pointwise flux at Gauss point tid
    wJq = vpoint_flux<P, T, CV, VO>(so, V1, G, Ji, detJ, gve, gamma, mu, kq, tid,
                                [&](int i, int r, T v) { G[i * 5 * NB + r * NB + tid] = v; });
  __syncthreads();
  if (node) {  // Y = sum_i Dq_i^T Ghat_i, minus the source tested with w detJ
    T y[5];
    contract_reg<P, 0, true>(Dq, G, tid, Rv);
    contract_reg<P, 1, true>(Dq, G + 5 * NB, tid, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) Rv[r] += y[r];
    contract_reg<P, 2, true>(Dq, G + 10 * NB, tid, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) Rv[r] = Rv[r] + y[r] - T(prm.src[r]) * wJq;
  }
  __syncthreads();

  vstage_faces<P, T, CV, VO>(e, Tr, nbr, so, sg, sX, geo, gf, gfe, prm, gamma, mu, kq, detJ, Ji, sa.flag, node, qx,
                             qy, qz, Rv);
  vstage_finish<P, T, CV, L>(e, sa, Rv, Ve, gve, detJd, sXb, so, sg, opsd, mu, kq, gfe, node, qx, qy, qz);
}

// The basis changes at the edges of the Gauss-point form, per element, FP64;
// out2 (may be null) receives a second copy of the result
// (mode: GB_TO_GAUSS V = B3 U, GB_TO_NODAL U = B3^-1 V; for adjoint vectors,
// J(U) = J(B3^-1 V): GB_ADJ_TO_GAUSS dJ/dV = B3^-T dJ/dU, GB_ADJ_TO_NODAL
// dJ/dU = B3^T dJ/dV).
template <int P, int MODE>
__global__ void __launch_bounds__(Cfg<P>::NT) gauss_basis_kernel(long E, const double* __restrict__ in,
                                                                 double* __restrict__ out,
                                                                 const double* __restrict__ opsd,
                                                                 double* __restrict__ out2)
{
  using C = Cfg<P>;
  constexpr int NB = C::NB;
  constexpr bool INV = MODE == GB_TO_NODAL || MODE == GB_ADJ_TO_GAUSS;  // B^-1 (else B)
  constexpr bool TR = MODE == GB_ADJ_TO_GAUSS || MODE == GB_ADJ_TO_NODAL;
  __shared__ __align__(16) double sm[2 * P * P + 10 * NB];
  double* M = sm;
  double* A = sm + 2 * P * P;
  double* Bf = A + 5 * NB;
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  constexpr int NT = C::NT, NL = (5 * NB + NT - 1) / NT;  // the launch has NT threads
  double al[NL];
  load_spread<5 * NB, NT>(in + e * 5 * NB, tid, al);
  for (int i = tid; i < P * P; i += NT) M[i] = opsd[(INV ? C::oBi : C::oB) + i];
#pragma unroll
  for (int k = 0; k < NL; ++k)
    if (tid + k * NT < 5 * NB) A[tid + k * NT] = al[k];
  __syncthreads();
  if (tid < NB) contract<P, 0, TR, false>(M, A, Bf, tid);
  __syncthreads();
  if (tid < NB) contract<P, 1, TR, false>(M, Bf, A, tid);
  __syncthreads();
  if (tid < NB) {
    double v[5];
    contract_reg<P, 2, TR>(M, A, tid, v);
#pragma unroll
    for (int r = 0; r < 5; ++r) out[e * 5 * NB + r * NB + tid] = v[r];
    if (out2) {
#pragma unroll
      for (int r = 0; r < 5; ++r) out2[e * 5 * NB + r * NB + tid] = v[r];
    }
  }
}

// ------------------------------------------------------------ paired FP32 form
//
// The mixed form's Gauss-point stage for two elements at once (e0 = 2k,
// e1 = 2k + 1): every thread computes its Gauss point of both with f2
// arithmetic, one packed FP32x2 instruction per operation (pair.cuh), so the
// instruction stream of the volume, face and trace work serves two elements.
// The arithmetic of each lane is the scalar FP32 kernel's.  Affine meshes
// with an even element count.  Face traces are kept pair-interleaved,
// Tr2[k][lf][10][NQF] of (e0, e1) values; interior faces run paired, and a
// face point where either element meets a boundary runs each element's
// lane through the scalar FP32 face routine (a call, pair_face_lane).  96
// registers (10 CTAs per SM) measured faster than 128 (8 CTAs) once the
// boundary lanes were out of the inlined path.
#ifndef DGB_STAGE_REGS_F2
#define DGB_STAGE_REGS_F2 96
#endif

template <int P>
struct MinBlocksPair {
  static constexpr int RAW = 65536 / (Cfg<P>::NTS * DGB_STAGE_REGS_F2);
  static constexpr int value = RAW < 1 ? 1 : (RAW > 16 ? 16 : RAW);
};

// extra shared memory of the paired kernels: the FP32 operator table and the
// two elements' FP32 geometry for the scalar boundary lanes
template <int P>
struct VPairSmem {
  using S = VStageSmem<P, f2>;
  static constexpr int oOpsF = S::TOTAL;
  static constexpr int oGeoF = oOpsF + align16(Cfg<P>::OPS * 4);
  static constexpr int TOTAL = oGeoF + align16(2 * kGeoStride * 4);
};

template <int P>
struct VTracePairSmem {
  using S = VTraceSmem<P, f2>;
  static constexpr int TOTAL = S::TOTAL;
};

// value of element e's lane in a pair-interleaved array (index idx of its pair)
__device__ __forceinline__ float pair_lane(const f2* a, long idx, long e)
{
  return reinterpret_cast<const float*>(a)[2 * idx + (e & 1)];
}

template <int P, bool HT>
__global__ void __launch_bounds__(Cfg<P>::NTS)
vtrace2_kernel(long E, const double* __restrict__ V, const float* __restrict__ opsg, const double* __restrict__ geo,
               f2* __restrict__ Tr2, DevParams prm)
{
  using C = Cfg<P>;
  using L = VTraceSmem<P, f2>;
  constexpr int NB = C::NB, NQF = C::NQF;
  extern __shared__ __align__(16) unsigned char smraw[];
  f2* so = reinterpret_cast<f2*>(smraw + L::oOps);
  f2* sg = reinterpret_cast<f2*>(smraw + L::oGeo);
  f2* sV = reinterpret_cast<f2*>(smraw + L::oU);
  f2* sN = reinterpret_cast<f2*>(smraw + L::oN);
  const long k = blockIdx.x, e0 = 2 * k, e1 = e0 + 1;
  const int tid = threadIdx.x;
  constexpr int NT = C::NTS, NL = (5 * NB + NT - 1) / NT;  // the launch has NTS threads
  double v0[NL], v1[NL];
  load_spread<5 * NB, NT>(V + e0 * 5 * NB, tid, v0);
  load_spread<5 * NB, NT>(V + e1 * 5 * NB, tid, v1);
  for (int i = tid; i < C::OPS; i += NT) so[i] = f2(opsg[i]);
  for (int i = tid; i < kGeoStride; i += NT)
    sg[i] = f2((float)geo[e0 * kGeoStride + i], (float)geo[e1 * kGeoStride + i]);
#pragma unroll
  for (int k = 0; k < NL; ++k)
    if (tid + k * NT < 5 * NB) sV[tid + k * NT] = f2((float)v0[k], (float)v1[k]);
  __syncthreads();
  f2* Te = Tr2 + k * 60 * NQF;
#pragma unroll 1
  for (int half = 0; half < 6 / VF<P>::FN; ++half) {
    if (half) __syncthreads();
    vtrace_half<P, f2, false>(half, sV, sN, so, sg, f2(prm.mu), HT ? f2(prm.kq) : f2(0.f), Te, nullptr);
  }
}

// One lane of a paired face point where either element meets a boundary,
// through the scalar FP32 face routine.  Not inlined: a call keeps the
// boundary code's registers out of the paired kernel's allocation (taken
// only at boundary faces).
template <int P, bool HT>
__device__ __noinline__ void pair_face_lane(int l, int nb, int lf, int fq, const f2* To, const f2* __restrict__ Tr2,
                                            const float* sof, const float* sgl, const double* __restrict__ geo,
                                            const DevParams prm, int* flag, f2* fa, f2* fb)
{
  using C = Cfg<P>;
  constexpr int NQF = C::NQF;
  float Uo[5], Qo[5], Un[5], Qn[5], lift_n = 0.f, fal[5], fbl[12];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    Uo[r] = To[r * NQF + fq].lane(l);
    Qo[r] = To[(5 + r) * NQF + fq].lane(l);
  }
  if (nb >= 0) {
    const long in = ((long)(nb / 2) * 6 + (lf ^ 1)) * 10 * NQF + fq;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      Un[r] = pair_lane(Tr2, in + r * NQF, nb);
      Qn[r] = pair_lane(Tr2, in + (5 + r) * NQF, nb);
    }
    lift_n = sof[C::oC + ((lf & 1) ^ 1)] / (float)geo[(long)nb * kGeoStride + kGeoDetJ];
  }
  face_point_fluxes<P, float, false, 1>(lf, fq, nb, Uo, Qo, Un, Qn, lift_n, sof, sgl, nullptr, prm,
                                        (float)prm.gamma, (float)prm.mu, HT ? (float)prm.kq : 0.f,
                                        sgl[kGeoDetJ], sgl + kGeoJinv, flag, fal, fbl);
#pragma unroll
  for (int r = 0; r < 5; ++r) reinterpret_cast<float*>(fa + r * NQF)[l] = fal[r];
#pragma unroll
  for (int i = 0; i < 12; ++i) reinterpret_cast<float*>(fb + i * NQF)[l] = fbl[i];
}

template <int P, bool HT>
__global__ void __launch_bounds__(Cfg<P>::NTS, (MinBlocksPair<P>::value))
vstage2_kernel(long E, const double* Vs, const f2* __restrict__ Tr2, const float* __restrict__ opsg,
               const double* __restrict__ opsd, const double* __restrict__ geo, const int* __restrict__ nbr,
               DevParams prm, StageArgs sa)
{
  using C = Cfg<P>;
  using L = VStageSmem<P, f2>;
  using LP = VPairSmem<P>;
  using T = f2;
  constexpr int NB = C::NB, NQF = C::NQF, FPP = VF<P>::FN, NH = FPP * NQF;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw + L::oOps);
  T* sg = reinterpret_cast<T*>(smraw + L::oGeo);
  float* sof = reinterpret_cast<float*>(smraw + LP::oOpsF);
  float* sgf = reinterpret_cast<float*>(smraw + LP::oGeoF);  // [2][kGeoStride]
  unsigned char* sXb = smraw + L::oX;
  T* sX = reinterpret_cast<T*>(sXb);
  const long k = sa.ebase + sa.estep * (long)blockIdx.x, e0 = 2 * k;
  const long el[2] = {e0, e0 + 1};
  const int tid = threadIdx.x;
  const bool node = tid < NB;
  const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);

  T* V1 = sX;
  T* G = sX + 5 * NB;
  if (DGB_PREFETCH_L2 && DGB_PREFETCH_L2_F32) {  // data read much later
    const int nt = blockDim.x;
    prefetch_range(Tr2 + k * 60 * NQF, 60L * NQF * sizeof(T), tid, nt);
    if (tid < 12) {
      const long e = el[tid / 6];
      const int lf = tid % 6, nb = nbr[e * 6 + lf];
      if (nb >= 0) prefetch_range(Tr2 + ((long)(nb / 2) * 6 + (lf ^ 1)) * 10 * NQF, 10L * NQF * sizeof(T), 0, 1);
    }
    for (int l = 0; l < 2; ++l) {
      if (sa.Ubase) prefetch_range(sa.Ubase + el[l] * 5 * NB, 40L * NB, tid, nt);
      if (sa.acc && sa.mode >= MODE_RK4_1 && sa.mode <= MODE_RK4_3)
        prefetch_range(sa.acc + el[l] * 5 * NB, 40L * NB, tid, nt);
    }
  }
  const double* Ve0 = Vs + el[0] * 5 * NB;
  const double* Ve1 = Vs + el[1] * 5 * NB;
  constexpr int NT = C::NTS, NL = (5 * NB + NT - 1) / NT;  // the launch has NTS threads
  double v0[NL], v1[NL];
  load_spread<5 * NB, NT>(Ve0, tid, v0);
  load_spread<5 * NB, NT>(Ve1, tid, v1);
  for (int i = tid; i < C::OPS; i += NT) {
    so[i] = T(opsg[i]);
    sof[i] = opsg[i];
  }
  for (int i = tid; i < kGeoStride; i += NT) {
    const float g0 = (float)geo[el[0] * kGeoStride + i], g1 = (float)geo[el[1] * kGeoStride + i];
    sg[i] = T(g0, g1);
    sgf[i] = g0;
    sgf[kGeoStride + i] = g1;
  }
#pragma unroll
  for (int k = 0; k < NL; ++k)
    if (tid + k * NT < 5 * NB) V1[tid + k * NT] = T((float)v0[k], (float)v1[k]);
  __syncthreads();

  const T* Dq = so + C::oDq;
  const T detJ = sg[kGeoDetJ];
  const T* Ji = sg + kGeoJinv;
  const T gamma = T(prm.gamma), mu = T(prm.mu), kq = HT ? T(prm.kq) : T(0.f);
  T Rv[5] = {T(0.f), T(0.f), T(0.f), T(0.f), T(0.f)};

  // ---------------- volume integral (solve.cpp:276-341) + source (345-360)
  if (node) {
    contract<P, 0, false, false>(Dq, V1, G, tid);
    contract<P, 1, false, false>(Dq, V1, G + 5 * NB, tid);
    contract<P, 2, false, false>(Dq, V1, G + 10 * NB, tid);
  }
  __syncthreads();
  T wJq = T(0.f);
  if (node) {
    const T* w = so + C::oW;
    wJq = w[qx] * w[qy] * w[qz] * detJ;
    T S[5], Gp[3][5], H[3][5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      S[r] = V1[r * NB + tid];
      const T g0 = G[r * NB + tid], g1 = G[5 * NB + r * NB + tid], g2 = G[10 * NB + r * NB + tid];
#pragma unroll
      for (int c = 0; c < 3; ++c) Gp[c][r] = Ji[c] * g0 + Ji[3 + c] * g1 + Ji[6 + c] * g2;
    }
    euler_flux(S, gamma, H);
    if (mu != T(0.f)) {
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
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int r = 0; r < 5; ++r)
        G[i * 5 * NB + r * NB + tid] = wJq * (Ji[3 * i] * H[0][r] + Ji[3 * i + 1] * H[1][r] + Ji[3 * i + 2] * H[2][r]);
  }
  __syncthreads();
  if (node) {
    T y[5];
    contract_reg<P, 0, true>(Dq, G, tid, Rv);
    contract_reg<P, 1, true>(Dq, G + 5 * NB, tid, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) Rv[r] += y[r];
    contract_reg<P, 2, true>(Dq, G + 10 * NB, tid, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) Rv[r] = Rv[r] + y[r] - T(prm.src[r]) * wJq;
  }
  __syncthreads();

  // ---------------- faces, FPP at a time
  T* Fa = sX;
  T* Fb = Fa + FPP * 5 * NQF;
  T* Gt = Fb + FPP * 12 * NQF;
#pragma unroll 1
  for (int half = 0; half < 6 / FPP; ++half) {
#pragma unroll 1
    for (int i = tid; i < NH; i += blockDim.x) {
      const int j = i / NQF, lf = FPP * half + j, fq = i % NQF;
      const int nb0 = nbr[el[0] * 6 + lf], nb1 = nbr[el[1] * 6 + lf];
      const T* To = Tr2 + (k * 6 + lf) * 10 * NQF;
      T* fa = Fa + j * 5 * NQF + fq;
      T* fb = Fb + j * 12 * NQF + fq;
      if (nb0 >= 0 && nb1 >= 0) {  // interior for both: paired
        T Uo[5], Qo[5], Un[5], Qn[5];
        const long i0 = ((long)(nb0 / 2) * 6 + (lf ^ 1)) * 10 * NQF + fq;
        const long i1 = ((long)(nb1 / 2) * 6 + (lf ^ 1)) * 10 * NQF + fq;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          Uo[r] = To[r * NQF + fq];
          Qo[r] = To[(5 + r) * NQF + fq];
          Un[r] = T(pair_lane(Tr2, i0 + r * NQF, nb0), pair_lane(Tr2, i1 + r * NQF, nb1));
          Qn[r] = T(pair_lane(Tr2, i0 + (5 + r) * NQF, nb0), pair_lane(Tr2, i1 + (5 + r) * NQF, nb1));
        }
        const T lift_n = T(sof[C::oC + ((lf & 1) ^ 1)]) /
                         T((float)geo[(long)nb0 * kGeoStride + kGeoDetJ], (float)geo[(long)nb1 * kGeoStride + kGeoDetJ]);
        face_point_fluxes<P, T, false>(lf, fq, 0, Uo, Qo, Un, Qn, lift_n, so, sg, nullptr, prm, gamma, mu, kq, detJ,
                                       Ji, sa.flag, fa, fb);
      } else {  // a boundary in either lane: each lane through the scalar routine
#pragma unroll 1
        for (int l = 0; l < 2; ++l)
          pair_face_lane<P, HT>(l, l ? nb1 : nb0, lf, fq, To, Tr2, sof, sgf + l * kGeoStride, geo, prm, sa.flag,
                                fa, fb);
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int i = tid; i < NH; i += blockDim.x) {  // tangential test derivatives: g = fa + Dq^T fb_ax1 + Dq^T fb_ax2, h = fb_a
      const int j = i / NQF, lf = FPP * half + j, fq = i % NQF, t1 = fq % P, t2 = fq / P, a = lf >> 1;
      const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
      const T* fa = Fa + j * 5 * NQF;
      const T* fb = Fb + j * 12 * NQF;
      T* gt = Gt + j * 9 * NQF;
      gt[fq] = fa[fq];
#pragma unroll
      for (int r = 1; r < 5; ++r) {
        T s = fa[r * NQF + fq];
#pragma unroll
        for (int q = 0; q < P; ++q) {
          s = fma(Dq[q * P + t1], fb[(ax1 * 4 + r - 1) * NQF + q + P * t2], s);
          s = fma(Dq[q * P + t2], fb[(ax2 * 4 + r - 1) * NQF + t1 + P * q], s);
        }
        gt[r * NQF + fq] = s;
        gt[(4 + r) * NQF + fq] = fb[(a * 4 + r - 1) * NQF + fq];
      }
    }
    __syncthreads();
    if (node) {
      const T* Ev = so + C::oEh;
      const T* Dv = so + C::oDh;
#pragma unroll
      for (int j = 0; j < FPP; ++j) {
        const int lf = FPP * half + j, a = lf >> 1, end = lf & 1;
        const int qa = a == 0 ? qx : a == 1 ? qy : qz;
        const int t1 = a == 0 ? qy : qx, t2 = a == 2 ? qy : qz;
        const T ev = Ev[end * P + qa], dv = Dv[end * P + qa];
        const T* gt = Gt + j * 9 * NQF + t1 + P * t2;
        Rv[0] += ev * gt[0];
#pragma unroll
        for (int r = 1; r < 5; ++r) Rv[r] += ev * gt[r * NQF] + dv * gt[(4 + r) * NQF];
      }
    }
    __syncthreads();
  }

  // ---------------- norm partials: the nodal residual R = B3^T Y of each element
  if (sa.part) {
    const T* B = so + C::oB;
    T* Y0 = sX;
    T* Y1 = sX + 5 * NB;
    if (node) {
#pragma unroll
      for (int r = 0; r < 5; ++r) Y0[r * NB + tid] = Rv[r];
    }
    __syncthreads();
    if (node) contract<P, 0, true, false>(B, Y0, Y1, tid);
    __syncthreads();
    if (node) contract<P, 1, true, false>(B, Y1, Y0, tid);
    __syncthreads();
    double s[2] = {0., 0.};
    if (node) {
      T rn[5];
      contract_reg<P, 2, true>(B, Y0, tid, rn);
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int l = 0; l < 2; ++l) s[l] += double(rn[r].lane(l)) * double(rn[r].lane(l));
    }
    double* red = reinterpret_cast<double*>(sXb + L::oRed);
    for (int l = 0; l < 2; ++l) {
      red[tid] = s[l];
      __syncthreads();
      if (tid == 0) {
        double t = 0.;
        for (int i = 0; i < C::NTS; ++i) t += red[i];
        sa.part[el[l]] = t;
      }
      __syncthreads();
    }
  }

  // ---------------- f_V = -Y / (w detJ) in FP64, RK update, per element
  T* sVn = reinterpret_cast<T*>(sXb + L::oTrU);
  if (node) {
    const double* w = opsd + C::oW;
    const double wq = w[qx] * w[qy] * w[qz];
    const double sc0 = -1.0 / (wq * geo[el[0] * kGeoStride + kGeoDetJ]);
    const double sc1 = -1.0 / (wq * geo[el[1] * kGeoStride + kGeoDetJ]);
    const long b0 = el[0] * 5 * NB + tid, b1 = el[1] * 5 * NB + tid;
    if (sa.mode == MODE_RESIDUAL) {
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        sa.fout[b0 + r * NB] = double(Rv[r].lane(0)) * sc0;
        sa.fout[b1 + r * NB] = double(Rv[r].lane(1)) * sc1;
      }
    } else {
      RkOperands q0[5], q1[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        q0[r] = rk_stage_load(sa, b0 + r * NB, Ve0 + r * NB + tid);
        q1[r] = rk_stage_load(sa, b1 + r * NB, Ve1 + r * NB + tid);
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const double un0 = rk_stage_apply(sa, b0 + r * NB, double(Rv[r].lane(0)) * sc0, q0[r]);
        const double un1 = rk_stage_apply(sa, b1 + r * NB, double(Rv[r].lane(1)) * sc1, q1[r]);
        sa.Uout[b0 + r * NB] = un0;
        sa.Uout[b1 + r * NB] = un1;
        sVn[r * NB + tid] = T((float)un0, (float)un1);
      }
    }
  }
  if (sa.Tnext) {
    __syncthreads();
    T* Te = reinterpret_cast<T*>(sa.Tnext) + k * 60 * NQF;
#pragma unroll 1
    for (int half = 0; half < 6 / FPP; ++half) {
      if (half) __syncthreads();
      vtrace_half<P, T, false>(half, sVn, sX, so, sg, mu, kq, Te, nullptr);
    }
  }
}

template <int P, bool HT>
cudaError_t vprepare2_p()
{
  cudaError_t e = cudaFuncSetAttribute(vtrace2_kernel<P, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       VTracePairSmem<P>::TOTAL);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vstage2_kernel<P, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             VPairSmem<P>::TOTAL);
  return e;
}

template <int P, bool HT>
cudaError_t vlaunch_trace2_p(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  vtrace2_kernel<P, HT><<<(unsigned)(L.E / 2), Cfg<P>::NTS, VTracePairSmem<P>::TOTAL, st>>>(
      L.E, V, reinterpret_cast<const float*>(L.ops), L.geo, reinterpret_cast<f2*>(Tout), L.prm);
  return cudaGetLastError();
}

// The stages with a group of warps per element or per pair of elements (one
// warp at p = 3, two at p = 4) (wstage.cuh, included at the end of this
// header).
#ifndef DGB_WARP_STAGE
#define DGB_WARP_STAGE 1
#endif
constexpr int kWarpElems = 2;  // elements (or pairs) per CTA of the warp-group stages
template <int P, class T>
struct WStageSmem;
template <int P, class T, bool CV, bool HT>
__global__ void wstage_kernel(long E, const double* Vs, const T* __restrict__ Tr, const T* __restrict__ opsg,
                              const double* __restrict__ opsd, const double* __restrict__ geo,
                              const double* __restrict__ gv, const double* __restrict__ gf,
                              const int* __restrict__ nbr, DevParams prm, StageArgs sa);

template <int P>
struct WPairSmem;
template <int P, bool HT>
__global__ void wstage2_kernel(long E, const double* Vs, const f2* __restrict__ Tr2, const float* __restrict__ opsg,
                               const double* __restrict__ opsd, const double* __restrict__ geo,
                               const int* __restrict__ nbr, DevParams prm, StageArgs sa);

template <int P, bool HT>
cudaError_t vlaunch_stage2_p(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                             cudaStream_t st)
{
  if constexpr (DGB_WARP_STAGE && (P == 4 || P == 5)) {  // (a CTA per pair at other orders)
    const unsigned npair = (unsigned)((sa.ecount ? sa.ecount : L.E) / 2);
    wstage2_kernel<P, HT><<<(npair + kWarpElems - 1) / kWarpElems, WPairSmem<P>::GT * kWarpElems,
                            WPairSmem<P>::TOTAL, st>>>(
        L.E, Vs, reinterpret_cast<const f2*>(Tin), reinterpret_cast<const float*>(L.ops), L.opsd, L.geo, L.nbr,
        L.prm, element_order(sa, L.E, 2));
    return cudaGetLastError();
  }
  vstage2_kernel<P, HT><<<(unsigned)((sa.ecount ? sa.ecount : L.E) / 2), Cfg<P>::NTS, VPairSmem<P>::TOTAL, st>>>(
      L.E, Vs, reinterpret_cast<const f2*>(Tin), reinterpret_cast<const float*>(L.ops), L.opsd, L.geo, L.nbr,
      L.prm, element_order(sa, L.E, 2));
  return cudaGetLastError();
}

// the paired form serves an FP32 launch on an affine mesh with an even
// element count; everything else takes the one-element kernels
inline bool use_pair(const KLaunch& L) { return L.pair; }

template <bool HT>
cudaError_t vprepare2_t(int P)
{
  switch (P) {
    case 1: return vprepare2_p<1, HT>();
    case 2: return vprepare2_p<2, HT>();
    case 3: return vprepare2_p<3, HT>();
    case 4: return vprepare2_p<4, HT>();
    case 5: return vprepare2_p<5, HT>();
    case 6: return vprepare2_p<6, HT>();
    case 7: return vprepare2_p<7, HT>();
  }
  return cudaErrorInvalidValue;
}

template <bool HT>
cudaError_t vlaunch_trace2_t(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  switch (L.P) {
    case 1: return vlaunch_trace2_p<1, HT>(L, V, Tout, st);
    case 2: return vlaunch_trace2_p<2, HT>(L, V, Tout, st);
    case 3: return vlaunch_trace2_p<3, HT>(L, V, Tout, st);
    case 4: return vlaunch_trace2_p<4, HT>(L, V, Tout, st);
    case 5: return vlaunch_trace2_p<5, HT>(L, V, Tout, st);
    case 6: return vlaunch_trace2_p<6, HT>(L, V, Tout, st);
    case 7: return vlaunch_trace2_p<7, HT>(L, V, Tout, st);
  }
  return cudaErrorInvalidValue;
}

template <bool HT>
cudaError_t vlaunch_stage2_t(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                             cudaStream_t st)
{
  switch (L.P) {
    case 1: return vlaunch_stage2_p<1, HT>(L, Vs, Tin, sa, st);
    case 2: return vlaunch_stage2_p<2, HT>(L, Vs, Tin, sa, st);
    case 3: return vlaunch_stage2_p<3, HT>(L, Vs, Tin, sa, st);
    case 4: return vlaunch_stage2_p<4, HT>(L, Vs, Tin, sa, st);
    case 5: return vlaunch_stage2_p<5, HT>(L, Vs, Tin, sa, st);
    case 6: return vlaunch_stage2_p<6, HT>(L, Vs, Tin, sa, st);
    case 7: return vlaunch_stage2_p<7, HT>(L, Vs, Tin, sa, st);
  }
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------------ host launchers

template <int P, class T, bool HT>
cudaError_t vprepare_p()
{
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vtrace_kernel<P, T, false, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             VTraceSmem<P, T>::TOTAL);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vtrace_kernel<P, T, true, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             VTraceSmem<P, T>::TOTAL);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vstage_kernel<P, T, false, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             VStageSmem<P, T>::TOTAL);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(vstage_kernel<P, T, true, HT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             VStageSmem<P, T>::TOTAL);
  return e;
}

template <int P, class T, bool HT>
cudaError_t vlaunch_trace_p(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  if (L.gf)
    vtrace_kernel<P, T, true, HT><<<(unsigned)L.E, Cfg<P>::NTS, VTraceSmem<P, T>::TOTAL, st>>>(
        L.E, V, reinterpret_cast<const T*>(L.ops), L.geo, L.gf, reinterpret_cast<T*>(Tout), L.prm);
  else
    vtrace_kernel<P, T, false, HT><<<(unsigned)L.E, Cfg<P>::NTS, VTraceSmem<P, T>::TOTAL, st>>>(
        L.E, V, reinterpret_cast<const T*>(L.ops), L.geo, nullptr, reinterpret_cast<T*>(Tout), L.prm);
  return cudaGetLastError();
}

template <int P, class T, bool HT>
cudaError_t vlaunch_stage_p(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                            cudaStream_t st)
{
  const unsigned grid = (unsigned)(sa.ecount ? sa.ecount : L.E);
  const StageArgs so = element_order(sa, L.E, 1);
  if constexpr (DGB_WARP_STAGE && (P == 4 || P == 5)) {
    const unsigned g = (grid + kWarpElems - 1) / kWarpElems;
    const int smem = WStageSmem<P, T>::TOTAL;
    constexpr int NT = WStageSmem<P, T>::GT * kWarpElems;
    if (L.gv)
      wstage_kernel<P, T, true, HT><<<g, NT, smem, st>>>(
          L.E, Vs, reinterpret_cast<const T*>(Tin), reinterpret_cast<const T*>(L.ops), L.opsd, L.geo, L.gv, L.gf,
          L.nbr, L.prm, so);
    else
      wstage_kernel<P, T, false, HT><<<g, NT, smem, st>>>(
          L.E, Vs, reinterpret_cast<const T*>(Tin), reinterpret_cast<const T*>(L.ops), L.opsd, L.geo, nullptr,
          nullptr, L.nbr, L.prm, so);
    return cudaGetLastError();
  }
  if (L.gv)
    vstage_kernel<P, T, true, HT><<<grid, Cfg<P>::NTS, VStageSmem<P, T>::TOTAL, st>>>(
        L.E, Vs, reinterpret_cast<const T*>(Tin), reinterpret_cast<const T*>(L.ops), L.opsd, L.geo, L.gv, L.gf,
        L.nbr, L.prm, so);
  else
    vstage_kernel<P, T, false, HT><<<grid, Cfg<P>::NTS, VStageSmem<P, T>::TOTAL, st>>>(
        L.E, Vs, reinterpret_cast<const T*>(Tin), reinterpret_cast<const T*>(L.ops), L.opsd, L.geo, nullptr,
        nullptr, L.nbr, L.prm, so);
  return cudaGetLastError();
}

template <class T, bool HT>
cudaError_t vprepare_t(int P)
{
  switch (P) {
    case 1: return vprepare_p<1, T, HT>();
    case 2: return vprepare_p<2, T, HT>();
    case 3: return vprepare_p<3, T, HT>();
    case 4: return vprepare_p<4, T, HT>();
    case 5: return vprepare_p<5, T, HT>();
    case 6: return vprepare_p<6, T, HT>();
    case 7: return vprepare_p<7, T, HT>();
  }
  return cudaErrorInvalidValue;
}

template <class T, bool HT>
cudaError_t vlaunch_trace_t(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  switch (L.P) {
    case 1: return vlaunch_trace_p<1, T, HT>(L, V, Tout, st);
    case 2: return vlaunch_trace_p<2, T, HT>(L, V, Tout, st);
    case 3: return vlaunch_trace_p<3, T, HT>(L, V, Tout, st);
    case 4: return vlaunch_trace_p<4, T, HT>(L, V, Tout, st);
    case 5: return vlaunch_trace_p<5, T, HT>(L, V, Tout, st);
    case 6: return vlaunch_trace_p<6, T, HT>(L, V, Tout, st);
    case 7: return vlaunch_trace_p<7, T, HT>(L, V, Tout, st);
  }
  return cudaErrorInvalidValue;
}

template <class T, bool HT>
cudaError_t vlaunch_stage_t(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                            cudaStream_t st)
{
  switch (L.P) {
    case 1: return vlaunch_stage_p<1, T, HT>(L, Vs, Tin, sa, st);
    case 2: return vlaunch_stage_p<2, T, HT>(L, Vs, Tin, sa, st);
    case 3: return vlaunch_stage_p<3, T, HT>(L, Vs, Tin, sa, st);
    case 4: return vlaunch_stage_p<4, T, HT>(L, Vs, Tin, sa, st);
    case 5: return vlaunch_stage_p<5, T, HT>(L, Vs, Tin, sa, st);
    case 6: return vlaunch_stage_p<6, T, HT>(L, Vs, Tin, sa, st);
    case 7: return vlaunch_stage_p<7, T, HT>(L, Vs, Tin, sa, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dgb

#include "wstage.cuh"
