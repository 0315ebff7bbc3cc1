// FP64 residual / RK-stage kernels for affine hexahedral elements.
//
// One CTA per element.  The tensor-product structure of the basis (equispaced
// Lagrange, basis.cpp:64-170) and of the quadrature (P = p+1 Gauss points per
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
#include <cuda_runtime.h>

#include "kernels.hpp"
#include "physics.cuh"

#ifndef DGB_STAGE_REGS
#define DGB_STAGE_REGS 96
#endif

namespace dgb {

// ------------------------------------------------------------ operator table

template <int P>
struct Cfg {
  static constexpr int NB = P * P * P;  // nodes = volume quadrature points
  static constexpr int NQF = P * P;     // face quadrature points
  static constexpr int NF = 6 * NQF;    // face points of one element
  static constexpr int NH = 3 * NQF;    // face points of half an element (3 faces)
  static constexpr int NT = (((NB > NH ? NB : NH) + 31) / 32) * 32;
  // resident CTAs per SM the stage kernel is compiled for: caps registers at
  // about DGB_STAGE_REGS per thread so occupancy is not register-limited
  static constexpr int MINB_RAW = 65536 / (NT * DGB_STAGE_REGS);
  static constexpr int MINB = MINB_RAW < 1 ? 1 : (MINB_RAW > 16 ? 16 : MINB_RAW);
  // operator table (doubles): B Bd Dq M1i K (P*P each), E0 E1 D0 D1 Wb w (P each), cend[2]
  static constexpr int oB = 0, oBd = P * P, oDq = 2 * P * P, oMi = 3 * P * P, oK = 4 * P * P;
  static constexpr int oE = 5 * P * P, oD = oE + 2 * P, oWb = oD + 2 * P, oW = oWb + P;
  static constexpr int oC = oW + P;
  static constexpr int OPS = oC + 2;
  static constexpr int OPSP = (OPS + 1) & ~1;
};

int ops_table_size(int P) { return 5 * P * P + 6 * P + 2; }

void pack_ops(const Ops1D& o, double* t)
{
  const int P = o.P, PP = P * P;
  for (int i = 0; i < PP; ++i) {
    t[i] = o.B[i];
    t[PP + i] = o.Bd[i];
    t[2 * PP + i] = o.Dq[i];
    t[3 * PP + i] = o.M1i[i];
    t[4 * PP + i] = o.K[i];
  }
  const int oE = 5 * PP, oD = oE + 2 * P, oWb = oD + 2 * P, oW = oWb + P, oC = oW + P;
  for (int i = 0; i < P; ++i) {
    t[oE + i] = o.E[0][i];
    t[oE + P + i] = o.E[1][i];
    t[oD + i] = o.D[0][i];
    t[oD + P + i] = o.D[1][i];
    t[oWb + i] = o.Wb[i];
    t[oW + i] = o.w[i];
  }
  t[oC] = o.cend[0];
  t[oC + 1] = o.cend[1];
}

// ------------------------------------------------------------ index helpers

// node index from the coordinate along face axis a and the two tangential
// coordinates (t1 < t2 in axis order: x faces (y,z), y faces (x,z), z faces (x,y))
template <int P>
__device__ __forceinline__ int face_node(int a, int ia, int t1, int t2)
{
  return a == 0 ? ia + P * (t1 + P * t2) : a == 1 ? t1 + P * (ia + P * t2) : t1 + P * (t2 + P * ia);
}

// one output point o of a 1D contraction along axis AX for all 5 variables:
//   out[r][o] (+)= scale * sum_k M(a, k) in[r][o with coordinate AX replaced by k]
// M(a,k) = Mat[a*P+k], or Mat[k*P+a] when TR.
template <int P, int AX, bool TR, bool ACC>
__device__ __forceinline__ void contract(const double* __restrict__ Mat, const double* in, double* out,
                                         int o, double scale = 1.0)
{
  constexpr int NB = P * P * P;
  constexpr int S = AX == 0 ? 1 : (AX == 1 ? P : P * P);
  const int a = (o / S) % P;
  const int base = o - a * S;
  double m[P];
#pragma unroll
  for (int k = 0; k < P; ++k) m[k] = TR ? Mat[k * P + a] : Mat[a * P + k];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < P; ++k) s = fma(m[k], in[r * NB + base + k * S], s);
    s *= scale;
    out[r * NB + o] = ACC ? out[r * NB + o] + s : s;
  }
}

// same, result returned in registers
template <int P, int AX, bool TR>
__device__ __forceinline__ void contract_reg(const double* __restrict__ Mat, const double* in, int o,
                                             double* res)
{
  constexpr int NB = P * P * P;
  constexpr int S = AX == 0 ? 1 : (AX == 1 ? P : P * P);
  const int a = (o / S) % P;
  const int base = o - a * S;
  double m[P];
#pragma unroll
  for (int k = 0; k < P; ++k) m[k] = TR ? Mat[k * P + a] : Mat[a * P + k];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < P; ++k) s = fma(m[k], in[r * NB + base + k * S], s);
    res[r] = s;
  }
}

// Dual-consistency test coefficients of one face point: with
// dc = A(S, d n^T) (solve.cpp:509-546, 720-741) the face term -grad(phi) . dc fJ w
// becomes sum_i d(phi)/d(xi_i) b_i with b_i = -fw sum_c Jinv[i][c] dc[c].
// Written for variables 1..4 (dc has no mass component): fb[(i*4 + r-1)*stride].
__device__ __forceinline__ void dual_consistency_ref(const double* S, const double* d, const double* n,
                                                     double mu, const double* Ji, double fw, double* fb,
                                                     int stride)
{
  const double lam = -(2.0 / 3.0) * mu;
  const double ir = 1.0 / S[0];
  const double vel[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  double a[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) a[i] = (d[1 + i] - d[0] * vel[i]) * ir;
  const double an = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
  double tau[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) tau[k][c] = mu * (a[k] * n[c] + a[c] * n[k]) + (k == c ? lam * an : 0.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double en = 0.;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double m = Ji[3 * i] * tau[k][0] + Ji[3 * i + 1] * tau[k][1] + Ji[3 * i + 2] * tau[k][2];
      fb[(i * 4 + k) * stride] = -fw * m;
      en += vel[k] * m;
    }
    fb[(i * 4 + 3) * stride] = -fw * en;
  }
}

// ------------------------------------------------------------- face traces

// Traces of a nodal state sUx[5][NB] (shared memory) on the three faces
// lf = 3*half + j, j < 3: at every face quadrature point the 5 conserved values
// and the viscous normal flux A(U, grad U).n_out, written to
// Te[(lf*10 + r)*NQF + fq] (Te = this element's slice of the trace buffer).
// Threads tid < 3*NQF each own one face point.  Scratch: sN[3][10][NQF],
// sY[3][15][NQF].  Both the trace kernel and the stage kernel's epilogue call
// this, so a trace is bit-identical whichever of them produced it.
template <int P>
__device__ __forceinline__ void trace_half(int half, const double* sUx, double* sN, double* sY,
                                           const double* so, const double* sg, double mu,
                                           double* __restrict__ Te)
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  const int tid = threadIdx.x;
  const double* B = so + C::oB;
  const double* Bd = so + C::oBd;
  if (tid < NH) {  // along the face normal: value and normal derivative
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
  if (tid < NH) {  // first tangential direction (index q1 = fq % P)
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
  if (tid < NH) {  // second tangential direction, physical gradient, A(U, grad U).n
    const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, q1 = fq % P, q2 = fq / P, a = lf >> 1;
    const double* in = sY + j * 15 * NQF;
    double S[5], g[3][5];
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
    double Qn[5] = {0., 0., 0., 0., 0.};
    if (mu != 0.) {
      const double* Ji = sg + kGeoJinv;
      double G[3][5], Q[3][5];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 5; ++r) G[c][r] = Ji[c] * g[0][r] + Ji[3 + c] * g[1][r] + Ji[6 + c] * g[2][r];
      visc_flux(S, G, mu, Q);
      const double* n = sg + kGeoN + 3 * lf;
#pragma unroll
      for (int r = 0; r < 5; ++r) Qn[r] = Q[0][r] * n[0] + Q[1][r] * n[1] + Q[2][r] * n[2];
    }
    double* T = Te + lf * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      T[r * NQF + fq] = S[r];
      T[(5 + r) * NQF + fq] = Qn[r];
    }
  }
}

// Face traces of U into Tr[e][lf][10][P*P] for every element.
template <int P>
__global__ void __launch_bounds__(Cfg<P>::NT)
trace_kernel(long E, const double* __restrict__ U, const double* __restrict__ opsg,
             const double* __restrict__ geo, double* __restrict__ Tr, DevParams prm)
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF;
  extern __shared__ double sm[];
  double* so = sm;                  // operators
  double* sg = so + C::OPSP;        // element geometry (kGeoStride)
  double* sU = sg + kGeoStride;     // [5][NB]
  double* sN = sU + 5 * NB;         // [3][10][NQF]
  double* sY = sN + 30 * NQF;       // [3][15][NQF]
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  for (int i = tid; i < C::OPS; i += blockDim.x) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += blockDim.x) sg[i] = geo[e * kGeoStride + i];
  const double* Ue = U + e * 5 * NB;
  for (int i = tid; i < 5 * NB; i += blockDim.x) sU[i] = Ue[i];
  __syncthreads();
  double* Te = Tr + e * 60 * NQF;
  trace_half<P>(0, sU, sN, sY, so, sg, prm.mu, Te);
  trace_half<P>(1, sU, sN, sY, so, sg, prm.mu, Te);
}

// ------------------------------------------------------------- stage kernel
//
// Shared memory: [operators | element geometry | misc] followed by one scratch
// region reused by the phases:
//   volume  V0[5NB] V1[5NB] G[3][5][NB]
//   faces   (three faces at a time)
//           Fa[3][5][NQF]   face flux coefficient of phi (then times fJ w)
//           Fb[3][12][NQF]  reference-space coefficient of grad phi, vars 1..4
//           Fz[3][4][NQF]   BR2 lifting source, vars 1..4 (var 0 has no viscous flux)
//           Fz2[3][4][NQF]  after the first lifting direction
//           Su[3][13][NQF]  test functions after the first tangential direction
//           Sc[3][9][NQF]   after the second (aliases Fb)
//   minv    M0[5NB] M1[5NB]
// The residual of the thread's own node stays in registers until the inverse
// mass matrix is applied.
template <int P>
struct StageSmem {
  using C = Cfg<P>;
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int oOps = 0;
  static constexpr int oGeo = C::OPSP;
  static constexpr int oMisc = oGeo + kGeoStride;
  static constexpr int oX = oMisc + 8;
  static constexpr int VOL = 25 * NB;
  static constexpr int FACE = 3 * (5 + 12 + 4 + 4 + 13) * NQF;
  static constexpr int MINV = 10 * NB;
  static constexpr int RED = C::NT;
  // epilogue traces of the new state: sN[3][10][NQF] sY[3][15][NQF], then the
  // new nodal state at oTrU
  static constexpr int oTrU = 75 * NQF;
  static constexpr int TRACE = oTrU + 5 * NB;
  static constexpr int X0 = VOL > FACE ? VOL : FACE;
  static constexpr int X1 = MINV > RED ? MINV : RED;
  static constexpr int X2 = X0 > X1 ? X0 : X1;
  static constexpr int X = X2 > TRACE ? X2 : TRACE;
  static constexpr int TOTAL = oX + X;
};

template <int P>
__global__ void __launch_bounds__(Cfg<P>::NT, Cfg<P>::MINB)
stage_kernel(long E, const double* Us, const double* __restrict__ Tr,
             const double* __restrict__ opsg, const double* __restrict__ geo,
             const int* __restrict__ nbr, DevParams prm, StageArgs sa)
{
  using C = Cfg<P>;
  using L = StageSmem<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NH = C::NH;
  extern __shared__ double sm[];
  double* so = sm + L::oOps;
  double* sg = sm + L::oGeo;
  double* sMisc = sm + L::oMisc;
  double* sX = sm + L::oX;
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  const bool node = tid < NB;  // thread owns node / volume point `tid`

  double* V0 = sX;
  double* V1 = sX + 5 * NB;
  double* G = sX + 10 * NB;
  for (int i = tid; i < C::OPS; i += blockDim.x) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += blockDim.x) sg[i] = geo[e * kGeoStride + i];
  const double* Ue = Us + e * 5 * NB;
  for (int i = tid; i < 5 * NB; i += blockDim.x) V0[i] = Ue[i];
  __syncthreads();

  const double* B = so + C::oB;
  const double* Bd = so + C::oBd;
  const double* Dq = so + C::oDq;
  const double detJ = sg[kGeoDetJ];
  const double* Ji = sg + kGeoJinv;
  double Rv[5] = {0., 0., 0., 0., 0.};  // residual of node tid

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
    const double* w = so + C::oW;
    const double wJ = w[qx] * w[qy] * w[qz] * detJ;
    double S[5], Gp[3][5], H[3][5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      S[r] = V1[r * NB + tid];
      const double g0 = G[r * NB + tid], g1 = G[5 * NB + r * NB + tid], g2 = G[10 * NB + r * NB + tid];
#pragma unroll
      for (int c = 0; c < 3; ++c) Gp[c][r] = Ji[c] * g0 + Ji[3 + c] * g1 + Ji[6 + c] * g2;
    }
    euler_flux(S, prm.gamma, H);
    if (prm.mu != 0.) {
      double Q[3][5];
      visc_flux(S, Gp, prm.mu, Q);
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
        G[i * 5 * NB + r * NB + tid] = wJ * (Ji[3 * i] * H[0][r] + Ji[3 * i + 1] * H[1][r] + Ji[3 * i + 2] * H[2][r]);
  }
  __syncthreads();
  if (node) {  // sum_i Dq_i^T Ghat_i
    contract<P, 0, true, false>(Dq, G, V0, tid);
    contract<P, 1, true, true>(Dq, G + 5 * NB, V0, tid);
    contract<P, 2, true, true>(Dq, G + 10 * NB, V0, tid);
  }
  __syncthreads();
  if (node) contract<P, 0, true, false>(B, V0, V1, tid);
  __syncthreads();
  if (node) contract<P, 1, true, false>(B, V1, V0, tid);
  __syncthreads();
  if (node) {
    contract_reg<P, 2, true>(B, V0, tid, Rv);
    const double* Wb = so + C::oWb;
    const int ix = tid % P, iy = (tid / P) % P, iz = tid / (P * P);
    const double ws = Wb[ix] * Wb[iy] * Wb[iz] * detJ;
#pragma unroll
    for (int r = 0; r < 5; ++r) Rv[r] -= prm.src[r] * ws;
  }
  __syncthreads();

  // ---------------- faces (solve.cpp:393-794), three at a time
  double* Fa = sX;
  double* Fb = Fa + 15 * NQF;
  double* Fz = Fb + 36 * NQF;
  double* Fz2 = Fz + 12 * NQF;
  double* Su = Fz2 + 12 * NQF;
  double* Sc = Fb;
  const double gamma = prm.gamma, mu = prm.mu;
  const double* K = so + C::oK;
  const double* w1 = so + C::oW;
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    if (tid < NH) {
      const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, q1 = fq % P, q2 = fq / P, end = lf & 1;
      const double* n = sg + kGeoN + 3 * lf;
      const double fw = sg[kGeoFJ + lf] * w1[q1] * w1[q2];
      const double* To = Tr + ((e * 6 + lf) * 10) * NQF;
      double Uo[5], Qo[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        Uo[r] = To[r * NQF + fq];
        Qo[r] = To[(5 + r) * NQF + fq];
      }
      const int nb = nbr[e * 6 + lf];
      double* fa = Fa + j * 5 * NQF + fq;
      double* fb = Fb + j * 12 * NQF + fq;
      double* fz = Fz + j * 4 * NQF + fq;
      if (nb >= 0) {
        const double* Tn = Tr + (((long)nb * 6 + (lf ^ 1)) * 10) * NQF;
        double Un[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) Un[r] = Tn[r * NQF + fq];
        {
          // Roe flux in one orientation for both sides: the element that sees
          // the face on its high side is "left"
          double F[5];
          if (end) {
            roe_flux(Uo, Un, n, gamma, F);
          } else {
            const double nn[3] = {-n[0], -n[1], -n[2]};
            roe_flux(Un, Uo, nn, gamma, F);
#pragma unroll
            for (int r = 0; r < 5; ++r) F[r] = -F[r];
          }
#pragma unroll
          for (int r = 0; r < 5; ++r) fa[r * NQF] = F[r] - 0.5 * (Qo[r] - Tn[(5 + r) * NQF + fq]);
        }
        if (mu != 0.) {
          double d[5];
#pragma unroll
          for (int r = 0; r < 5; ++r) d[r] = Uo[r] - 0.5 * (Uo[r] + Un[r]);  // Uo - Uhat
          dual_consistency_ref(Uo, d, n, mu, Ji, fw, fb, NQF);
#pragma unroll
          for (int r = 0; r < 5; ++r) d[r] = Uo[r] - Un[r];  // jump
          double ro[5], rn[5];
          visc_jump_n(Uo, d, n, mu, ro);  // BR2 lifting sources of both sides
          visc_jump_n(Un, d, n, mu, rn);
          const double co = 0.5 * fw * so[C::oC + end] / detJ;
          const double cn = 0.5 * fw * so[C::oC + (end ^ 1)] / geo[(long)nb * kGeoStride + kGeoDetJ];
#pragma unroll
          for (int r = 1; r < 5; ++r) fz[(r - 1) * NQF] = co * ro[r] + cn * rn[r];
        }
        if (fq == 0) sMisc[j] = 0.5;
      } else {
        double Ub[5];
        const int bad = boundary_state(nb, Uo, n, prm, Ub);
        if (bad && sa.flag) atomicOr(sa.flag, 2);
        {
          double F[5];
          euler_flux_n(Ub, gamma, n, F);
#pragma unroll
          for (int r = 0; r < 5; ++r) fa[r * NQF] = F[r] - Qo[r];
        }
        if (mu != 0.) {
          double d[5], rb[5];
#pragma unroll
          for (int r = 0; r < 5; ++r) d[r] = Uo[r] - Ub[r];
          dual_consistency_ref(Uo, d, n, mu, Ji, fw, fb, NQF);
          visc_jump_n(Ub, d, n, mu, rb);
          const double co = fw * so[C::oC + end] / detJ;
#pragma unroll
          for (int r = 1; r < 5; ++r) fz[(r - 1) * NQF] = co * rb[r];
        }
        if (fq == 0) sMisc[j] = 1.0;
      }
      if (mu == 0.) {
#pragma unroll
        for (int i = 0; i < 12; ++i) fb[i * NQF] = 0.;
#pragma unroll
        for (int r = 0; r < 4; ++r) fz[r * NQF] = 0.;
      }
    }
    __syncthreads();
    if (tid < NH) {  // lifting operator, first face direction
      const int j = tid / NQF, fq = tid % NQF, q1 = fq % P, q2 = fq / P;
      const double* fz = Fz + j * 4 * NQF;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        double s = 0.;
#pragma unroll
        for (int k = 0; k < P; ++k) s = fma(K[q1 * P + k], fz[v * NQF + k + P * q2], s);
        Fz2[(j * 4 + v) * NQF + fq] = s;
      }
    }
    __syncthreads();
    if (tid < NH) {  // second direction; a = (F - Qhat.n) fJ w
      const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, q1 = fq % P, q2 = fq / P;
      const double fw = sg[kGeoFJ + lf] * w1[q1] * w1[q2];
      const double ef = prm.eta * sMisc[j];
      double* fa = Fa + j * 5 * NQF;
      const double* fz2 = Fz2 + j * 4 * NQF;
      fa[fq] *= fw;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        double s = 0.;
#pragma unroll
        for (int k = 0; k < P; ++k) s = fma(K[q2 * P + k], fz2[v * NQF + q1 + P * k], s);
        fa[(v + 1) * NQF + fq] = (fa[(v + 1) * NQF + fq] + ef * s) * fw;
      }
    }
    __syncthreads();
    if (tid < NH) {  // test functions, first tangential direction: items (j, t1, q2)
      const int j = tid / NQF, lf = 3 * half + j, fq = tid % NQF, t1 = fq % P, q2 = fq / P, a = lf >> 1;
      const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
      const double* fa = Fa + j * 5 * NQF;
      const double* fb = Fb + j * 12 * NQF;
      double u1[5], u2[4], un[4];
#pragma unroll
      for (int r = 0; r < 5; ++r) u1[r] = 0.;
#pragma unroll
      for (int r = 0; r < 4; ++r) u2[r] = un[r] = 0.;
#pragma unroll
      for (int q1 = 0; q1 < P; ++q1) {
        const int q = q1 + P * q2;
        const double b = B[q1 * P + t1], bd = Bd[q1 * P + t1];
        u1[0] = fma(b, fa[q], u1[0]);
#pragma unroll
        for (int r = 1; r < 5; ++r) {
          u1[r] = fma(b, fa[r * NQF + q], u1[r]);
          u1[r] = fma(bd, fb[(ax1 * 4 + r - 1) * NQF + q], u1[r]);
          u2[r - 1] = fma(b, fb[(ax2 * 4 + r - 1) * NQF + q], u2[r - 1]);
          un[r - 1] = fma(b, fb[(a * 4 + r - 1) * NQF + q], un[r - 1]);
        }
      }
      double* su = Su + j * 13 * NQF;
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
      const double* su = Su + j * 13 * NQF;
      double c0[5], cn[4];
#pragma unroll
      for (int r = 0; r < 5; ++r) c0[r] = 0.;
#pragma unroll
      for (int r = 0; r < 4; ++r) cn[r] = 0.;
#pragma unroll
      for (int q2 = 0; q2 < P; ++q2) {
        const int q = t1 + P * q2;
        const double b = B[q2 * P + t2], bd = Bd[q2 * P + t2];
        c0[0] = fma(b, su[q], c0[0]);
#pragma unroll
        for (int r = 1; r < 5; ++r) {
          c0[r] = fma(b, su[r * NQF + q], c0[r]);
          c0[r] = fma(bd, su[(4 + r) * NQF + q], c0[r]);
          cn[r - 1] = fma(b, su[(8 + r) * NQF + q], cn[r - 1]);
        }
      }
      double* sc = Sc + j * 9 * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) sc[r * NQF + fq] = c0[r];
#pragma unroll
      for (int r = 0; r < 4; ++r) sc[(5 + r) * NQF + fq] = cn[r];
    }
    __syncthreads();
    if (node) {  // scatter to the node through the normal-direction factors
      const int ix = tid % P, iy = (tid / P) % P, iz = tid / (P * P);
      const double* Ev = so + C::oE;
      const double* Dv = so + C::oD;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int lf = 3 * half + j, a = lf >> 1, end = lf & 1;
        const int ia = a == 0 ? ix : a == 1 ? iy : iz;
        const int t1 = a == 0 ? iy : ix, t2 = a == 2 ? iy : iz;
        const double ev = Ev[end * P + ia], dv = Dv[end * P + ia];
        const double* sc = Sc + j * 9 * NQF + t1 + P * t2;
        Rv[0] += ev * sc[0];
#pragma unroll
        for (int r = 1; r < 5; ++r) Rv[r] += ev * sc[r * NQF] + dv * sc[(4 + r) * NQF];
      }
    }
    __syncthreads();
  }

  // ---------------- norm partial, f = -Minv R (solve.cpp:800-804), RK update
  if (sa.part) {  // sum of R^2 over the element, fixed order
    double s = 0.;
    if (node) {
#pragma unroll
      for (int r = 0; r < 5; ++r) s += Rv[r] * Rv[r];
    }
    double* red = sX;
    red[tid] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.;
      for (int i = 0; i < C::NT; ++i) t += red[i];
      sa.part[e] = t;
    }
    __syncthreads();
  }
  double* M0 = sX;
  double* M1 = sX + 5 * NB;
  const double* Mi = so + C::oMi;
  if (node) {
#pragma unroll
    for (int r = 0; r < 5; ++r) M0[r * NB + tid] = Rv[r];
  }
  __syncthreads();
  if (node) contract<P, 0, false, false>(Mi, M0, M1, tid);
  __syncthreads();
  if (node) contract<P, 1, false, false>(Mi, M1, M0, tid);
  __syncthreads();
  if (node) {
    double f[5];
    contract_reg<P, 2, false>(Mi, M0, tid, f);
    const double sc = -1.0 / detJ;
    const long base = e * 5 * NB;
    const double dt = sa.dt;
    double* sUn = sX + L::oTrU;  // new state for the epilogue traces (disjoint from M0/M1)
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const long i = base + r * NB + tid;
      const double fr = f[r] * sc;
      double un = 0.;
      switch (sa.mode) {
        case MODE_RESIDUAL:
          sa.fout[i] = fr;
          if (sa.Rout) sa.Rout[i] = Rv[r];
          break;
        case MODE_RK4_0:
          sa.acc[i] = fr;
          un = sa.Ubase[i] + dt * fr * 0.5;
          break;
        case MODE_RK4_1:
          sa.acc[i] = sa.acc[i] + 2. * fr;
          un = sa.Ubase[i] + dt * fr * 0.5;
          break;
        case MODE_RK4_2:
          sa.acc[i] = sa.acc[i] + 2. * fr;
          un = sa.Ubase[i] + dt * fr;
          break;
        case MODE_RK4_3:
          un = sa.Ubase[i] + (1. / 6.) * (sa.acc[i] + fr) * dt;
          break;
        case MODE_TVD_0:
          un = sa.Ubase[i] + dt * fr;
          break;
        case MODE_TVD_1:
          un = 0.75 * sa.Ubase[i] + 0.25 * Ue[r * NB + tid] + 0.25 * dt * fr;
          break;
        case MODE_TVD_2:
          un = (1. / 3.) * sa.Ubase[i] + (2. / 3.) * Ue[r * NB + tid] + (2. / 3.) * dt * fr;
          break;
      }
      if (sa.mode != MODE_RESIDUAL) {
        sa.Uout[i] = un;
        sUn[r * NB + tid] = un;
      }
    }
  }
  // ---------------- face traces of the new state for the next stage
  if (sa.Tnext) {
    __syncthreads();
    double* Te = sa.Tnext + e * 60 * NQF;
    trace_half<P>(0, sX + L::oTrU, sX, sX + 30 * NQF, so, sg, prm.mu, Te);
    trace_half<P>(1, sX + L::oTrU, sX, sX + 30 * NQF, so, sg, prm.mu, Te);
  }
}

// sqrt(sum(part) / size) into norms[*counter], deterministic fixed-order sum
__global__ void norm_kernel(long E, const double* __restrict__ part, double inv_size,
                            double* norms, int* counter, int* flag)
{
  __shared__ double red[1024];
  const int tid = threadIdx.x;
  double s = 0.;
  for (long i = tid; i < E; i += blockDim.x) s += part[i];
  red[tid] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid == 0) {
    const int c = *counter;
    const double v = sqrt(red[0] * inv_size);
    norms[c] = v;
    if (!isfinite(v)) *flag |= 1;
    *counter = c + 1;
  }
}

// ------------------------------------------------------------ host launchers

template <int P>
static size_t trace_smem()
{
  using C = Cfg<P>;
  return sizeof(double) * (C::OPSP + kGeoStride + 5 * C::NB + 75 * C::NQF);
}

template <int P>
static size_t stage_smem()
{
  return sizeof(double) * StageSmem<P>::TOTAL;
}

template <int P>
static cudaError_t prepare_p()
{
  cudaError_t e = cudaFuncSetAttribute(trace_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)trace_smem<P>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(stage_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)stage_smem<P>());
}

template <int P>
static cudaError_t launch_trace_p(const Fp64Launch& L, const double* U, double* Tout, cudaStream_t st)
{
  trace_kernel<P><<<(unsigned)L.E, Cfg<P>::NT, trace_smem<P>(), st>>>(L.E, U, L.ops, L.geo, Tout, L.prm);
  return cudaGetLastError();
}

template <int P>
static cudaError_t launch_stage_p(const Fp64Launch& L, const double* Us, const double* Tin,
                                  const StageArgs& sa, cudaStream_t st)
{
  stage_kernel<P><<<(unsigned)L.E, Cfg<P>::NT, stage_smem<P>(), st>>>(L.E, Us, Tin, L.ops, L.geo, L.nbr,
                                                                       L.prm, sa);
  return cudaGetLastError();
}

cudaError_t prepare_fp64_kernels(int P)
{
  switch (P) {
    case 1: return prepare_p<1>();
    case 2: return prepare_p<2>();
    case 3: return prepare_p<3>();
    case 4: return prepare_p<4>();
    case 5: return prepare_p<5>();
    case 6: return prepare_p<6>();
    case 7: return prepare_p<7>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_trace(const Fp64Launch& L, const double* U, double* Tout, cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_trace_p<1>(L, U, Tout, st);
    case 2: return launch_trace_p<2>(L, U, Tout, st);
    case 3: return launch_trace_p<3>(L, U, Tout, st);
    case 4: return launch_trace_p<4>(L, U, Tout, st);
    case 5: return launch_trace_p<5>(L, U, Tout, st);
    case 6: return launch_trace_p<6>(L, U, Tout, st);
    case 7: return launch_trace_p<7>(L, U, Tout, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage(const Fp64Launch& L, const double* Us, const double* Tin, const StageArgs& sa,
                         cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_stage_p<1>(L, Us, Tin, sa, st);
    case 2: return launch_stage_p<2>(L, Us, Tin, sa, st);
    case 3: return launch_stage_p<3>(L, Us, Tin, sa, st);
    case 4: return launch_stage_p<4>(L, Us, Tin, sa, st);
    case 5: return launch_stage_p<5>(L, Us, Tin, sa, st);
    case 6: return launch_stage_p<6>(L, Us, Tin, sa, st);
    case 7: return launch_stage_p<7>(L, Us, Tin, sa, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_norm(long E, const double* part, double inv_size, double* norms, int* counter,
                        int* flag, cudaStream_t st)
{
  norm_kernel<<<1, 1024, 0, st>>>(E, part, inv_size, norms, counter, flag);
  return cudaGetLastError();
}

size_t stage_smem_bytes(int P)
{
  switch (P) {
    case 1: return stage_smem<1>();
    case 2: return stage_smem<2>();
    case 3: return stage_smem<3>();
    case 4: return stage_smem<4>();
    case 5: return stage_smem<5>();
    case 6: return stage_smem<6>();
    case 7: return stage_smem<7>();
  }
  return 0;
}

}  // namespace dgb
