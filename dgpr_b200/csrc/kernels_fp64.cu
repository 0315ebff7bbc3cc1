// FP64 residual / RK-stage kernels for affine hexahedral elements.
//
// One CTA per element.  The tensor-product structure of the basis (equispaced
// Lagrange, basis.cpp:64-170) and of the quadrature (P = p+1 Gauss points per
// direction, geometry_common.cpp:176-177) is used throughout: every
// interpolation / projection is a sequence of 1D P x P contractions on
// shared-memory element tiles (sum factorisation), never the dense nb x nqv
// tables the reference streams from HBM.
//
// Pipeline per RK stage (state layout U[e][r][b], the reference's):
//   trace_kernel : U_s -> face traces T[e][lf][10][P*P]
//                  (5 conserved values and the viscous normal flux
//                   A(U, grad U).n_out at every face quadrature point)
//   stage_kernel : U_s, T -> R (volume + source + faces), f = -Minv R, RK update
// The face kernel of the reference (solve.cpp:393-794) is folded into the
// stage kernel: each element evaluates its own six faces from its own traces
// and its neighbours' traces, so no per-face residual slots are written
// (the reference's FACERESID gather, solve_cuda.cu:1192-1210).
#include <cuda_runtime.h>

#include "kernels.hpp"
#include "physics.cuh"

namespace dgb {

// ------------------------------------------------------------ operator table

template <int P>
struct Cfg {
  static constexpr int NB = P * P * P;       // nodes = volume quadrature points
  static constexpr int NQF = P * P;          // face quadrature points
  static constexpr int NF = 6 * NQF;         // face points of one element
  static constexpr int NTRAW = NB > NF ? NB : NF;
  static constexpr int NT = ((NTRAW + 31) / 32) * 32;
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
//   out[r][o] (+)= sum_k M(a, k) in[r][o with coordinate AX replaced by k]
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

// ------------------------------------------------------------- trace kernel

template <int P>
__global__ void __launch_bounds__(Cfg<P>::NT)
trace_kernel(long E, const double* __restrict__ U, const double* __restrict__ opsg,
             const double* __restrict__ geo, double* __restrict__ Tr, DevParams prm)
{
  using C = Cfg<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NF = C::NF;
  extern __shared__ double sm[];
  double* so = sm;                  // operators
  double* sg = so + C::OPSP;        // element geometry (kGeoStride)
  double* sU = sg + kGeoStride;     // [5][NB]
  double* sN = sU + 5 * NB;         // [6][10][NQF]  normal contraction: value(5), d/dn(5)
  double* sY = sN + 60 * NQF;       // [6][15][NQF]  after t1 contraction
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  for (int i = tid; i < C::OPS; i += blockDim.x) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += blockDim.x) sg[i] = geo[e * kGeoStride + i];
  const double* Ue = U + e * 5 * NB;
  for (int i = tid; i < 5 * NB; i += blockDim.x) sU[i] = Ue[i];
  __syncthreads();
  const bool visc = prm.mu != 0.;

  if (tid < NF) {  // contract along the face normal: value and normal derivative
    const int lf = tid / NQF, fq = tid % NQF, t1 = fq % P, t2 = fq / P, a = lf >> 1, end = lf & 1;
    const double* Ev = so + C::oE + end * P;
    const double* Dv = so + C::oD + end * P;
    double* out = sN + lf * 10 * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double v = 0., dn = 0.;
#pragma unroll
      for (int ia = 0; ia < P; ++ia) {
        const double u = sU[r * NB + face_node<P>(a, ia, t1, t2)];
        v = fma(Ev[ia], u, v);
        dn = fma(Dv[ia], u, dn);
      }
      out[r * NQF + fq] = v;
      out[(5 + r) * NQF + fq] = dn;
    }
  }
  __syncthreads();
  if (tid < NF) {  // contract tangential direction 1 (index q1 = tid % P)
    const int lf = tid / NQF, fq = tid % NQF, q1 = fq % P, t2 = fq / P;
    const double* B = so + C::oB;
    const double* Bd = so + C::oBd;
    const double* in = sN + lf * 10 * NQF;
    double* out = sY + lf * 15 * NQF;
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
  if (tid < NF) {  // contract tangential direction 2, physical gradient, A(U,grad U).n
    const int lf = tid / NQF, fq = tid % NQF, q1 = fq % P, q2 = fq / P, a = lf >> 1;
    const double* B = so + C::oB;
    const double* Bd = so + C::oBd;
    const double* in = sY + lf * 15 * NQF;
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
    if (visc) {
      const double* Ji = sg + kGeoJinv;
      double G[3][5], Q[3][5];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 5; ++r) G[c][r] = Ji[c] * g[0][r] + Ji[3 + c] * g[1][r] + Ji[6 + c] * g[2][r];
      visc_flux(S, G, prm.mu, Q);
      const double* n = sg + kGeoN + 3 * lf;
#pragma unroll
      for (int r = 0; r < 5; ++r) Qn[r] = Q[0][r] * n[0] + Q[1][r] * n[1] + Q[2][r] * n[2];
    }
    double* T = Tr + ((e * 6 + lf) * 10) * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      T[r * NQF + fq] = S[r];
      T[(5 + r) * NQF + fq] = Qn[r];
    }
  }
}

// ------------------------------------------------------------- stage kernel

template <int P>
struct StageSmem {
  using C = Cfg<P>;
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int oOps = 0;
  static constexpr int oGeo = C::OPSP;
  static constexpr int oMisc = oGeo + kGeoStride;      // per-face factors [6], flags
  static constexpr int oU = oMisc + 8;                 // [5][NB]
  static constexpr int oR = oU + 5 * NB;               // [5][NB]
  static constexpr int oX = oR + 5 * NB;               // scratch
  // volume scratch: A[5NB] Bv[5NB] G[15NB]
  static constexpr int VOL = 25 * NB;
  // face scratch: Fa[6][5][NQF] Fb[6][15][NQF] Fz[6][5][NQF] Fz2[6][5][NQF] Su[6][15][NQF]
  // (Sc[6][10][NQF] reuses Fz+Fz2)
  static constexpr int FACE = 270 * NQF;
  static constexpr int X = VOL > FACE ? VOL : FACE;
  static constexpr int TOTAL = oX + X;
};

template <int P>
__global__ void __launch_bounds__(Cfg<P>::NT)
stage_kernel(long E, const double* Us, const double* __restrict__ Tr,
             const double* __restrict__ opsg, const double* __restrict__ geo,
             const int* __restrict__ nbr, DevParams prm, StageArgs sa)
{
  using C = Cfg<P>;
  using L = StageSmem<P>;
  constexpr int NB = C::NB, NQF = C::NQF, NF = C::NF;
  extern __shared__ double sm[];
  double* so = sm + L::oOps;
  double* sg = sm + L::oGeo;
  double* sMisc = sm + L::oMisc;
  double* sU = sm + L::oU;
  double* sR = sm + L::oR;
  double* sX = sm + L::oX;
  const long e = blockIdx.x;
  const int tid = threadIdx.x;

  for (int i = tid; i < C::OPS; i += blockDim.x) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += blockDim.x) sg[i] = geo[e * kGeoStride + i];
  const double* Ue = Us + e * 5 * NB;
  for (int i = tid; i < 5 * NB; i += blockDim.x) sU[i] = Ue[i];
  __syncthreads();

  const double* B = so + C::oB;
  const double* Bd = so + C::oBd;
  const double* Dq = so + C::oDq;
  const double detJ = sg[kGeoDetJ];
  const double* Ji = sg + kGeoJinv;

  // ---------------- volume integral (solve.cpp:276-341) + source (345-360)
  {
    double* sA = sX;
    double* sB = sX + 5 * NB;
    double* sG = sX + 10 * NB;  // [3][5][NB]
    const bool act = tid < NB;
    if (act) contract<P, 0, false, false>(B, sU, sA, tid);
    __syncthreads();
    if (act) contract<P, 1, false, false>(B, sA, sB, tid);
    __syncthreads();
    if (act) contract<P, 2, false, false>(B, sB, sA, tid);  // sA: values at quadrature points
    __syncthreads();
    if (act) {
      contract<P, 0, false, false>(Dq, sA, sG, tid);
      contract<P, 1, false, false>(Dq, sA, sG + 5 * NB, tid);
      contract<P, 2, false, false>(Dq, sA, sG + 10 * NB, tid);
    }
    __syncthreads();
    if (act) {  // pointwise flux at quadrature point tid
      const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);
      const double* w = so + C::oW;
      const double wJ = w[qx] * w[qy] * w[qz] * detJ;
      double S[5], G[3][5], H[3][5];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        S[r] = sA[r * NB + tid];
        const double g0 = sG[r * NB + tid], g1 = sG[5 * NB + r * NB + tid], g2 = sG[10 * NB + r * NB + tid];
#pragma unroll
        for (int c = 0; c < 3; ++c) G[c][r] = Ji[c] * g0 + Ji[3 + c] * g1 + Ji[6 + c] * g2;
      }
      euler_flux(S, prm.gamma, H);
      if (prm.mu != 0.) {
        double Q[3][5];
        visc_flux(S, G, prm.mu, Q);
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
          sG[i * 5 * NB + r * NB + tid] = wJ * (Ji[3 * i] * H[0][r] + Ji[3 * i + 1] * H[1][r] + Ji[3 * i + 2] * H[2][r]);
    }
    __syncthreads();
    if (act) {  // sum_i Dq_i^T Ghat_i
      contract<P, 0, true, false>(Dq, sG, sB, tid);
      contract<P, 1, true, true>(Dq, sG + 5 * NB, sB, tid);
      contract<P, 2, true, true>(Dq, sG + 10 * NB, sB, tid);
    }
    __syncthreads();
    if (act) contract<P, 0, true, false>(B, sB, sA, tid);
    __syncthreads();
    if (act) contract<P, 1, true, false>(B, sA, sB, tid);
    __syncthreads();
    if (act) {
      contract<P, 2, true, false>(B, sB, sR, tid);
      const double* Wb = so + C::oWb;
      const int ix = tid % P, iy = (tid / P) % P, iz = tid / (P * P);
      const double ws = Wb[ix] * Wb[iy] * Wb[iz] * detJ;
#pragma unroll
      for (int r = 0; r < 5; ++r) sR[r * NB + tid] -= prm.src[r] * ws;
    }
    __syncthreads();
  }

  // ---------------- faces (solve.cpp:393-794)
  {
    double* sFa = sX;                  // [6][5][NQF]
    double* sFb = sFa + 30 * NQF;      // [6][15][NQF]  reference-space dual-consistency vectors
    double* sFz = sFb + 90 * NQF;      // [6][5][NQF]   lifting source
    double* sFz2 = sFz + 30 * NQF;     // [6][5][NQF]
    double* sSu = sFz2 + 30 * NQF;     // [6][15][NQF]
    double* sSc = sFz;                 // [6][10][NQF]  (reuses Fz, Fz2)
    const double gamma = prm.gamma, mu = prm.mu;
    if (tid < NF) {
      const int lf = tid / NQF, fq = tid % NQF, q1 = fq % P, q2 = fq / P, end = lf & 1;
      const double* w = so + C::oW;
      const double* n = sg + kGeoN + 3 * lf;
      const double fw = sg[kGeoFJ + lf] * w[q1] * w[q2];
      const double* To = Tr + ((e * 6 + lf) * 10) * NQF;
      double Uo[5], Qo[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        Uo[r] = To[r * NQF + fq];
        Qo[r] = To[(5 + r) * NQF + fq];
      }
      const int nb = nbr[e * 6 + lf];
      double F[5], ap[5], z[5], dc[3][5];
      if (nb >= 0) {
        const double* Tn = Tr + (((long)nb * 6 + (lf ^ 1)) * 10) * NQF;
        double Un[5], Qnb[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          Un[r] = Tn[r * NQF + fq];
          Qnb[r] = Tn[(5 + r) * NQF + fq];
        }
        // Roe flux in one orientation for both sides: the element that sees
        // the face on its high side is "left"
        if (end) {
          roe_flux(Uo, Un, n, gamma, F);
        } else {
          const double nn[3] = {-n[0], -n[1], -n[2]};
          roe_flux(Un, Uo, nn, gamma, F);
#pragma unroll
          for (int r = 0; r < 5; ++r) F[r] = -F[r];
        }
        // dual consistency A(Uo, (Uo - Uhat) n)
        double dd[5], jmp[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          dd[r] = Uo[r] - 0.5 * (Uo[r] + Un[r]);
          jmp[r] = Uo[r] - Un[r];
        }
        if (mu != 0.) {
          visc_rank1(Uo, dd, n, mu, dc);
          // BR2 lifting sources of both sides, weighted by their inverse-mass factor
          double ro[5], rn[5];
          visc_jump_n(Uo, jmp, n, mu, ro);
          visc_jump_n(Un, jmp, n, mu, rn);
          const double co = so[C::oC + end] / detJ;
          const double cn = so[C::oC + (end ^ 1)] / geo[(long)nb * kGeoStride + kGeoDetJ];
#pragma unroll
          for (int r = 0; r < 5; ++r) z[r] = (co * (0.5 * ro[r]) + cn * (0.5 * rn[r])) * fw;
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 5; ++r) dc[c][r] = 0.;
#pragma unroll
          for (int r = 0; r < 5; ++r) z[r] = 0.;
        }
#pragma unroll
        for (int r = 0; r < 5; ++r) ap[r] = F[r] - 0.5 * (Qo[r] - Qnb[r]);
        if (fq == 0) sMisc[lf] = 0.5;
      } else {
        double Ub[5];
        const int bad = boundary_state(nb, Uo, n, prm, Ub);
        if (bad && sa.flag) atomicOr(sa.flag, 2);
        euler_flux_n(Ub, gamma, n, F);
        double dd[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) dd[r] = Uo[r] - Ub[r];
        if (mu != 0.) {
          visc_rank1(Uo, dd, n, mu, dc);
          double rb[5];
          visc_jump_n(Ub, dd, n, mu, rb);
          const double co = so[C::oC + end] / detJ;
#pragma unroll
          for (int r = 0; r < 5; ++r) z[r] = co * rb[r] * fw;
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 5; ++r) dc[c][r] = 0.;
#pragma unroll
          for (int r = 0; r < 5; ++r) z[r] = 0.;
        }
#pragma unroll
        for (int r = 0; r < 5; ++r) ap[r] = F[r] - Qo[r];
        if (fq == 0) sMisc[lf] = 1.0;
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        sFa[(lf * 5 + r) * NQF + fq] = ap[r];
        sFz[(lf * 5 + r) * NQF + fq] = z[r];
      }
      // -grad(phi) . dc  ->  reference-space vector b_i = -fw sum_c Jinv[i][c] dc[c]
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int r = 0; r < 5; ++r)
          sFb[(lf * 15 + i * 5 + r) * NQF + fq] =
              -fw * (Ji[3 * i] * dc[0][r] + Ji[3 * i + 1] * dc[1][r] + Ji[3 * i + 2] * dc[2][r]);
    }
    __syncthreads();
    const double* K = so + C::oK;
    if (tid < NF) {  // lifting operator, first face direction
      const int lf = tid / NQF, fq = tid % NQF, q1 = fq % P, q2 = fq / P;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        double s = 0.;
#pragma unroll
        for (int k = 0; k < P; ++k) s = fma(K[q1 * P + k], sFz[(lf * 5 + r) * NQF + k + P * q2], s);
        sFz2[(lf * 5 + r) * NQF + fq] = s;
      }
    }
    __syncthreads();
    if (tid < NF) {  // second direction; a = (F - Qhat.n) fJ w
      const int lf = tid / NQF, fq = tid % NQF, q1 = fq % P, q2 = fq / P;
      const double* w = so + C::oW;
      const double fw = sg[kGeoFJ + lf] * w[q1] * w[q2];
      const double ef = prm.eta * sMisc[lf];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        double s = 0.;
#pragma unroll
        for (int k = 0; k < P; ++k) s = fma(K[q2 * P + k], sFz2[(lf * 5 + r) * NQF + q1 + P * k], s);
        sFa[(lf * 5 + r) * NQF + fq] = (sFa[(lf * 5 + r) * NQF + fq] + ef * s) * fw;
      }
    }
    __syncthreads();
    if (tid < NF) {  // test functions, first tangential direction: items (lf, t1, q2)
      const int lf = tid / NQF, fq = tid % NQF, t1 = fq % P, q2 = fq / P, a = lf >> 1;
      const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
      const double* fa = sFa + lf * 5 * NQF;
      const double* fb = sFb + lf * 15 * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        double u1 = 0., u2 = 0., un = 0.;
#pragma unroll
        for (int q1 = 0; q1 < P; ++q1) {
          const int q = q1 + P * q2;
          const double b = B[q1 * P + t1], bd = Bd[q1 * P + t1];
          u1 = fma(b, fa[r * NQF + q], u1);
          u1 = fma(bd, fb[(ax1 * 5 + r) * NQF + q], u1);
          u2 = fma(b, fb[(ax2 * 5 + r) * NQF + q], u2);
          un = fma(b, fb[(a * 5 + r) * NQF + q], un);
        }
        sSu[(lf * 15 + r) * NQF + fq] = u1;
        sSu[(lf * 15 + 5 + r) * NQF + fq] = u2;
        sSu[(lf * 15 + 10 + r) * NQF + fq] = un;
      }
    }
    __syncthreads();
    if (tid < NF) {  // second tangential direction: items (lf, t1, t2)
      const int lf = tid / NQF, fq = tid % NQF, t1 = fq % P, t2 = fq / P;
      const double* su = sSu + lf * 15 * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        double c0 = 0., cn = 0.;
#pragma unroll
        for (int q2 = 0; q2 < P; ++q2) {
          const int q = t1 + P * q2;
          const double b = B[q2 * P + t2], bd = Bd[q2 * P + t2];
          c0 = fma(b, su[r * NQF + q], c0);
          c0 = fma(bd, su[(5 + r) * NQF + q], c0);
          cn = fma(b, su[(10 + r) * NQF + q], cn);
        }
        sSc[(lf * 10 + r) * NQF + fq] = c0;
        sSc[(lf * 10 + 5 + r) * NQF + fq] = cn;
      }
    }
    __syncthreads();
    if (tid < NB) {  // scatter to the element's nodes through the normal-direction factors
      const int ix = tid % P, iy = (tid / P) % P, iz = tid / (P * P);
      const double* Ev = so + C::oE;
      const double* Dv = so + C::oD;
      double acc[5] = {0., 0., 0., 0., 0.};
#pragma unroll
      for (int lf = 0; lf < 6; ++lf) {
        const int a = lf >> 1, end = lf & 1;
        const int ia = a == 0 ? ix : a == 1 ? iy : iz;
        const int t1 = a == 0 ? iy : ix, t2 = a == 2 ? iy : iz;
        const double ev = Ev[end * P + ia], dv = Dv[end * P + ia];
        const int fq = t1 + P * t2;
#pragma unroll
        for (int r = 0; r < 5; ++r)
          acc[r] += ev * sSc[(lf * 10 + r) * NQF + fq] + dv * sSc[(lf * 10 + 5 + r) * NQF + fq];
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) sR[r * NB + tid] += acc[r];
    }
    __syncthreads();
  }

  // ---------------- norm partial, f = -Minv R (solve.cpp:800-804), RK update
  {
    if (sa.part) {  // sum of R^2 over the element, fixed order
      double s = 0.;
      if (tid < NB) {
#pragma unroll
        for (int r = 0; r < 5; ++r) s += sR[r * NB + tid] * sR[r * NB + tid];
      }
      double* red = sX;  // scratch is free here
      red[tid] = s;
      __syncthreads();
      if (tid == 0) {
        double t = 0.;
        for (int i = 0; i < blockDim.x; ++i) t += red[i];
        sa.part[e] = t;
      }
      __syncthreads();
    }
    double* sA = sX;
    double* sB = sX + 5 * NB;
    const double* Mi = so + C::oMi;
    const bool act = tid < NB;
    if (act) contract<P, 0, false, false>(Mi, sR, sA, tid);
    __syncthreads();
    if (act) contract<P, 1, false, false>(Mi, sA, sB, tid);
    __syncthreads();
    if (act) {
      contract<P, 2, false, false>(Mi, sB, sA, tid, -1.0 / detJ);  // sA = f
      const long base = e * 5 * NB;
      const double dt = sa.dt;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const long i = base + r * NB + tid;
        const double f = sA[r * NB + tid];
        switch (sa.mode) {
          case MODE_RESIDUAL:
            sa.fout[i] = f;
            if (sa.Rout) sa.Rout[i] = sR[r * NB + tid];
            break;
          case MODE_RK4_0:
            sa.acc[i] = f;
            sa.Uout[i] = sa.Ubase[i] + dt * f * 0.5;
            break;
          case MODE_RK4_1:
            sa.acc[i] = sa.acc[i] + 2. * f;
            sa.Uout[i] = sa.Ubase[i] + dt * f * 0.5;
            break;
          case MODE_RK4_2:
            sa.acc[i] = sa.acc[i] + 2. * f;
            sa.Uout[i] = sa.Ubase[i] + dt * f;
            break;
          case MODE_RK4_3:
            sa.Uout[i] = sa.Ubase[i] + (1. / 6.) * (sa.acc[i] + f) * dt;
            break;
          case MODE_TVD_0:
            sa.Uout[i] = sa.Ubase[i] + dt * f;
            break;
          case MODE_TVD_1:
            sa.Uout[i] = 0.75 * sa.Ubase[i] + 0.25 * sU[r * NB + tid] + 0.25 * dt * f;
            break;
          case MODE_TVD_2:
            sa.Uout[i] = (1. / 3.) * sa.Ubase[i] + (2. / 3.) * sU[r * NB + tid] + (2. / 3.) * dt * f;
            break;
        }
      }
    }
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
  return sizeof(double) * (C::OPSP + kGeoStride + 5 * C::NB + 60 * C::NQF + 90 * C::NQF);
}

template <int P>
static cudaError_t prepare_p()
{
  cudaError_t e = cudaFuncSetAttribute(trace_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)trace_smem<P>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(stage_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(double) * StageSmem<P>::TOTAL));
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

template <int P>
static cudaError_t launch_trace_p(const Fp64Launch& L, const double* U, cudaStream_t st)
{
  using C = Cfg<P>;
  const size_t smem = trace_smem<P>();
  trace_kernel<P><<<(unsigned)L.E, C::NT, smem, st>>>(L.E, U, L.ops, L.geo, L.trace, L.prm);
  return cudaGetLastError();
}

template <int P>
static cudaError_t launch_stage_p(const Fp64Launch& L, const double* Us, const StageArgs& sa,
                                  cudaStream_t st)
{
  using C = Cfg<P>;
  const size_t smem = sizeof(double) * StageSmem<P>::TOTAL;
  stage_kernel<P><<<(unsigned)L.E, C::NT, smem, st>>>(L.E, Us, L.trace, L.ops, L.geo, L.nbr, L.prm, sa);
  return cudaGetLastError();
}

cudaError_t launch_trace(const Fp64Launch& L, const double* U, cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_trace_p<1>(L, U, st);
    case 2: return launch_trace_p<2>(L, U, st);
    case 3: return launch_trace_p<3>(L, U, st);
    case 4: return launch_trace_p<4>(L, U, st);
    case 5: return launch_trace_p<5>(L, U, st);
    case 6: return launch_trace_p<6>(L, U, st);
    case 7: return launch_trace_p<7>(L, U, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage(const Fp64Launch& L, const double* Us, const StageArgs& sa, cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_stage_p<1>(L, Us, sa, st);
    case 2: return launch_stage_p<2>(L, Us, sa, st);
    case 3: return launch_stage_p<3>(L, Us, sa, st);
    case 4: return launch_stage_p<4>(L, Us, sa, st);
    case 5: return launch_stage_p<5>(L, Us, sa, st);
    case 6: return launch_stage_p<6>(L, Us, sa, st);
    case 7: return launch_stage_p<7>(L, Us, sa, st);
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
    case 1: return sizeof(double) * StageSmem<1>::TOTAL;
    case 2: return sizeof(double) * StageSmem<2>::TOTAL;
    case 3: return sizeof(double) * StageSmem<3>::TOTAL;
    case 4: return sizeof(double) * StageSmem<4>::TOTAL;
    case 5: return sizeof(double) * StageSmem<5>::TOTAL;
    case 6: return sizeof(double) * StageSmem<6>::TOTAL;
    case 7: return sizeof(double) * StageSmem<7>::TOTAL;
  }
  return 0;
}

}  // namespace dgb
