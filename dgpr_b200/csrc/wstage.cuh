// The Gauss-point stage with a group of warps per element: one warp at p = 3
// (64 Gauss points, two per lane; 16 face points per face, two faces per
// pass, one per lane), two at p = 4 (125 Gauss points; 50 face points a pass;
// the group on a named barrier).  A CTA holds two independent elements, one
// per group, sharing the operator table: the only block barrier is the one
// after the table is loaded, and the phases of an element are ordered by its
// group's own synchronization.  The arithmetic is the
// element-per-CTA kernel's own (vpoint_flux, load_face_point,
// face_point_fluxes, vtrace_half, rk_stage_apply in the same order), so the
// state comes out bit for bit the same; only the per-element residual norm
// partial is summed in another order.
#pragma once

#include "vspace.cuh"

namespace dgb {

template <int P, class T>
struct WStageSmem {
  using C = Cfg<P>;
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int ST = (int)sizeof(T);
  static constexpr int FPW = 2;                // faces per pass
  static constexpr int GT = P <= 4 ? 32 : 64;  // threads per element
  static constexpr int OPSB = align16(C::OPS * ST);
  // per element: [geometry | Y (V first) : 5 NB | R]
  static constexpr int eGeo = 0;
  static constexpr int eY = align16(kGeoStride * ST);
  static constexpr int eR = eY + align16(5 * NB * ST);
  // R: gradients, then contravariant fluxes G[3][5][NB]; the face buffers
  // Fa[FPW][5][NQF] Fb[FPW][12][NQF] Gt[FPW][9][NQF]; the norm's two nodal
  // buffers [2][5][NB]; the new state [5][LS P^2] (x-lines LS apart,
  // tile_node) and the trace scratch [FPW][10][NQF]
  static constexpr int LS = P == 4 ? P + 1 : P;
  static constexpr int RG = 15 * NB * ST;
  static constexpr int RF = FPW * 26 * NQF * ST;
  static constexpr int RN = 10 * NB * ST;
  static constexpr int RT = 5 * LS * P * P * ST + FPW * 10 * NQF * ST;
  static constexpr int RMAX = RG > RF ? (RG > RN ? (RG > RT ? RG : RT) : (RN > RT ? RN : RT))
                                      : (RF > RN ? (RF > RT ? RF : RT) : (RN > RT ? RN : RT));
  static constexpr int eRed = eR + align16(RMAX);  // per-warp sums of the norm partial
  static constexpr int eNb = eRed + 16;              // the neighbours across the six faces
  static constexpr int ELEM = eNb + 32;
  static constexpr int TOTAL = OPSB + kWarpElems * ELEM;
};

// The sum over a group's threads of one value each, in a fixed order; valid
// in thread 0 of the group.
template <int GT>
__device__ __forceinline__ double group_sum(double s, int t, double* slots, int bar)
{
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
  if constexpr (GT > 32) {
    if ((t & 31) == 0) slots[t >> 5] = s;
    group_sync<GT>(bar);
    if (t == 0)
      for (int w = 1; w < GT / 32; ++w) s += slots[w];
    group_sync<GT>(bar);
  }
  return s;
}

template <int P, class T, bool CV, bool HT>
__global__ void __launch_bounds__(WStageSmem<P, T>::GT * kWarpElems, (MinBlocks<P, T>::value))
wstage_kernel(long E, const double* Vs, const T* __restrict__ Tr, const T* __restrict__ opsg,
              const double* __restrict__ opsd, const double* __restrict__ geo, const double* __restrict__ gv,
              const double* __restrict__ gf, const int* __restrict__ nbr, DevParams prm, StageArgs sa)
{
  using C = Cfg<P>;
  using L = WStageSmem<P, T>;
  constexpr int NB = C::NB, NQF = C::NQF, FPW = L::FPW, NH = FPW * NQF;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw);
  for (int i = threadIdx.x; i < C::OPS; i += blockDim.x) so[i] = opsg[i];
  __syncthreads();  // the operator table, shared by the CTA's elements
  constexpr int GT = L::GT;
  const int grp = threadIdx.x / GT, lt = threadIdx.x % GT, bar = 1 + grp;  // element group, thread in it
  const long u = (long)kWarpElems * blockIdx.x + grp;
  if (u >= (sa.ecount ? sa.ecount : E)) return;
  const long e = sa.ebase + sa.estep * u;
  unsigned char* eb = smraw + L::OPSB + grp * L::ELEM;
  T* sg = reinterpret_cast<T*>(eb + L::eGeo);
  T* Y = reinterpret_cast<T*>(eb + L::eY);  // the state V first, the Gauss-point residual Y later
  T* V1 = Y;
  T* R = reinterpret_cast<T*>(eb + L::eR);
  T* G = R;

  // L2 prefetch of the traces and RK operands read later: FP64 on affine
  // elements only (on curved elements, and in FP32, measured 1-3% faster
  // without, once the operands were loaded ahead of the stores)
  constexpr bool kPrefetch = DGB_PREFETCH_L2 && sizeof(T) == 8 && !CV;
  int* sNb = reinterpret_cast<int*>(eb + L::eNb);
  if (lt < 6) {  // the neighbours, read by the face passes from shared memory
    const int nb = nbr[e * 6 + lt];
    sNb[lt] = nb;
    if (nb >= 0 && kPrefetch) {
      prefetch_l2(geo + (long)nb * kGeoStride + kGeoDetJ);
      prefetch_range(Tr + ((long)nb * 6 + (lt ^ 1)) * 10 * NQF, 10L * NQF * sizeof(T), 0, 1);
    }
  }
  if (kPrefetch) {  // data read much later
    prefetch_range(Tr + e * 60 * NQF, 60L * NQF * sizeof(T), lt, GT);
    if (sa.Ubase) prefetch_range(sa.Ubase + e * 5 * NB, 40L * NB, lt, GT);
    if (sa.acc && sa.mode >= MODE_RK4_1 && sa.mode <= MODE_RK4_3) prefetch_range(sa.acc + e * 5 * NB, 40L * NB, lt, GT);
  }
  const double* Ve = Vs + e * 5 * NB;
  constexpr int NVL = (5 * NB + GT - 1) / GT;  // state entries per thread
  double vl[NVL];
  load_spread<5 * NB, GT>(Ve, lt, vl);
  for (int i = lt; i < kGeoStride; i += GT) sg[i] = T(geo[e * kGeoStride + i]);
#pragma unroll
  for (int k = 0; k < NVL; ++k) {
    const int i = lt + k * GT;
    if (i < 5 * NB) V1[i] = T(vl[k]);
  }
  group_sync<GT>(bar);

  const T* Dq = so + C::oDq;
  const T* w = so + C::oW;
  const double detJd = geo[e * kGeoStride + kGeoDetJ];
  const T detJ = sg[kGeoDetJ];
  const T* Ji = sg + kGeoJinv;
  const T gamma = T(prm.gamma), mu = T(prm.mu), kq = HT ? T(prm.kq) : T(0);
  const double* gve = CV ? gv + e * kVolC * NB : nullptr;
  const double* gfe = CV ? gf + e * 6 * kFaceC * NQF : nullptr;

  // ---------------- volume integral (solve.cpp:276-341) + source (345-360)
  for (int o = lt; o < NB; o += GT) {  // reference gradients
    contract<P, 0, false, false>(Dq, V1, G, o);
    contract<P, 1, false, false>(Dq, V1, G + 5 * NB, o);
    contract<P, 2, false, false>(Dq, V1, G + 10 * NB, o);
  }
  group_sync<GT>(bar);
  for (int o = lt; o < NB; o += GT)  // pointwise flux at o, in place of its gradients
    vpoint_flux<P, T, CV, false>(so, V1, G, Ji, detJ, gve, gamma, mu, kq, o,
                                 [&](int i, int r, T v) { G[i * 5 * NB + r * NB + o] = v; });
  group_sync<GT>(bar);
  // This thread's face point in each face pass (one at most: NH <= GT) and
  // its loads: its traces and the neighbour's as load_face_point, the
  // neighbour from shared memory.  (Issuing a pass's loads a phase ahead,
  // during the volume divergence or the previous pass's test-function
  // phases, measured 4-5% slower: the registers held across them spill.)
  static_assert(NH <= GT, "one face point per thread and pass");
  const bool fp = lt < NH;
  const int fj = lt / NQF, fq0 = lt % NQF;
  T Uo[5], Qo[5], Un[5], Qn[5], lift_n;
  auto load_face = [&](int pass) {
    const int lf = FPW * pass + fj, nb = sNb[lf];
    const T* To = Tr + ((e * 6 + lf) * 10) * NQF;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      Uo[r] = To[r * NQF + fq0];
      Qo[r] = To[(5 + r) * NQF + fq0];
    }
    lift_n = T(0);
    if (nb >= 0) {
      const T* Tn = Tr + (((long)nb * 6 + (lf ^ 1)) * 10) * NQF;
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        Un[r] = Tn[r * NQF + fq0];
        Qn[r] = Tn[(5 + r) * NQF + fq0];
      }
      if constexpr (CV)
        lift_n = T(gf[(((long)nb * 6 + (lf ^ 1)) * kFaceC + kFaceLift) * NQF + fq0]);
      else
        lift_n = so[C::oC + ((lf & 1) ^ 1)] / T(geo[(long)nb * kGeoStride + kGeoDetJ]);
    }
  };
  for (int o = lt; o < NB; o += GT) {  // Y = sum_i Dq_i^T Ghat_i minus the source tested with w detJ (over V)
    const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
    const T wJq = w[qx] * w[qy] * w[qz] * (CV ? T(gve[kVolDetJ * NB + o]) : detJ);
    T rv[5], y[5];
    contract_reg<P, 0, true>(Dq, G, o, rv);
    contract_reg<P, 1, true>(Dq, G + 5 * NB, o, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) rv[r] += y[r];
    contract_reg<P, 2, true>(Dq, G + 10 * NB, o, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) Y[r * NB + o] = rv[r] + y[r] - T(prm.src[r]) * wJq;
  }
  group_sync<GT>(bar);

  // ---------------- faces (solve.cpp:393-794), FPW at a time
  T* Fa = R;                    // [FPW][5][NQF]
  T* Fb = Fa + FPW * 5 * NQF;   // [FPW][12][NQF]
  T* Gt = Fb + FPW * 12 * NQF;  // [FPW][9][NQF]
#pragma unroll 1
  for (int pass = 0; pass < 6 / FPW; ++pass) {
    if (fp) {
      load_face(pass);
      const int lf = FPW * pass + fj;
      face_point_fluxes<P, T, CV>(lf, fq0, sNb[lf], Uo, Qo, Un, Qn, lift_n, so, sg, gfe, prm, gamma, mu, kq, detJ,
                                  Ji, sa.flag, Fa + fj * 5 * NQF + fq0, Fb + fj * 12 * NQF + fq0);
    }
    group_sync<GT>(bar);
#pragma unroll 1
    for (int i = lt; i < NH; i += GT) {  // tangential test derivatives: g = fa + Dq^T fb_ax1 + Dq^T fb_ax2, h = fb_a
      const int j = i / NQF, lf = FPW * pass + j, fq = i % NQF, t1 = fq % P, t2 = fq / P, a = lf >> 1;
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
    group_sync<GT>(bar);
    for (int o = lt; o < NB; o += GT) {  // each Gauss point gathers from the face points on its normal lines
      const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
      const T* Ev = so + C::oEh;
      const T* Dv = so + C::oDh;
      T rv[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) rv[r] = Y[r * NB + o];
#pragma unroll
      for (int j = 0; j < FPW; ++j) {
        const int lf = FPW * pass + j, a = lf >> 1, end = lf & 1;
        const int qa = a == 0 ? qx : a == 1 ? qy : qz;
        const int t1 = a == 0 ? qy : qx, t2 = a == 2 ? qy : qz;
        const T ev = Ev[end * P + qa], dv = Dv[end * P + qa];
        const T* gt = Gt + j * 9 * NQF + t1 + P * t2;
        rv[0] += ev * gt[0];
#pragma unroll
        for (int r = 1; r < 5; ++r) rv[r] += ev * gt[r * NQF] + dv * gt[(4 + r) * NQF];
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) Y[r * NB + o] = rv[r];
    }
    group_sync<GT>(bar);
  }

  // ---------------- norm partial: the nodal residual R = B3^T Y
  if (sa.part) {
    const T* B = so + C::oB;
    T* A0 = R;
    T* A1 = R + 5 * NB;
    for (int o = lt; o < NB; o += GT) contract<P, 0, true, false>(B, Y, A0, o);
    group_sync<GT>(bar);
    for (int o = lt; o < NB; o += GT) contract<P, 1, true, false>(B, A0, A1, o);
    group_sync<GT>(bar);
    double s = 0.;
    for (int o = lt; o < NB; o += GT) {
      T rn[5];
      contract_reg<P, 2, true>(B, A1, o, rn);
#pragma unroll
      for (int r = 0; r < 5; ++r) s += double(rn[r]) * double(rn[r]);
    }
    s = group_sum<GT>(s, lt, reinterpret_cast<double*>(eb + L::eRed), bar);
    if (lt == 0) sa.part[e] = s;
    group_sync<GT>(bar);
  }

  // ---------------- f_V = -Y / (w detJ) in FP64, RK update
  T* sVn = R;  // the new state for the epilogue traces
  constexpr int LS = L::LS;
  constexpr int NPT = (NB + GT - 1) / GT;  // Gauss points per thread
  const long base = e * 5 * NB;
  const double* wd = opsd + C::oW;
  auto point_scale = [&](int o) {
    const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
    const double jd = CV ? gve[kVolDetJ * NB + o] : detJd;
    return -1.0 / (wd[qx] * wd[qy] * wd[qz] * jd);
  };
  if (sa.mode == MODE_RESIDUAL) {
    for (int o = lt; o < NB; o += GT) {
      const double sc = point_scale(o);
#pragma unroll
      for (int r = 0; r < 5; ++r) sa.fout[base + r * NB + o] = double(Y[r * NB + o]) * sc;
    }
  } else {
    RkOperands q[NPT][5];
#pragma unroll
    for (int k = 0; k < NPT; ++k) {
      const int o = lt + k * GT;
      if (o < NB)
#pragma unroll
        for (int r = 0; r < 5; ++r) q[k][r] = rk_stage_load(sa, base + r * NB + o, Ve + r * NB + o);
    }
#pragma unroll
    for (int k = 0; k < NPT; ++k) {
      const int o = lt + k * GT;
      if (o < NB) {
        const double sc = point_scale(o);
        const int on = o + (LS - P) * (o / P);  // o in the tile with x-lines LS apart
#pragma unroll
        for (int r = 0; r < 5; ++r) {
          const double un = rk_stage_apply(sa, base + r * NB + o, double(Y[r * NB + o]) * sc, q[k][r]);
          sa.Uout[base + r * NB + o] = un;
          sVn[r * LS * P * P + on] = T(un);
        }
      }
    }
  }
  // ---------------- face traces of the new state for the next stage
  if (sa.Tnext) {
    group_sync<GT>(bar);
    T* Te = reinterpret_cast<T*>(sa.Tnext) + e * 60 * NQF;
    T* sN = R + 5 * LS * P * P;
#pragma unroll 1
    for (int pass = 0; pass < 6 / FPW; ++pass) {
      if (pass) group_sync<GT>(bar);
      vtrace_half<P, T, CV, FPW, GT, LS>(pass, sVn, sN, so, sg, mu, kq, Te, gfe, bar);
    }
  }
}

// The paired mixed stage (vstage2_kernel: two elements per thread in FP32x2)
// with a group of warps per pair: a CTA holds two independent pairs, one per
// group, sharing the operator tables.  Same arithmetic as vstage2_kernel.
// Used at p = 3 (one warp a pair) and p = 4 (two warps a pair).
template <int P>
struct WPairSmem {
  using C = Cfg<P>;
  static constexpr int NB = C::NB, NQF = C::NQF;
  static constexpr int FPW = 2;
  static constexpr int GT = P <= 4 ? 32 : 64;                // threads per pair
  static constexpr int oOpsF = align16(C::OPS * 8);         // after the f2 table
  static constexpr int OPSB = oOpsF + align16(C::OPS * 4);  // f2 and float operator tables
  // per pair: [f2 geometry | float geometry of each element | Y : 5 NB | R]
  static constexpr int eGeo = 0;
  static constexpr int eGeoF = align16(kGeoStride * 8);
  static constexpr int eY = eGeoF + align16(2 * kGeoStride * 4);
  static constexpr int eR = eY + align16(5 * NB * 8);
  static constexpr int RG = 15 * NB * 8;
  static constexpr int RF = FPW * 26 * NQF * 8;
  static constexpr int RN = 10 * NB * 8;
  static constexpr int LS = P == 4 ? P + 1 : P;  // x-line stride of the new state's tile (tile_node)
  static constexpr int RT = 5 * LS * P * P * 8 + FPW * 10 * NQF * 8;
  static constexpr int RMAX = RG > RF ? (RG > RN ? (RG > RT ? RG : RT) : (RN > RT ? RN : RT))
                                      : (RF > RN ? (RF > RT ? RF : RT) : (RN > RT ? RN : RT));
  static constexpr int eRed = eR + align16(RMAX);  // per-warp sums of the norm partials
  static constexpr int ELEM = eRed + 32;
  static constexpr int TOTAL = OPSB + kWarpElems * ELEM;
};

template <int P, bool HT>
__global__ void __launch_bounds__(WPairSmem<P>::GT * kWarpElems, (MinBlocksPair<P>::value))
wstage2_kernel(long E, const double* Vs, const f2* __restrict__ Tr2, const float* __restrict__ opsg,
               const double* __restrict__ opsd, const double* __restrict__ geo, const int* __restrict__ nbr,
               DevParams prm, StageArgs sa)
{
  using C = Cfg<P>;
  using L = WPairSmem<P>;
  using T = f2;
  constexpr int NB = C::NB, NQF = C::NQF, FPW = L::FPW, NH = FPW * NQF, GT = L::GT;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw);
  float* sof = reinterpret_cast<float*>(smraw + L::oOpsF);
  for (int i = threadIdx.x; i < C::OPS; i += blockDim.x) {
    so[i] = T(opsg[i]);
    sof[i] = opsg[i];
  }
  __syncthreads();  // the operator tables, shared by the CTA's pairs
  const int grp = threadIdx.x / GT, lt = threadIdx.x % GT, bar = 1 + grp;  // pair group, thread in it
  const long u = (long)kWarpElems * blockIdx.x + grp;
  if (u >= (sa.ecount ? sa.ecount : E) / 2) return;
  const long k = sa.ebase + sa.estep * u, e0 = 2 * k;
  const long el[2] = {e0, e0 + 1};
  unsigned char* eb = smraw + L::OPSB + grp * L::ELEM;
  T* sg = reinterpret_cast<T*>(eb + L::eGeo);
  float* sgf = reinterpret_cast<float*>(eb + L::eGeoF);  // [2][kGeoStride]
  T* Y = reinterpret_cast<T*>(eb + L::eY);
  T* V1 = Y;
  T* R = reinterpret_cast<T*>(eb + L::eR);
  T* G = R;

  // (no L2 prefetch of the data read later, unlike the FP64 warp stage:
  // measured 1% faster without at p = 3, once the operands were loaded
  // ahead of the stores)
  const double* Ve0 = Vs + el[0] * 5 * NB;
  const double* Ve1 = Vs + el[1] * 5 * NB;
  constexpr int NVL = (5 * NB + GT - 1) / GT;  // state entries per thread and element
  double v0[NVL], v1[NVL];
  load_spread<5 * NB, GT>(Ve0, lt, v0);
  load_spread<5 * NB, GT>(Ve1, lt, v1);
  for (int i = lt; i < kGeoStride; i += GT) {
    const float g0 = (float)geo[el[0] * kGeoStride + i], g1 = (float)geo[el[1] * kGeoStride + i];
    sg[i] = T(g0, g1);
    sgf[i] = g0;
    sgf[kGeoStride + i] = g1;
  }
#pragma unroll
  for (int k = 0; k < NVL; ++k)
    if (lt + k * GT < 5 * NB) V1[lt + k * GT] = T((float)v0[k], (float)v1[k]);
  group_sync<GT>(bar);

  const T* Dq = so + C::oDq;
  const T* w = so + C::oW;
  const T detJ = sg[kGeoDetJ];
  const T* Ji = sg + kGeoJinv;
  const T gamma = T(prm.gamma), mu = T(prm.mu), kq = HT ? T(prm.kq) : T(0.f);

  // ---------------- volume integral (solve.cpp:276-341) + source (345-360)
  for (int o = lt; o < NB; o += GT) {
    contract<P, 0, false, false>(Dq, V1, G, o);
    contract<P, 1, false, false>(Dq, V1, G + 5 * NB, o);
    contract<P, 2, false, false>(Dq, V1, G + 10 * NB, o);
  }
  group_sync<GT>(bar);
  for (int o = lt; o < NB; o += GT)
    vpoint_flux<P, T, false, false>(so, V1, G, Ji, detJ, nullptr, gamma, mu, kq, o,
                                    [&](int i, int r, T v) { G[i * 5 * NB + r * NB + o] = v; });
  group_sync<GT>(bar);
  for (int o = lt; o < NB; o += GT) {
    const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
    const T wJq = w[qx] * w[qy] * w[qz] * detJ;
    T rv[5], y[5];
    contract_reg<P, 0, true>(Dq, G, o, rv);
    contract_reg<P, 1, true>(Dq, G + 5 * NB, o, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) rv[r] += y[r];
    contract_reg<P, 2, true>(Dq, G + 10 * NB, o, y);
#pragma unroll
    for (int r = 0; r < 5; ++r) Y[r * NB + o] = rv[r] + y[r] - T(prm.src[r]) * wJq;
  }
  group_sync<GT>(bar);

  // ---------------- faces, FPW at a time
  T* Fa = R;
  T* Fb = Fa + FPW * 5 * NQF;
  T* Gt = Fb + FPW * 12 * NQF;
#pragma unroll 1
  for (int pass = 0; pass < 6 / FPW; ++pass) {
#pragma unroll 1
    for (int i = lt; i < NH; i += GT) {
      const int j = i / NQF, lf = FPW * pass + j, fq = i % NQF;
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
    group_sync<GT>(bar);
#pragma unroll 1
    for (int i = lt; i < NH; i += GT) {  // tangential test derivatives
      const int j = i / NQF, lf = FPW * pass + j, fq = i % NQF, t1 = fq % P, t2 = fq / P, a = lf >> 1;
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
    group_sync<GT>(bar);
    for (int o = lt; o < NB; o += GT) {
      const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
      const T* Ev = so + C::oEh;
      const T* Dv = so + C::oDh;
      T rv[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) rv[r] = Y[r * NB + o];
#pragma unroll
      for (int j = 0; j < FPW; ++j) {
        const int lf = FPW * pass + j, a = lf >> 1, end = lf & 1;
        const int qa = a == 0 ? qx : a == 1 ? qy : qz;
        const int t1 = a == 0 ? qy : qx, t2 = a == 2 ? qy : qz;
        const T ev = Ev[end * P + qa], dv = Dv[end * P + qa];
        const T* gt = Gt + j * 9 * NQF + t1 + P * t2;
        rv[0] += ev * gt[0];
#pragma unroll
        for (int r = 1; r < 5; ++r) rv[r] += ev * gt[r * NQF] + dv * gt[(4 + r) * NQF];
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) Y[r * NB + o] = rv[r];
    }
    group_sync<GT>(bar);
  }

  // ---------------- norm partials: the nodal residual R = B3^T Y of each element
  if (sa.part) {
    const T* B = so + C::oB;
    T* A0 = R;
    T* A1 = R + 5 * NB;
    for (int o = lt; o < NB; o += GT) contract<P, 0, true, false>(B, Y, A0, o);
    group_sync<GT>(bar);
    for (int o = lt; o < NB; o += GT) contract<P, 1, true, false>(B, A0, A1, o);
    group_sync<GT>(bar);
    double s[2] = {0., 0.};
    for (int o = lt; o < NB; o += GT) {
      T rn[5];
      contract_reg<P, 2, true>(B, A1, o, rn);
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int l = 0; l < 2; ++l) s[l] += double(rn[r].lane(l)) * double(rn[r].lane(l));
    }
#pragma unroll
    for (int l = 0; l < 2; ++l) s[l] = group_sum<GT>(s[l], lt, reinterpret_cast<double*>(eb + L::eRed) + 2 * l, bar);
    if (lt == 0) {
      sa.part[el[0]] = s[0];
      sa.part[el[1]] = s[1];
    }
    group_sync<GT>(bar);
  }

  // ---------------- f_V = -Y / (w detJ) in FP64, RK update, per element
  T* sVn = R;
  const double* wd = opsd + C::oW;
  const double dj0 = geo[el[0] * kGeoStride + kGeoDetJ], dj1 = geo[el[1] * kGeoStride + kGeoDetJ];
  for (int o = lt; o < NB; o += GT) {
    const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
    const double wq = wd[qx] * wd[qy] * wd[qz];
    const double sc0 = -1.0 / (wq * dj0);
    const double sc1 = -1.0 / (wq * dj1);
    const long b0 = el[0] * 5 * NB + o, b1 = el[1] * 5 * NB + o;
    if (sa.mode == MODE_RESIDUAL) {
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const T yv = Y[r * NB + o];
        sa.fout[b0 + r * NB] = double(yv.lane(0)) * sc0;
        sa.fout[b1 + r * NB] = double(yv.lane(1)) * sc1;
      }
    } else {
      RkOperands q0[5], q1[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        q0[r] = rk_stage_load(sa, b0 + r * NB, Ve0 + r * NB + o);
        q1[r] = rk_stage_load(sa, b1 + r * NB, Ve1 + r * NB + o);
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        const T yv = Y[r * NB + o];
        const double un0 = rk_stage_apply(sa, b0 + r * NB, double(yv.lane(0)) * sc0, q0[r]);
        const double un1 = rk_stage_apply(sa, b1 + r * NB, double(yv.lane(1)) * sc1, q1[r]);
        sa.Uout[b0 + r * NB] = un0;
        sa.Uout[b1 + r * NB] = un1;
        sVn[r * L::LS * P * P + o + (L::LS - P) * (o / P)] = T((float)un0, (float)un1);
      }
    }
  }
  if (sa.Tnext) {
    group_sync<GT>(bar);
    T* Te = reinterpret_cast<T*>(sa.Tnext) + k * 60 * NQF;
    T* sN = R + 5 * L::LS * P * P;
#pragma unroll 1
    for (int pass = 0; pass < 6 / FPW; ++pass) {
      if (pass) group_sync<GT>(bar);
      vtrace_half<P, T, false, FPW, GT, L::LS>(pass, sVn, sN, so, sg, mu, kq, Te, nullptr, bar);
    }
  }
}

}  // namespace dgb
