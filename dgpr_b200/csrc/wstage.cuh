// The Gauss-point stage with one warp per element (p = 3: 64 Gauss points,
// two per lane; 16 face points per face, two faces per pass, one per lane).
// A CTA holds two independent elements, one per warp, sharing the operator
// table: the only block barrier is the one after the table is loaded, the
// phases of an element are ordered by __syncwarp alone, and faces go two at
// a time, so each pass is one full round of the warp.  The arithmetic is the
// element-per-CTA kernel's own (vpoint_flux, load_face_point,
// face_point_fluxes, vtrace_half, rk_stage_value in the same order), so the
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
  static constexpr int FPW = 2;  // faces per pass
  static constexpr int OPSB = align16(C::OPS * ST);
  // per element: [geometry | Y (V first) : 5 NB | R]
  static constexpr int eGeo = 0;
  static constexpr int eY = align16(kGeoStride * ST);
  static constexpr int eR = eY + align16(5 * NB * ST);
  // R: gradients, then contravariant fluxes G[3][5][NB]; the face buffers
  // Fa[FPW][5][NQF] Fb[FPW][12][NQF] Gt[FPW][9][NQF]; the norm's two nodal
  // buffers [2][5][NB]; the new state [5][NB] and the trace scratch
  // [FPW][10][NQF]
  static constexpr int RG = 15 * NB * ST;
  static constexpr int RF = FPW * 26 * NQF * ST;
  static constexpr int RN = 10 * NB * ST;
  static constexpr int RT = 5 * NB * ST + FPW * 10 * NQF * ST;
  static constexpr int RMAX = RG > RF ? (RG > RN ? (RG > RT ? RG : RT) : (RN > RT ? RN : RT))
                                      : (RF > RN ? (RF > RT ? RF : RT) : (RN > RT ? RN : RT));
  static constexpr int ELEM = eR + align16(RMAX);
  static constexpr int TOTAL = OPSB + kWarpElems * ELEM;
};

template <int P, class T, bool CV, bool HT>
__global__ void __launch_bounds__(32 * kWarpElems, (MinBlocks<P, T>::value))
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
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long u = (long)kWarpElems * blockIdx.x + warp;
  if (u >= (sa.ecount ? sa.ecount : E)) return;
  const long e = sa.ebase + sa.estep * u;
  unsigned char* eb = smraw + L::OPSB + warp * L::ELEM;
  T* sg = reinterpret_cast<T*>(eb + L::eGeo);
  T* Y = reinterpret_cast<T*>(eb + L::eY);  // the state V first, the Gauss-point residual Y later
  T* V1 = Y;
  T* R = reinterpret_cast<T*>(eb + L::eR);
  T* G = R;

  if (DGB_PREFETCH_L2 && (sizeof(T) == 8 || DGB_PREFETCH_L2_F32)) {  // data read much later
    prefetch_range(Tr + e * 60 * NQF, 60L * NQF * sizeof(T), lane, 32);
    if (lane < 6) {
      const int nb = nbr[e * 6 + lane];
      if (nb >= 0) prefetch_range(Tr + ((long)nb * 6 + (lane ^ 1)) * 10 * NQF, 10L * NQF * sizeof(T), 0, 1);
    }
    if (sa.Ubase) prefetch_range(sa.Ubase + e * 5 * NB, 40L * NB, lane, 32);
    if (sa.acc && sa.mode >= MODE_RK4_1 && sa.mode <= MODE_RK4_3) prefetch_range(sa.acc + e * 5 * NB, 40L * NB, lane, 32);
  }
  for (int i = lane; i < kGeoStride; i += 32) sg[i] = T(geo[e * kGeoStride + i]);
  const double* Ve = Vs + e * 5 * NB;
  for (int i = lane; i < 5 * NB; i += 32) V1[i] = T(Ve[i]);
  __syncwarp();

  const T* Dq = so + C::oDq;
  const T* w = so + C::oW;
  const double detJd = geo[e * kGeoStride + kGeoDetJ];
  const T detJ = sg[kGeoDetJ];
  const T* Ji = sg + kGeoJinv;
  const T gamma = T(prm.gamma), mu = T(prm.mu), kq = HT ? T(prm.kq) : T(0);
  const double* gve = CV ? gv + e * kVolC * NB : nullptr;
  const double* gfe = CV ? gf + e * 6 * kFaceC * NQF : nullptr;

  // ---------------- volume integral (solve.cpp:276-341) + source (345-360)
  for (int o = lane; o < NB; o += 32) {  // reference gradients
    contract<P, 0, false, false>(Dq, V1, G, o);
    contract<P, 1, false, false>(Dq, V1, G + 5 * NB, o);
    contract<P, 2, false, false>(Dq, V1, G + 10 * NB, o);
  }
  __syncwarp();
  for (int o = lane; o < NB; o += 32)  // pointwise flux at o, in place of its gradients
    vpoint_flux<P, T, CV, false>(so, V1, G, Ji, detJ, gve, gamma, mu, kq, o,
                                 [&](int i, int r, T v) { G[i * 5 * NB + r * NB + o] = v; });
  __syncwarp();
  for (int o = lane; o < NB; o += 32) {  // Y = sum_i Dq_i^T Ghat_i minus the source tested with w detJ (over V)
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
  __syncwarp();

  // ---------------- faces (solve.cpp:393-794), FPW at a time
  T* Fa = R;                    // [FPW][5][NQF]
  T* Fb = Fa + FPW * 5 * NQF;   // [FPW][12][NQF]
  T* Gt = Fb + FPW * 12 * NQF;  // [FPW][9][NQF]
#pragma unroll 1
  for (int pass = 0; pass < 6 / FPW; ++pass) {
#pragma unroll 1
    for (int i = lane; i < NH; i += 32) {
      const int j = i / NQF, lf = FPW * pass + j, fq = i % NQF;
      T Uo[5], Qo[5], Un[5], Qn[5], lift_n;
      const int nb = load_face_point<P, T, CV>(e, lf, fq, Tr, nbr, so, geo, gf, Uo, Qo, Un, Qn, lift_n);
      face_point_fluxes<P, T, CV>(lf, fq, nb, Uo, Qo, Un, Qn, lift_n, so, sg, gfe, prm, gamma, mu, kq, detJ, Ji,
                                  sa.flag, Fa + j * 5 * NQF + fq, Fb + j * 12 * NQF + fq);
    }
    __syncwarp();
#pragma unroll 1
    for (int i = lane; i < NH; i += 32) {  // tangential test derivatives: g = fa + Dq^T fb_ax1 + Dq^T fb_ax2, h = fb_a
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
    __syncwarp();
    for (int o = lane; o < NB; o += 32) {  // each Gauss point gathers from the face points on its normal lines
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
    __syncwarp();
  }

  // ---------------- norm partial: the nodal residual R = B3^T Y
  if (sa.part) {
    const T* B = so + C::oB;
    T* A0 = R;
    T* A1 = R + 5 * NB;
    for (int o = lane; o < NB; o += 32) contract<P, 0, true, false>(B, Y, A0, o);
    __syncwarp();
    for (int o = lane; o < NB; o += 32) contract<P, 1, true, false>(B, A0, A1, o);
    __syncwarp();
    double s = 0.;
    for (int o = lane; o < NB; o += 32) {
      T rn[5];
      contract_reg<P, 2, true>(B, A1, o, rn);
#pragma unroll
      for (int r = 0; r < 5; ++r) s += double(rn[r]) * double(rn[r]);
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
    if (lane == 0) sa.part[e] = s;
    __syncwarp();
  }

  // ---------------- f_V = -Y / (w detJ) in FP64, RK update
  T* sVn = R;  // the new state for the epilogue traces
  for (int o = lane; o < NB; o += 32) {
    const int qx = o % P, qy = (o / P) % P, qz = o / (P * P);
    const double* wd = opsd + C::oW;
    const double jd = CV ? gve[kVolDetJ * NB + o] : detJd;
    const double sc = -1.0 / (wd[qx] * wd[qy] * wd[qz] * jd);
    const long base = e * 5 * NB;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      const long i = base + r * NB + o;
      const double fr = double(Y[r * NB + o]) * sc;
      if (sa.mode == MODE_RESIDUAL) {
        sa.fout[i] = fr;
      } else {
        const double un = rk_stage_value(sa, i, fr, Ve[r * NB + o]);
        sa.Uout[i] = un;
        sVn[r * NB + o] = T(un);
      }
    }
  }
  // ---------------- face traces of the new state for the next stage
  if (sa.Tnext) {
    __syncwarp();
    T* Te = reinterpret_cast<T*>(sa.Tnext) + e * 60 * NQF;
    T* sN = R + 5 * NB;
#pragma unroll 1
    for (int pass = 0; pass < 6 / FPW; ++pass) {
      if (pass) __syncwarp();
      vtrace_half<P, T, CV, FPW, true>(pass, sVn, sN, so, sg, mu, kq, Te, gfe);
    }
  }
}

}  // namespace dgb
