// Pointwise physics shared by the kernels, written for a generic real type T
// (double in the FP64 path, float in the mixed path, f2 for two elements of
// the mixed path in lockstep, pair.cuh).  Formulas follow the
// reference's flux.cpp and bound_states.cpp; the cited lines name the
// equations restated here.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "pair.cuh"

// host + device: the kernels use these, and the host-side check hooks run the
// same code on the CPU
#define DGB_HD __host__ __device__ __forceinline__

namespace dgb {

struct DevParams {
  double gamma, R, mu, P, Pt, Tt, eta;
  double kq;  // heat-flux coefficient mu gamma / Pr (0: no heat conduction, the reference's physics)
  double Tw;  // temperature of isothermal walls (btype -8, an extension)
  double Ufr[5];
  double src[5];
};

// F(U) . n for the Euler flux (flux.cpp:24-48).
template <class T>
DGB_HD void euler_flux_n(const T* U, T gamma, const T* n, T* Fn)
{
  const T r = U[0], ir = T(1) / r, u = U[1] * ir, v = U[2] * ir, w = U[3] * ir;
  const T p = (gamma - T(1)) * (U[4] - T(0.5) * r * (u * u + v * v + w * w));
  const T un = u * n[0] + v * n[1] + w * n[2];
  const T H = (U[4] + p) * ir;
  Fn[0] = r * un;
  Fn[1] = r * u * un + p * n[0];
  Fn[2] = r * v * un + p * n[1];
  Fn[3] = r * w * un + p * n[2];
  Fn[4] = r * H * un;
}

// Full Euler flux, F[c][r] for direction c (flux.cpp:24-48).
template <class T>
DGB_HD void euler_flux(const T* U, T gamma, T F[3][5])
{
  const T r = U[0], ir = T(1) / r, u = U[1] * ir, v = U[2] * ir, w = U[3] * ir;
  const T p = (gamma - T(1)) * (U[4] - T(0.5) * r * (u * u + v * v + w * w));
  const T H = (U[4] + p) * ir;
  const T vel[3] = {u, v, w};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T m = r * vel[c];
    F[c][0] = m;
    F[c][1] = m * u;
    F[c][2] = m * v;
    F[c][3] = m * w;
    F[c][4] = m * H;
    F[c][1 + c] += p;
  }
}

// Heat conduction, an extension the reference does not have (its A has no
// heat flux, flux.cpp:185-201): the energy flux gains kappa dT/dx with
// kappa = mu c_p / Pr, T = p / (rho R), which is kq Y with kq = mu gamma / Pr
// and Y = d(E/rho) - u . du = (1/rho) [dE - e drho - u . dm + |u|^2 drho]
// for a derivative g = dS of the conserved state (e = E/rho).
template <class T>
DGB_HD T heat_y(const T* S, const T* g)
{
  const T ir = T(1) / S[0];
  const T e = S[4] * ir, u = S[1] * ir, v = S[2] * ir, w = S[3] * ir;
  return ir * (g[4] - e * g[0] - (u * g[1] + v * g[2] + w * g[3]) + (u * u + v * v + w * w) * g[0]);
}

// Viscous (Stokes) flux Q[c][r] = A(S, grad S) (flux.cpp:156-202), plus the
// optional heat flux kq Y_c in the energy row.  G[c][r] = d S_r / d x_c.
template <class T>
DGB_HD void visc_flux(const T* S, const T G[3][5], T mu, T Q[3][5], T kq = T(0))
{
  const T lam = -(T(2) / T(3)) * mu;
  const T ir = T(1) / S[0];
  const T u = S[1] * ir, v = S[2] * ir, w = S[3] * ir;
  T du[3][3];  // du[i][c] = d vel_i / d x_c
  const T vel[3] = {u, v, w};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) du[i][c] = (G[c][1 + i] - G[c][0] * vel[i]) * ir;
  const T dv = du[0][0] + du[1][1] + du[2][2];
  T tau[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) tau[i][c] = mu * (du[i][c] + du[c][i]);
#pragma unroll
  for (int i = 0; i < 3; ++i) tau[i][i] = lam * dv + T(2) * mu * du[i][i];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Q[c][0] = T(0);
    Q[c][1] = tau[0][c];
    Q[c][2] = tau[1][c];
    Q[c][3] = tau[2][c];
    Q[c][4] = u * tau[0][c] + v * tau[1][c] + w * tau[2][c];
  }
  if (kq != T(0)) {
#pragma unroll
    for (int c = 0; c < 3; ++c) Q[c][4] += kq * heat_y(S, G[c]);
  }
}

// A(S, d (x) n): the viscous flux of a rank-one "gradient" d n^T, the argument
// of the BR2 lifting and dual-consistency terms (solve.cpp:432-444, 516-528,
// 657-667).  With a_i = (d_{1+i} - d_0 vel_i) / rho the velocity gradient is
// a n^T, so tau = mu (a n^T + n a^T) + lam (a.n) I.
template <class T>
DGB_HD void visc_rank1(const T* S, const T* d, const T* n, T mu, T Q[3][5], T kq = T(0))
{
  const T lam = -(T(2) / T(3)) * mu;
  const T ir = T(1) / S[0];
  const T vel[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  T a[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) a[i] = (d[1 + i] - d[0] * vel[i]) * ir;
  const T an = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    T e = T(0);
    Q[c][0] = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T t = mu * (a[i] * n[c] + a[c] * n[i]);
      if (i == c) t += lam * an;
      Q[c][1 + i] = t;
      e += vel[i] * t;
    }
    Q[c][4] = e;
  }
  if (kq != T(0)) {  // the heat flux of the gradient d n^T: kq Y(d) n
    const T h = kq * heat_y(S, d);
#pragma unroll
    for (int c = 0; c < 3; ++c) Q[c][4] += h * n[c];
  }
}

// A(S, d (x) n) . n, the normal component only.
template <class T>
DGB_HD void visc_jump_n(const T* S, const T* d, const T* n, T mu, T* Qn, T kq = T(0))
{
  const T lam = -(T(2) / T(3)) * mu;
  const T ir = T(1) / S[0];
  const T vel[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  T a[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) a[i] = (d[1 + i] - d[0] * vel[i]) * ir;
  const T an = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
  const T nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
  Qn[0] = T(0);
  T e = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T t = mu * (a[i] * nn + an * n[i]) + lam * an * n[i];
    Qn[1 + i] = t;
    e += vel[i] * t;
  }
  Qn[4] = e;
  if (kq != T(0)) Qn[4] += kq * heat_y(S, d) * nn;
}

// Roe flux with the entropy fix at 5% of the Roe sound speed (flux.cpp:56-154).
// roe_dissipation: |A_roe| (Ur - Ul) at the Roe average (u, v, w, H)
// (roe_dissipation_jump takes the jump Ur - Ul itself).
template <class T>
DGB_HD void roe_dissipation_jump(const T* jump, const T* n, T gm1, T u, T v, T w, T H, T* d)
{
  const T dr = jump[0], dmx = jump[1], dmy = jump[2], dmz = jump[3];
  const T dE = jump[4];
  const T q2 = u * u + v * v + w * w;
  const T c = sqrt(gm1 * (H - T(0.5) * q2));
  const T ic = T(1) / c;
  const T un = u * n[0] + v * n[1] + w * n[2];
  const T l1 = un + c, l2 = un - c, l3 = un, eps = T(0.05) * c;
  T a1 = fabs(l1), a2 = fabs(l2), a3 = fabs(l3);
  if constexpr (is_pair<T>::value) {  // two elements in lockstep: the fix lane by lane
    if (any_lt(a1, eps) || any_lt(a2, eps) || any_lt(a3, eps)) {
      const T i2e = T(1) / (T(2) * eps);
      a1 = select_lt(a1, eps, fabs((eps * eps + l1 * l1) * i2e), a1);
      a2 = select_lt(a2, eps, fabs((eps * eps + l2 * l2) * i2e), a2);
      a3 = select_lt(a3, eps, fabs((eps * eps + l3 * l3) * i2e), a3);
    }
  } else if (a1 < eps || a2 < eps || a3 < eps) {  // entropy fix, rarely taken
    const T i2e = T(1) / (T(2) * eps);
    if (a1 < eps) a1 = fabs((eps * eps + l1 * l1) * i2e);
    if (a2 < eps) a2 = fabs((eps * eps + l2 * l2) * i2e);
    if (a3 < eps) a3 = fabs((eps * eps + l3 * l3) * i2e);
  }
  const T s1 = T(0.5) * (a1 + a2), s2 = T(0.5) * (a1 - a2);
  const T G1 = gm1 * (T(0.5) * q2 * dr - (u * dmx + v * dmy + w * dmz) + dE);
  const T G2 = -un * dr + (dmx * n[0] + dmy * n[1] + dmz * n[2]);
  const T C1 = (G1 * ic * ic) * (s1 - a3) + (G2 * ic) * s2;
  const T C2 = (G1 * ic) * s2 + (s1 - a3) * G2;
  d[0] = a3 * dr + C1;
  d[1] = a3 * dmx + C1 * u + C2 * n[0];
  d[2] = a3 * dmy + C1 * v + C2 * n[1];
  d[3] = a3 * dmz + C1 * w + C2 * n[2];
  d[4] = a3 * dE + C1 * H + C2 * un;
}

template <class T>
DGB_HD void roe_dissipation(const T* Ul, const T* Ur, const T* n, T gm1, T u, T v, T w, T H, T* d)
{
  T jump[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) jump[k] = Ur[k] - Ul[k];
  roe_dissipation_jump<T>(jump, n, gm1, u, v, w, H, d);
}

// f = 1/2 (F(Ul) + F(Ur)).n - 1/2 |A_roe| (Ur - Ul), the two sides taken in
// turn: each side's central flux goes into f, and only what the Roe average
// needs (sqrt(rho) and sqrt(rho) (u, v, w, H)) stays live, so the sides'
// primitive variables are dead before the dissipation.  That keeps the FP64
// face kernels' registers down (measured 3.5% faster stage); the packed pair
// type keeps the plain form below, which measured faster there.
template <class T>
DGB_HD void roe_flux(const T* Ul, const T* Ur, const T* n, T g, T* f)
{
  const T gm1 = g - T(1);
  if constexpr (!is_pair<T>::value) {
    T sq[2], sa[2][4];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const T* U = s ? Ur : Ul;
      const T r = U[0], ir = T(1) / r, uu = U[1] * ir, vv = U[2] * ir, ww = U[3] * ir;
      const T p = gm1 * (U[4] - T(0.5) * r * (uu * uu + vv * vv + ww * ww));
      const T Hs = (U[4] + p) * ir;
      const T m = r * (uu * n[0] + vv * n[1] + ww * n[2]);
      const T c[5] = {m, m * uu + p * n[0], m * vv + p * n[1], m * ww + p * n[2], m * Hs};
#pragma unroll
      for (int k = 0; k < 5; ++k) f[k] = s ? f[k] + c[k] : c[k];
      sq[s] = sqrt(r);
      sa[s][0] = sq[s] * uu;
      sa[s][1] = sq[s] * vv;
      sa[s][2] = sq[s] * ww;
      sa[s][3] = sq[s] * Hs;
    }
    const T iden = T(1) / (sq[0] + sq[1]);
    T d[5];
    roe_dissipation<T>(Ul, Ur, n, gm1, (sa[0][0] + sa[1][0]) * iden, (sa[0][1] + sa[1][1]) * iden,
                    (sa[0][2] + sa[1][2]) * iden, (sa[0][3] + sa[1][3]) * iden, d);
#pragma unroll
    for (int k = 0; k < 5; ++k) f[k] = T(0.5) * f[k] - T(0.5) * d[k];
  } else {
    const T rl = Ul[0], irl = T(1) / rl, ul = Ul[1] * irl, vl = Ul[2] * irl, wl = Ul[3] * irl;
    const T pl = gm1 * (Ul[4] - T(0.5) * rl * (ul * ul + vl * vl + wl * wl));
    const T Hl = (Ul[4] + pl) * irl;
    const T rr = Ur[0], irr = T(1) / rr, ur = Ur[1] * irr, vr = Ur[2] * irr, wr = Ur[3] * irr;
    const T pr = gm1 * (Ur[4] - T(0.5) * rr * (ur * ur + vr * vr + wr * wr));
    const T Hr = (Ur[4] + pr) * irr;
    const T sl = sqrt(rl), sr = sqrt(rr), iden = T(1) / (sl + sr);
    T d[5];
    roe_dissipation<T>(Ul, Ur, n, gm1, (sl * ul + sr * ur) * iden, (sl * vl + sr * vr) * iden,
                    (sl * wl + sr * wr) * iden, (sl * Hl + sr * Hr) * iden, d);
    const T unl = ul * n[0] + vl * n[1] + wl * n[2];
    const T unr = ur * n[0] + vr * n[1] + wr * n[2];
    f[0] = T(0.5) * (rl * unl + rr * unr) - T(0.5) * d[0];
    f[1] = T(0.5) * (rl * ul * unl + pl * n[0] + rr * ur * unr + pr * n[0]) - T(0.5) * d[1];
    f[2] = T(0.5) * (rl * vl * unl + pl * n[1] + rr * vr * unr + pr * n[1]) - T(0.5) * d[2];
    f[3] = T(0.5) * (rl * wl * unl + pl * n[2] + rr * wr * unr + pr * n[2]) - T(0.5) * d[3];
    f[4] = T(0.5) * (rl * Hl * unl + rr * Hr * unr) - T(0.5) * d[4];
  }
}

// roe_flux(UL, UR, sgn n) with (UL, UR) = (Uo, Un) on a high face (end 1)
// and (Un, Uo) on a low one, without copies of the two states: each side is
// picked as it is used and the jumps are sgn (Un - Uo), which equals UR - UL
// exactly.  Same bits as the copying call; fewer live registers.
template <class T>
DGB_HD void roe_flux_oriented(const T* Uo, const T* Un, int end, const T* n, T g, T* f)
{
  const T gm1 = g - T(1);
  const T sgn = end ? T(1) : T(-1);
  const T nn[3] = {sgn * n[0], sgn * n[1], sgn * n[2]};
  T sq[2], sa[2][4];
#pragma unroll
  for (int s = 0; s < 2; ++s) {  // s = 0 the left state, 1 the right
    const bool own = (s == 1) != (end != 0);
    T U[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) U[k] = own ? Uo[k] : Un[k];
    const T r = U[0], ir = T(1) / r, uu = U[1] * ir, vv = U[2] * ir, ww = U[3] * ir;
    const T p = gm1 * (U[4] - T(0.5) * r * (uu * uu + vv * vv + ww * ww));
    const T Hs = (U[4] + p) * ir;
    const T m = r * (uu * nn[0] + vv * nn[1] + ww * nn[2]);
    const T c[5] = {m, m * uu + p * nn[0], m * vv + p * nn[1], m * ww + p * nn[2], m * Hs};
#pragma unroll
    for (int k = 0; k < 5; ++k) f[k] = s ? f[k] + c[k] : c[k];
    sq[s] = sqrt(r);
    sa[s][0] = sq[s] * uu;
    sa[s][1] = sq[s] * vv;
    sa[s][2] = sq[s] * ww;
    sa[s][3] = sq[s] * Hs;
  }
  const T iden = T(1) / (sq[0] + sq[1]);
  T jump[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) jump[k] = sgn * (Un[k] - Uo[k]);
  T d[5];
  roe_dissipation_jump<T>(jump, nn, gm1, (sa[0][0] + sa[1][0]) * iden, (sa[0][1] + sa[1][1]) * iden,
                       (sa[0][2] + sa[1][2]) * iden, (sa[0][3] + sa[1][3]) * iden, d);
#pragma unroll
  for (int k = 0; k < 5; ++k) f[k] = T(0.5) * f[k] - T(0.5) * d[k];
}

// Ghost state for a boundary face (bound_states.cpp:24-130, selected as in
// solve.cpp:235-252), plus the isothermal wall -8 the reference lacks.
// Returns 1 when subsonic inflow has no non-negative boundary Mach root (the
// reference aborts there on the host, :80-83).
template <class T>
DGB_HD int boundary_state(int bt, const T* UL, const T* n, const DevParams& prm, T* Ub)
{
  const T gamma = T(prm.gamma), gm1 = gamma - T(1);
  const T u = UL[1] / UL[0], v = UL[2] / UL[0], w = UL[3] / UL[0];
  if (bt == -3) {  // freestream
#pragma unroll
    for (int r = 0; r < 5; ++r) Ub[r] = T(prm.Ufr[r]);
    return 0;
  }
  if (bt == -4) {  // inviscid wall: remove the normal velocity
    const T vn = u * n[0] + v * n[1] + w * n[2];
    Ub[0] = UL[0];
    Ub[1] = UL[0] * (u - vn * n[0]);
    Ub[2] = UL[0] * (v - vn * n[1]);
    Ub[3] = UL[0] * (w - vn * n[2]);
    Ub[4] = UL[4];
    return 0;
  }
  if (bt == -8) {  // isothermal no-slip wall (an extension): zero velocity, interior density, wall temperature
    Ub[0] = UL[0];
    Ub[1] = T(0);
    Ub[2] = T(0);
    Ub[3] = T(0);
    Ub[4] = UL[0] * T(prm.R) * T(prm.Tw) / gm1;
    return 0;
  }
  if (bt == -7) {  // no-slip wall: zero velocity, interior total energy
    Ub[0] = UL[0];
    Ub[1] = T(0);
    Ub[2] = T(0);
    Ub[3] = T(0);
    Ub[4] = UL[4];
    return 0;
  }
  const T q2 = u * u + v * v + w * w;
  const T pp = gm1 * (UL[4] - T(0.5) * UL[0] * q2);
  const T unp = u * n[0] + v * n[1] + w * n[2];
  const T cp = sqrt(gamma * pp / UL[0]);
  const T Jp = unp + T(2) * cp / gm1;
  if (bt == -5) {  // subsonic inflow: total T and p, outgoing Riemann invariant
    const T RTt = gamma * T(prm.R) * T(prm.Tt);
    const T a = RTt - T(0.5) * gm1 * Jp * Jp;
    const T b = -T(4) * RTt / gm1;
    const T c = T(4) * RTt / (gm1 * gm1) - Jp * Jp;
    const T disc = sqrt(b * b - T(4) * a * c);
    const T s0 = (-b + disc) / (T(2) * a), s1 = (-b - disc) / (T(2) * a);
    T Mb = T(0);
    int bad = 0;
    if (s0 >= T(0) && s1 >= T(0)) Mb = s0 < s1 ? s0 : s1;
    else if (s0 >= T(0)) Mb = s0;
    else if (s1 >= T(0)) Mb = s1;
    else bad = 1;
    const T Tb = T(prm.Tt) / (T(1) + T(0.5) * gm1 * Mb * Mb);
    const T Pb = T(prm.Pt) * pow(Tb / T(prm.Tt), gamma / gm1);
    const T rb = Pb / (T(prm.R) * Tb);
    const T cb = sqrt(gamma * Pb / rb);
    const T ub = -Mb * cb * n[0], vb = -Mb * cb * n[1], wb = -Mb * cb * n[2];
    Ub[0] = rb;
    Ub[1] = rb * ub;
    Ub[2] = rb * vb;
    Ub[3] = rb * wb;
    Ub[4] = Pb / gm1 + T(0.5) * rb * (ub * ub + vb * vb + wb * wb);
    return bad;
  }
  // subsonic outflow: fixed static pressure, interior entropy and invariant
  const T Pf = T(prm.P);
  const T Sp = pp / pow(UL[0], gamma);
  const T rb = pow(Pf / Sp, T(1) / gamma);
  const T cb = sqrt(gamma * Pf / rb);
  const T unb = Jp - T(2) * cb / gm1;
  const T ub = u - unp * n[0] + unb * n[0], vb = v - unp * n[1] + unb * n[1];
  const T wb = w - unp * n[2] + unb * n[2];
  Ub[0] = rb;
  Ub[1] = rb * ub;
  Ub[2] = rb * vb;
  Ub[3] = rb * wb;
  Ub[4] = Pf / gm1 + T(0.5) * rb * (ub * ub + vb * vb + wb * wb);
  return 0;
}

}  // namespace dgb
