// Hand-written reverse mode (vector-Jacobian products) of the pointwise
// physics in physics.cuh.  Each *_vjp function takes the forward inputs and
// the adjoint of the forward outputs and ADDS the adjoint of the inputs to
// the *bar arguments.  The forward is recomputed inside, statement by
// statement, and the statements are then reversed; branch decisions (the
// Roe entropy fix) follow the forward evaluation at the same point.
#pragma once

#include "physics.cuh"

namespace dgb {

// Euler flux F[c][r] (euler_flux): Fbar[3][5] -> Ubar[5]
template <class T>
DGB_HD void euler_flux_vjp(const T* U, T gamma, const T Fbar[3][5], T* Ubar)
{
  const T gm1 = gamma - T(1);
  const T r = U[0], ir = T(1) / r;
  const T v[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
  const T q2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const T p = gm1 * (U[4] - T(0.5) * r * q2);
  const T H = (U[4] + p) * ir;
  T mbar[3] = {T(0), T(0), T(0)}, vbar[3] = {T(0), T(0), T(0)};
  T pbar = T(0), Hbar = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T m = r * v[c];
    mbar[c] += Fbar[c][0] + Fbar[c][4] * H;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      mbar[c] += Fbar[c][1 + i] * v[i];
      vbar[i] += Fbar[c][1 + i] * m;
    }
    pbar += Fbar[c][1 + c];
    Hbar += Fbar[c][4] * m;
  }
  T rbar = T(0), irbar = T(0), U4bar = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {  // m_c = r v_c
    rbar += mbar[c] * v[c];
    vbar[c] += mbar[c] * r;
  }
  // H = (U4 + p) ir
  U4bar += Hbar * ir;
  pbar += Hbar * ir;
  irbar += Hbar * (U[4] + p);
  // p = gm1 (U4 - r q2 / 2)
  U4bar += gm1 * pbar;
  rbar += -T(0.5) * gm1 * q2 * pbar;
  const T q2bar = -T(0.5) * gm1 * r * pbar;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    vbar[i] += T(2) * v[i] * q2bar;
    Ubar[1 + i] += vbar[i] * ir;  // v_i = U_{1+i} ir
    irbar += vbar[i] * U[1 + i];
  }
  rbar += -irbar * ir * ir;
  Ubar[0] += rbar;
  Ubar[4] += U4bar;
}

// Euler flux along n (euler_flux_n): Fnbar[5] -> Ubar[5]
template <class T>
DGB_HD void euler_flux_n_vjp(const T* U, T gamma, const T* n, const T* Fnbar, T* Ubar)
{
  T Fbar[3][5];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 5; ++r) Fbar[c][r] = Fnbar[r] * n[c];
  euler_flux_vjp(U, gamma, Fbar, Ubar);
}

// Heat-flux scalar Y(S, g) (heat_y): ybar -> Sbar[5], gbar[5].  With
// ir = 1/S_0, v = S_{1..3} ir, e = S_4 ir and
// B = g_4 + g_0 (|v|^2 - e) - v . g_{1..3}, Y = ir B.
template <class T>
DGB_HD void heat_y_vjp(const T* S, const T* g, T yb, T* Sbar, T* gbar)
{
  const T ir = T(1) / S[0];
  const T e = S[4] * ir, v[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  const T q2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const T B = g[4] + g[0] * (q2 - e) - (v[0] * g[1] + v[1] * g[2] + v[2] * g[3]);
  const T yi = yb * ir;
  gbar[4] += yi;
  gbar[0] += yi * (q2 - e);
  T irbar = yb * B;
  const T ebar = -yi * g[0];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    gbar[1 + i] += -yi * v[i];
    const T vb = yi * (T(2) * g[0] * v[i] - g[1 + i]);
    Sbar[1 + i] += vb * ir;
    irbar += vb * S[1 + i];
  }
  Sbar[4] += ebar * ir;
  irbar += ebar * S[4];
  Sbar[0] += -irbar * ir * ir;
}

// Viscous flux Q = A(S, G) (visc_flux): Qbar[3][5] -> Sbar[5], Gbar[3][5]
template <class T>
DGB_HD void visc_flux_vjp(const T* S, const T G[3][5], T mu, const T Qbar[3][5], T* Sbar, T Gbar[3][5],
                          T kq = T(0))
{
  if (kq != T(0)) {
#pragma unroll
    for (int c = 0; c < 3; ++c) heat_y_vjp(S, G[c], kq * Qbar[c][4], Sbar, Gbar[c]);
  }
  const T lam = -(T(2) / T(3)) * mu;
  const T ir = T(1) / S[0];
  const T v[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  T du[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) du[i][c] = (G[c][1 + i] - G[c][0] * v[i]) * ir;
  const T dv = du[0][0] + du[1][1] + du[2][2];
  T tau[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) tau[i][c] = mu * (du[i][c] + du[c][i]) + (i == c ? lam * dv : T(0));
  // Q[c][1+i] = tau[i][c]; Q[c][4] = sum_i v_i tau[i][c]
  T taub[3][3], vbar[3] = {T(0), T(0), T(0)};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      taub[i][c] = Qbar[c][1 + i] + Qbar[c][4] * v[i];
      vbar[i] += Qbar[c][4] * tau[i][c];
    }
  const T trb = taub[0][0] + taub[1][1] + taub[2][2];
  T irbar = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T dub = mu * (taub[i][c] + taub[c][i]) + (i == c ? lam * trb : T(0));
      // du[i][c] = (G[c][1+i] - G[c][0] v_i) ir
      Gbar[c][1 + i] += dub * ir;
      Gbar[c][0] += -dub * v[i] * ir;
      vbar[i] += -dub * G[c][0] * ir;
      irbar += dub * (G[c][1 + i] - G[c][0] * v[i]);
    }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    Sbar[1 + i] += vbar[i] * ir;
    irbar += vbar[i] * S[1 + i];
  }
  Sbar[0] += -irbar * ir * ir;
}

// shared tail of the rank-one forms: a_k = (d_{1+k} - d_0 v_k) ir with
// v = S_{1..3} ir, ir = 1/S_0; given abar, vbar, irbar -> Sbar, dbar
template <class T>
DGB_HD void rank1_tail_vjp(const T* S, const T* d, const T* v, T ir, const T* abar, T* vbar, T irbar, T* Sbar,
                           T* dbar)
{
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dbar[1 + k] += abar[k] * ir;
    dbar[0] += -abar[k] * v[k] * ir;
    vbar[k] += -abar[k] * d[0] * ir;
    irbar += abar[k] * (d[1 + k] - d[0] * v[k]);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Sbar[1 + k] += vbar[k] * ir;
    irbar += vbar[k] * S[1 + k];
  }
  Sbar[0] += -irbar * ir * ir;
}

// Rank-one viscous flux Q = A(S, d n^T) (visc_rank1): Qbar[3][5] -> Sbar, dbar.
// The _r forms take ir = 1 / S[0] from the caller, which divides once per
// face state for all the VJPs that state enters.
template <class T>
DGB_HD void visc_rank1_vjp_r(const T* S, T ir, const T* d, const T* n, T mu, const T Qbar[3][5], T* Sbar, T* dbar,
                             T kq = T(0))
{
  if (kq != T(0)) heat_y_vjp(S, d, kq * (Qbar[0][4] * n[0] + Qbar[1][4] * n[1] + Qbar[2][4] * n[2]), Sbar, dbar);
  const T lam = -(T(2) / T(3)) * mu;
  const T v[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  T a[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) a[k] = (d[1 + k] - d[0] * v[k]) * ir;
  const T an = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
  T tau[3][3], taub[3][3], vbar[3] = {T(0), T(0), T(0)};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) tau[k][c] = mu * (a[k] * n[c] + a[c] * n[k]) + (k == c ? lam * an : T(0));
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      taub[k][c] = Qbar[c][1 + k] + Qbar[c][4] * v[k];
      vbar[k] += Qbar[c][4] * tau[k][c];
    }
  const T anbar = lam * (taub[0][0] + taub[1][1] + taub[2][2]);
  T abar[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    T s = T(0);
#pragma unroll
    for (int c = 0; c < 3; ++c) s += (taub[j][c] + taub[c][j]) * n[c];
    abar[j] = mu * s + anbar * n[j];
  }
  rank1_tail_vjp(S, d, v, ir, abar, vbar, T(0), Sbar, dbar);
}

template <class T>
DGB_HD void visc_rank1_vjp(const T* S, const T* d, const T* n, T mu, const T Qbar[3][5], T* Sbar, T* dbar,
                           T kq = T(0))
{
  visc_rank1_vjp_r(S, T(1) / S[0], d, n, mu, Qbar, Sbar, dbar, kq);
}

// Normal component A(S, d n^T).n (visc_jump_n): Qnbar[5] -> Sbar, dbar
template <class T>
DGB_HD void visc_jump_n_vjp_r(const T* S, T ir, const T* d, const T* n, T mu, const T* Qnbar, T* Sbar, T* dbar,
                              T kq = T(0))
{
  if (kq != T(0))
    heat_y_vjp(S, d, kq * Qnbar[4] * (n[0] * n[0] + n[1] * n[1] + n[2] * n[2]), Sbar, dbar);
  const T lam = -(T(2) / T(3)) * mu;
  const T v[3] = {S[1] * ir, S[2] * ir, S[3] * ir};
  T a[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) a[k] = (d[1 + k] - d[0] * v[k]) * ir;
  const T an = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
  const T nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
  // t_i = mu (a_i nn + an n_i) + lam an n_i ; Qn[1+i] = t_i ; Qn[4] = sum v_i t_i
  T tb[3], vbar[3];
  T anbar = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T t = mu * (a[i] * nn + an * n[i]) + lam * an * n[i];
    tb[i] = Qnbar[1 + i] + Qnbar[4] * v[i];
    vbar[i] = Qnbar[4] * t;
    anbar += tb[i] * (mu + lam) * n[i];
  }
  T abar[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) abar[j] = mu * nn * tb[j] + anbar * n[j];
  rank1_tail_vjp(S, d, v, ir, abar, vbar, T(0), Sbar, dbar);
}

template <class T>
DGB_HD void visc_jump_n_vjp(const T* S, const T* d, const T* n, T mu, const T* Qnbar, T* Sbar, T* dbar,
                            T kq = T(0))
{
  visc_jump_n_vjp_r(S, T(1) / S[0], d, n, mu, Qnbar, Sbar, dbar, kq);
}

// Normal Euler flux F(U).n of one side: Fnbar[5] -> Ubar (accumulated),
// written out directly (no 3x5 intermediate).  With u = m / r, un = u.n,
// q = |u|^2, p = (g - 1)(E - r q / 2), H = (E + p) / r:
//   F = (r un, m un + p n, (E + p) un).  ir = 1 / r from the caller.
template <class T>
DGB_HD void euler_normal_flux_vjp(const T* U, T ir, T g, const T* n, const T* fb, T* Ubar)
{
  const T gm1 = g - T(1);
  const T u[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
  const T un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
  const T q = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const T p = gm1 * (U[4] - T(0.5) * U[0] * q);
  const T H = (U[4] + p) * ir;
  const T fbn = fb[1] * n[0] + fb[2] * n[1] + fb[3] * n[2];
  const T fbu = fb[1] * u[0] + fb[2] * u[1] + fb[3] * u[2];
  Ubar[0] += -un * fbu + T(0.5) * gm1 * q * fbn + fb[4] * un * (T(0.5) * gm1 * q - H);
#pragma unroll
  for (int j = 0; j < 3; ++j)
    Ubar[1 + j] += (fb[0] + fbu + fb[4] * H) * n[j] + fb[1 + j] * un - gm1 * u[j] * (fbn + fb[4] * un);
  Ubar[4] += gm1 * fbn + g * un * fb[4];
}

// Roe flux with entropy fix (roe_flux, flux.cpp:56-154): fbar[5] -> Ulbar,
// Urbar (accumulated).  The central part 1/2 (F(Ul) + F(Ur)).n goes side by side through
// euler_normal_flux_vjp; the dissipation -1/2 |A_roe| (Ur - Ul) reverses
// through the Roe average, and each side's share of the average is taken
// from its own sqrt(rho), velocity and enthalpy.  Few values are live at a
// time, which keeps the adjoint face kernel's registers down.
// irl, irr: 1 / Ul[0], 1 / Ur[0] from the caller.  The reverse part divides
// by nothing: 1 / (2 c) and 1 / (2 sqrt(r)) come from 1 / c and sqrt(r) / r.
template <class T>
DGB_HD void roe_flux_vjp_r(const T* Ul, const T* Ur, T irl, T irr, const T* n, T g, const T* fbar, T* Ulbar,
                           T* Urbar)
{
  const T gm1 = g - T(1), h = T(0.5);
  {
    T hb[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) hb[k] = h * fbar[k];
    euler_normal_flux_vjp(Ul, irl, g, n, hb, Ulbar);
    euler_normal_flux_vjp(Ur, irr, g, n, hb, Urbar);
  }
  // ---- forward of the dissipation
  T sq[2], us[2][3], Hs[2];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const T* U = s ? Ur : Ul;
    const T ir = s ? irr : irl;
#pragma unroll
    for (int k = 0; k < 3; ++k) us[s][k] = U[1 + k] * ir;
    const T p = gm1 * (U[4] - T(0.5) * U[0] * (us[s][0] * us[s][0] + us[s][1] * us[s][1] + us[s][2] * us[s][2]));
    Hs[s] = (U[4] + p) * ir;
    sq[s] = sqrt(U[0]);
  }
  const T iden = T(1) / (sq[0] + sq[1]);
  T uk[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) uk[k] = (sq[0] * us[0][k] + sq[1] * us[1][k]) * iden;
  const T H = (sq[0] * Hs[0] + sq[1] * Hs[1]) * iden;
  const T dr = Ur[0] - Ul[0];
  const T dm[3] = {Ur[1] - Ul[1], Ur[2] - Ul[2], Ur[3] - Ul[3]};
  const T dE = Ur[4] - Ul[4];
  const T q2 = uk[0] * uk[0] + uk[1] * uk[1] + uk[2] * uk[2];
  const T c = sqrt(gm1 * (H - T(0.5) * q2));
  const T ic = T(1) / c;
  const T un = uk[0] * n[0] + uk[1] * n[1] + uk[2] * n[2];
  const T l[3] = {un + c, un - c, un};
  const T eps = T(0.05) * c;
  T a[3];
  bool fix[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    a[i] = fabs(l[i]);
    fix[i] = a[i] < eps;
    if (fix[i]) a[i] = fabs((eps * eps + l[i] * l[i]) / (T(2) * eps));
  }
  const T s1 = T(0.5) * (a[0] + a[1]), s2 = T(0.5) * (a[0] - a[1]);
  const T G1 = gm1 * (T(0.5) * q2 * dr - (uk[0] * dm[0] + uk[1] * dm[1] + uk[2] * dm[2]) + dE);
  const T G2 = -un * dr + (dm[0] * n[0] + dm[1] * n[1] + dm[2] * n[2]);
  const T C1 = (G1 * ic * ic) * (s1 - a[2]) + (G2 * ic) * s2;
  const T C2 = (G1 * ic) * s2 + (s1 - a[2]) * G2;

  // ---- reverse: -1/2 (a3 dr + C1), -1/2 (a3 dm_k + C1 u_k + C2 n_k), -1/2 (a3 dE + C1 H + C2 un)
  T ukb[3], Hb, unb, drb, dmb[3], dEb;
  T a3b = -h * (fbar[0] * dr + fbar[1] * dm[0] + fbar[2] * dm[1] + fbar[3] * dm[2] + fbar[4] * dE);
  drb = -h * fbar[0] * a[2];
  dEb = -h * fbar[4] * a[2];
  T C1b = -h * (fbar[0] + fbar[4] * H);
  T C2b = -h * fbar[4] * un;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dmb[k] = -h * fbar[1 + k] * a[2];
    C1b += -h * fbar[1 + k] * uk[k];
    C2b += -h * fbar[1 + k] * n[k];
    ukb[k] = -h * fbar[1 + k] * C1;
  }
  Hb = -h * fbar[4] * C1;
  unb = -h * fbar[4] * C2;
  // C1 = G1 ic^2 (s1 - a3) + G2 ic s2 ; C2 = G1 ic s2 + (s1 - a3) G2
  const T G1b = C1b * ic * ic * (s1 - a[2]) + C2b * ic * s2;
  const T G2b = C1b * ic * s2 + C2b * (s1 - a[2]);
  const T icb = C1b * (T(2) * G1 * ic * (s1 - a[2]) + G2 * s2) + C2b * G1 * s2;
  const T s1b = C1b * G1 * ic * ic + C2b * G2;
  const T s2b = C1b * G2 * ic + C2b * G1 * ic;
  a3b += -C1b * G1 * ic * ic - C2b * G2;
  // G2 = -un dr + dm . n
  unb += -G2b * dr;
  drb += -G2b * un;
#pragma unroll
  for (int k = 0; k < 3; ++k) dmb[k] += G2b * n[k];
  // G1 = gm1 (q2 dr / 2 - uk . dm + dE)
  T q2b = G1b * gm1 * h * dr;
  drb += G1b * gm1 * h * q2;
  dEb += G1b * gm1;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    ukb[k] += -G1b * gm1 * dm[k];
    dmb[k] += -G1b * gm1 * uk[k];
  }
  // s1, s2, then a_i from l_i (with the entropy fix where it was taken)
  const T ab[3] = {h * (s1b + s2b), h * (s1b - s2b), a3b};
  T lb[3], epsb = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (fix[i]) {
      lb[i] = ab[i] * l[i] / eps;
      epsb += ab[i] * (h - l[i] * l[i] / (T(2) * eps * eps));
    } else {
      lb[i] = l[i] >= T(0) ? ab[i] : -ab[i];
    }
  }
  unb += lb[0] + lb[1] + lb[2];
  T cb = lb[0] - lb[1] + T(0.05) * epsb;
  // un = uk . n ; ic = 1/c ; c = sqrt(gm1 (H - q2/2)) ; q2 = |uk|^2
  cb += -icb * ic * ic;
  const T c2b = cb * (h * ic);
  Hb += gm1 * c2b;
  q2b += -h * gm1 * c2b;
#pragma unroll
  for (int k = 0; k < 3; ++k) ukb[k] += unb * n[k] + T(2) * uk[k] * q2b;
  // the jumps
  Urbar[0] += drb;
  Ulbar[0] -= drb;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Urbar[1 + k] += dmb[k];
    Ulbar[1 + k] -= dmb[k];
  }
  Urbar[4] += dEb;
  Ulbar[4] -= dEb;
  // the Roe average, side by side: uk = (sl ul + sr ur) iden, H likewise;
  // d/d s_side = (side value - average) iden, d/d side value = s_side iden;
  // then u = m / r, H = g E / r - (g - 1) |u|^2 / 2, s = sqrt(r)
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const T* U = s ? Ur : Ul;
    T* Ub = s ? Urbar : Ulbar;
    const T ir = s ? irr : irl, w = sq[s] * iden;
    T sqb = Hb * (Hs[s] - H), ub[3], qs = T(0), uub = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sqb += ukb[k] * (us[s][k] - uk[k]);
      ub[k] = ukb[k] * w;
      qs += us[s][k] * us[s][k];
      uub += ub[k] * us[s][k];
    }
    const T Hsb = Hb * w;
    Ub[4] += Hsb * g * ir;
#pragma unroll
    for (int k = 0; k < 3; ++k) Ub[1 + k] += (ub[k] - Hsb * gm1 * us[s][k]) * ir;
    Ub[0] += sqb * iden * (h * sq[s] * ir) + (-uub + Hsb * (gm1 * qs - g * U[4] * ir)) * ir;
  }
}

template <class T>
DGB_HD void roe_flux_vjp(const T* Ul, const T* Ur, const T* n, T g, const T* fbar, T* Ulbar, T* Urbar)
{
  roe_flux_vjp_r(Ul, Ur, T(1) / Ul[0], T(1) / Ur[0], n, g, fbar, Ulbar, Urbar);
}


// Boundary ghost state (boundary_state): Ubbar -> ULbar for every boundary
// type.  Subsonic inflow depends on UL only through the outgoing Riemann
// invariant Jp (the boundary Mach number is a root of a quadratic in Jp, the
// same root as the forward picks; none -> no dependence); subsonic outflow
// through Jp, the entropy pp / rho^gamma and the tangential velocity.
// Returns 0 (1 is kept for a boundary type without an adjoint).
template <class T>
DGB_HD int boundary_state_vjp(int bt, const T* UL, const T* n, const DevParams& prm, const T* Ubbar, T* ULbar)
{
  if (bt == -3) return 0;  // freestream: constant
  if (bt == -4) {
    // Ub = (r, r (v - (v.n) n), E) with v = m / r
    const T ir = T(1) / UL[0];
    const T v[3] = {UL[1] * ir, UL[2] * ir, UL[3] * ir};
    const T vn = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
    T vbar[3], vnbar = T(0), rbar = Ubbar[0];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T vt = v[k] - vn * n[k];
      rbar += Ubbar[1 + k] * vt;
      vbar[k] = Ubbar[1 + k] * UL[0];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) vnbar += -vbar[k] * n[k];
    T irbar = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T vk = vbar[k] + vnbar * n[k];
      ULbar[1 + k] += vk * ir;
      irbar += vk * UL[1 + k];
    }
    ULbar[0] += rbar - irbar * ir * ir;
    ULbar[4] += Ubbar[4];
    return 0;
  }
  if (bt == -7) {
    ULbar[0] += Ubbar[0];
    ULbar[4] += Ubbar[4];
    return 0;
  }
  if (bt == -8) {  // Ub = (r, 0, 0, 0, r R Tw / (gamma - 1))
    ULbar[0] += Ubbar[0] + Ubbar[4] * T(prm.R) * T(prm.Tw) / (T(prm.gamma) - T(1));
    return 0;
  }
  if (bt != -5 && bt != -6) return 1;

  // forward quantities shared by inflow and outflow
  const T gamma = T(prm.gamma), gm1 = gamma - T(1);
  const T r0 = UL[0], ir = T(1) / r0;
  const T v[3] = {UL[1] * ir, UL[2] * ir, UL[3] * ir};
  const T q2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const T pp = gm1 * (UL[4] - T(0.5) * r0 * q2);
  const T unp = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
  const T cp = sqrt(gamma * pp / r0);
  const T Jp = unp + T(2) * cp / gm1;
  T Jpbar = T(0), unpbar = T(0), vbar[3] = {T(0), T(0), T(0)}, ppbar = T(0), r0bar = T(0);

  if (bt == -5) {  // subsonic inflow
    const T RTt = gamma * T(prm.R) * T(prm.Tt);
    const T a = RTt - T(0.5) * gm1 * Jp * Jp;
    const T b = -T(4) * RTt / gm1;
    const T c = T(4) * RTt / (gm1 * gm1) - Jp * Jp;
    const T disc = sqrt(b * b - T(4) * a * c);
    const T s0 = (-b + disc) / (T(2) * a), s1 = (-b - disc) / (T(2) * a);
    int pick = -1;  // 0: s0, 1: s1 (the forward's choice)
    if (s0 >= T(0) && s1 >= T(0)) pick = s0 < s1 ? 0 : 1;
    else if (s0 >= T(0)) pick = 0;
    else if (s1 >= T(0)) pick = 1;
    if (pick < 0) return 0;  // no root: the ghost state does not depend on UL
    const T Mb = pick == 0 ? s0 : s1;
    const T Tt = T(prm.Tt), Pt = T(prm.Pt), R = T(prm.R);
    const T den = T(1) + T(0.5) * gm1 * Mb * Mb;
    const T Tb = Tt / den;
    const T Pb = Pt * pow(Tb / Tt, gamma / gm1);
    const T rb = Pb / (R * Tb);
    const T cb = sqrt(gamma * Pb / rb);
    // Ub = (rb, rb ub, Pb/gm1 + rb |ub|^2 / 2), ub = -Mb cb n
    T rbbar = Ubbar[0], Mbbar = T(0), cbbar = T(0), Pbbar = Ubbar[4] / gm1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T ubk = -Mb * cb * n[k];
      rbbar += Ubbar[1 + k] * ubk;
      const T ubbar = Ubbar[1 + k] * rb;
      Mbbar += -ubbar * cb * n[k];
      cbbar += -ubbar * Mb * n[k];
    }
    rbbar += T(0.5) * Ubbar[4] * Mb * Mb * cb * cb;
    Mbbar += Ubbar[4] * rb * Mb * cb * cb;
    cbbar += Ubbar[4] * rb * Mb * Mb * cb;
    // cb = sqrt(gamma Pb / rb)
    Pbbar += cbbar * cb / (T(2) * Pb);
    rbbar += -cbbar * cb / (T(2) * rb);
    // rb = Pb / (R Tb)
    Pbbar += rbbar / (R * Tb);
    T Tbbar = -rbbar * rb / Tb;
    // Pb = Pt (Tb/Tt)^(gamma/gm1)
    Tbbar += Pbbar * Pb * (gamma / gm1) / Tb;
    // Tb = Tt / den, den = 1 + gm1 Mb^2 / 2
    Mbbar += -Tbbar * Tb / den * gm1 * Mb;
    // Mb = (-b +- disc) / (2 a)
    const T sgn = pick == 0 ? T(1) : T(-1);
    const T discbar = Mbbar * sgn / (T(2) * a);
    T abar = -Mbbar * Mb / a;
    // disc = sqrt(b^2 - 4 a c)
    abar += -discbar * T(2) * c / disc;
    const T cbar = -discbar * T(2) * a / disc;
    // a = RTt - gm1 Jp^2 / 2, c = 4 RTt / gm1^2 - Jp^2
    Jpbar = -abar * gm1 * Jp - cbar * T(2) * Jp;
  } else {  // subsonic outflow
    const T Pf = T(prm.P);
    const T Sp = pp / pow(r0, gamma);
    const T rb = pow(Pf / Sp, T(1) / gamma);
    const T cb = sqrt(gamma * Pf / rb);
    const T unb = Jp - T(2) * cb / gm1;
    T ub[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) ub[k] = v[k] - unp * n[k] + unb * n[k];
    // Ub = (rb, rb ub, Pf/gm1 + rb |ub|^2 / 2)
    T rbbar = Ubbar[0], unbbar = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      rbbar += Ubbar[1 + k] * ub[k] + T(0.5) * Ubbar[4] * ub[k] * ub[k];
      const T ubbar = Ubbar[1 + k] * rb + Ubbar[4] * rb * ub[k];
      vbar[k] += ubbar;
      unpbar += -ubbar * n[k];
      unbbar += ubbar * n[k];
    }
    // unb = Jp - 2 cb / gm1
    Jpbar += unbbar;
    const T cbbar = -T(2) * unbbar / gm1;
    // cb = sqrt(gamma Pf / rb)
    rbbar += -cbbar * cb / (T(2) * rb);
    // rb = (Pf / Sp)^(1/gamma)
    const T Spbar = -rbbar * rb / (gamma * Sp);
    // Sp = pp rho^-gamma
    ppbar += Spbar * Sp / pp;
    r0bar += -Spbar * gamma * Sp / r0;
  }
  // Jp = unp + 2 cp / gm1, cp = sqrt(gamma pp / rho)
  unpbar += Jpbar;
  const T cpbar = T(2) * Jpbar / gm1;
  ppbar += cpbar * cp / (T(2) * pp);
  r0bar += -cpbar * cp / (T(2) * r0);
  // unp = v . n
#pragma unroll
  for (int k = 0; k < 3; ++k) vbar[k] += unpbar * n[k];
  // pp = gm1 (E - rho q2 / 2)
  ULbar[4] += gm1 * ppbar;
  r0bar += -T(0.5) * gm1 * q2 * ppbar;
  const T q2bar = -T(0.5) * gm1 * r0 * ppbar;
  // q2 = |v|^2, v = m / rho
  T irbar = T(0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T vk = vbar[k] + T(2) * v[k] * q2bar;
    ULbar[1 + k] += vk * ir;
    irbar += vk * UL[1 + k];
  }
  ULbar[0] += r0bar - irbar * ir * ir;
  return 0;
}

}  // namespace dgb
