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

// Rank-one viscous flux Q = A(S, d n^T) (visc_rank1): Qbar[3][5] -> Sbar, dbar
template <class T>
DGB_HD void visc_rank1_vjp(const T* S, const T* d, const T* n, T mu, const T Qbar[3][5], T* Sbar, T* dbar,
                           T kq = T(0))
{
  if (kq != T(0)) heat_y_vjp(S, d, kq * (Qbar[0][4] * n[0] + Qbar[1][4] * n[1] + Qbar[2][4] * n[2]), Sbar, dbar);
  const T lam = -(T(2) / T(3)) * mu;
  const T ir = T(1) / S[0];
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

// Normal component A(S, d n^T).n (visc_jump_n): Qnbar[5] -> Sbar, dbar
template <class T>
DGB_HD void visc_jump_n_vjp(const T* S, const T* d, const T* n, T mu, const T* Qnbar, T* Sbar, T* dbar,
                            T kq = T(0))
{
  if (kq != T(0))
    heat_y_vjp(S, d, kq * Qnbar[4] * (n[0] * n[0] + n[1] * n[1] + n[2] * n[2]), Sbar, dbar);
  const T lam = -(T(2) / T(3)) * mu;
  const T ir = T(1) / S[0];
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

// Roe flux with entropy fix (roe_flux): fbar[5] -> Ulbar, Urbar
template <class T>
DGB_HD void roe_flux_vjp(const T* Ul, const T* Ur, const T* n, T g, const T* fbar, T* Ulbar, T* Urbar)
{
  // ---- forward, as roe_flux
  const T gm1 = g - T(1);
  const T rl = Ul[0], irl = T(1) / rl, ul = Ul[1] * irl, vl = Ul[2] * irl, wl = Ul[3] * irl;
  const T ql2 = ul * ul + vl * vl + wl * wl;
  const T pl = gm1 * (Ul[4] - T(0.5) * rl * ql2);
  const T Hl = (Ul[4] + pl) * irl;
  const T rr = Ur[0], irr = T(1) / rr, ur = Ur[1] * irr, vr = Ur[2] * irr, wr = Ur[3] * irr;
  const T qr2 = ur * ur + vr * vr + wr * wr;
  const T pr = gm1 * (Ur[4] - T(0.5) * rr * qr2);
  const T Hr = (Ur[4] + pr) * irr;
  const T sl = sqrt(rl), sr = sqrt(rr), iden = T(1) / (sl + sr);
  const T uk[3] = {(sl * ul + sr * ur) * iden, (sl * vl + sr * vr) * iden, (sl * wl + sr * wr) * iden};
  const T H = (sl * Hl + sr * Hr) * iden;
  const T dr = rr - rl;
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
  const T ulk[3] = {ul, vl, wl}, urk[3] = {ur, vr, wr};
  const T unl = ul * n[0] + vl * n[1] + wl * n[2];
  const T unr = ur * n[0] + vr * n[1] + wr * n[2];

  // ---- reverse
  T rlb = T(0), rrb = T(0), unlb = T(0), unrb = T(0), plb = T(0), prb = T(0), Hlb = T(0), Hrb = T(0);
  T ulkb[3] = {T(0), T(0), T(0)}, urkb[3] = {T(0), T(0), T(0)}, ukb[3] = {T(0), T(0), T(0)};
  T a3b = T(0), drb = T(0), dmb[3] = {T(0), T(0), T(0)}, dEb = T(0), Hb = T(0), unb = T(0);
  const T h = T(0.5);
  // central parts
  rlb += h * fbar[0] * unl + h * fbar[4] * Hl * unl;
  rrb += h * fbar[0] * unr + h * fbar[4] * Hr * unr;
  unlb += h * fbar[0] * rl + h * fbar[4] * rl * Hl;
  unrb += h * fbar[0] * rr + h * fbar[4] * rr * Hr;
  Hlb += h * fbar[4] * rl * unl;
  Hrb += h * fbar[4] * rr * unr;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T fb = fbar[1 + k];
    rlb += h * fb * ulk[k] * unl;
    rrb += h * fb * urk[k] * unr;
    unlb += h * fb * rl * ulk[k];
    unrb += h * fb * rr * urk[k];
    ulkb[k] += h * fb * rl * unl;
    urkb[k] += h * fb * rr * unr;
    plb += h * fb * n[k];
    prb += h * fb * n[k];
  }
  // dissipation: -1/2 (a3 dr + C1), -1/2 (a3 dm_k + C1 u_k + C2 n_k), -1/2 (a3 dE + C1 H + C2 un)
  a3b += -h * (fbar[0] * dr + fbar[1] * dm[0] + fbar[2] * dm[1] + fbar[3] * dm[2] + fbar[4] * dE);
  drb += -h * fbar[0] * a[2];
  dEb += -h * fbar[4] * a[2];
  T C1b = -h * (fbar[0] + fbar[4] * H);
  T C2b = -h * fbar[4] * un;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dmb[k] += -h * fbar[1 + k] * a[2];
    C1b += -h * fbar[1 + k] * uk[k];
    C2b += -h * fbar[1 + k] * n[k];
    ukb[k] += -h * fbar[1 + k] * C1;
  }
  Hb += -h * fbar[4] * C1;
  unb += -h * fbar[4] * C2;
  // unl = ulk . n, unr = urk . n
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    ulkb[k] += unlb * n[k];
    urkb[k] += unrb * n[k];
  }
  // C1 = G1 ic^2 (s1 - a3) + G2 ic s2 ; C2 = G1 ic s2 + (s1 - a3) G2
  T G1b = C1b * ic * ic * (s1 - a[2]) + C2b * ic * s2;
  T G2b = C1b * ic * s2 + C2b * (s1 - a[2]);
  T icb = C1b * (T(2) * G1 * ic * (s1 - a[2]) + G2 * s2) + C2b * G1 * s2;
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
  // s1, s2
  T ab[3] = {h * (s1b + s2b), h * (s1b - s2b), a3b};
  // a_i from l_i (with the entropy fix where it was taken)
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
  // un = uk . n
#pragma unroll
  for (int k = 0; k < 3; ++k) ukb[k] += unb * n[k];
  // ic = 1/c ; c = sqrt(gm1 (H - q2/2))
  cb += -icb * ic * ic;
  const T c2b = cb / (T(2) * c);
  Hb += gm1 * c2b;
  q2b += -h * gm1 * c2b;
#pragma unroll
  for (int k = 0; k < 3; ++k) ukb[k] += T(2) * uk[k] * q2b;
  // differences
  rrb += drb;
  rlb -= drb;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Urbar[1 + k] += dmb[k];
    Ulbar[1 + k] -= dmb[k];
  }
  Urbar[4] += dEb;
  Ulbar[4] -= dEb;
  // Roe averages: uk = (sl ulk + sr urk) iden, H = (sl Hl + sr Hr) iden
  T slb = Hb * Hl * iden, srb = Hb * Hr * iden;
  T idenb = Hb * (sl * Hl + sr * Hr);
  Hlb += Hb * sl * iden;
  Hrb += Hb * sr * iden;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    slb += ukb[k] * ulk[k] * iden;
    srb += ukb[k] * urk[k] * iden;
    ulkb[k] += ukb[k] * sl * iden;
    urkb[k] += ukb[k] * sr * iden;
    idenb += ukb[k] * (sl * ulk[k] + sr * urk[k]);
  }
  const T sumb = -idenb * iden * iden;
  slb += sumb;
  srb += sumb;
  rlb += slb / (T(2) * sl);
  rrb += srb / (T(2) * sr);
  // H_side = (U4 + p) ir ; p = gm1 (U4 - r q2/2) ; u = U_{1..3} ir
  T irlb = Hlb * (Ul[4] + pl), irrb = Hrb * (Ur[4] + pr);
  plb += Hlb * irl;
  prb += Hrb * irr;
  Ulbar[4] += Hlb * irl + gm1 * plb;
  Urbar[4] += Hrb * irr + gm1 * prb;
  rlb += -h * gm1 * ql2 * plb;
  rrb += -h * gm1 * qr2 * prb;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    ulkb[k] += -gm1 * rl * ulk[k] * plb;
    urkb[k] += -gm1 * rr * urk[k] * prb;
    Ulbar[1 + k] += ulkb[k] * irl;
    Urbar[1 + k] += urkb[k] * irr;
    irlb += ulkb[k] * Ul[1 + k];
    irrb += urkb[k] * Ur[1 + k];
  }
  rlb += -irlb * irl * irl;
  rrb += -irrb * irr * irr;
  Ulbar[0] += rlb;
  Urbar[0] += rrb;
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
