// Host-side check hooks (include/dgb200_check.h): the pointwise physics the
// kernels use and its hand-written reverse mode, run on the CPU so tests can
// compare the VJPs with finite differences without a GPU.
#include <cstring>

#include "../../include/dgb200.h"
#include "../../include/dgb200_check.h"
#include "host.hpp"
#include "physics_vjp.cuh"

using namespace dgb;

extern "C" int dgb_check_pointwise(int which, const double* x, const double* ybar, const double* aux, double* y,
                                   double* xbar)
{
  if (!x || !aux || !y) return DGB_ERR_ARG;
  switch (which) {
    case DGB_CHECK_EULER_FLUX: {  // x = U[5], aux = {gamma}
      double F[3][5];
      euler_flux(x, aux[0], F);
      std::memcpy(y, F, sizeof F);
      if (xbar && ybar) {
        double Fb[3][5];
        std::memcpy(Fb, ybar, sizeof Fb);
        for (int i = 0; i < 5; ++i) xbar[i] = 0.;
        euler_flux_vjp(x, aux[0], Fb, xbar);
      }
      return DGB_OK;
    }
    case DGB_CHECK_EULER_FLUX_N: {  // x = U[5], aux = {gamma, n[3]}
      euler_flux_n(x, aux[0], aux + 1, y);
      if (xbar && ybar) {
        for (int i = 0; i < 5; ++i) xbar[i] = 0.;
        euler_flux_n_vjp(x, aux[0], aux + 1, ybar, xbar);
      }
      return DGB_OK;
    }
    case DGB_CHECK_VISC_FLUX:       // x = S[5] G[3][5], aux = {mu}
    case DGB_CHECK_VISC_FLUX_HEAT: {  // aux = {mu, kq}
      const double kq = which == DGB_CHECK_VISC_FLUX_HEAT ? aux[1] : 0.;
      double G[3][5], Q[3][5];
      std::memcpy(G, x + 5, sizeof G);
      visc_flux(x, G, aux[0], Q, kq);
      std::memcpy(y, Q, sizeof Q);
      if (xbar && ybar) {
        double Qb[3][5], Gb[3][5] = {};
        std::memcpy(Qb, ybar, sizeof Qb);
        for (int i = 0; i < 5; ++i) xbar[i] = 0.;
        visc_flux_vjp(x, G, aux[0], Qb, xbar, Gb, kq);
        std::memcpy(xbar + 5, Gb, sizeof Gb);
      }
      return DGB_OK;
    }
    case DGB_CHECK_VISC_RANK1:       // x = S[5] d[5], aux = {mu, n[3]}
    case DGB_CHECK_VISC_RANK1_HEAT: {  // aux = {mu, n[3], kq}
      const double kq = which == DGB_CHECK_VISC_RANK1_HEAT ? aux[4] : 0.;
      double Q[3][5];
      visc_rank1(x, x + 5, aux + 1, aux[0], Q, kq);
      std::memcpy(y, Q, sizeof Q);
      if (xbar && ybar) {
        double Qb[3][5];
        std::memcpy(Qb, ybar, sizeof Qb);
        for (int i = 0; i < 10; ++i) xbar[i] = 0.;
        visc_rank1_vjp(x, x + 5, aux + 1, aux[0], Qb, xbar, xbar + 5, kq);
      }
      return DGB_OK;
    }
    case DGB_CHECK_VISC_JUMP_N:       // x = S[5] d[5], aux = {mu, n[3]}
    case DGB_CHECK_VISC_JUMP_N_HEAT: {  // aux = {mu, n[3], kq}
      const double kq = which == DGB_CHECK_VISC_JUMP_N_HEAT ? aux[4] : 0.;
      visc_jump_n(x, x + 5, aux + 1, aux[0], y, kq);
      if (xbar && ybar) {
        for (int i = 0; i < 10; ++i) xbar[i] = 0.;
        visc_jump_n_vjp(x, x + 5, aux + 1, aux[0], ybar, xbar, xbar + 5, kq);
      }
      return DGB_OK;
    }
    case DGB_CHECK_ROE: {  // x = Ul[5] Ur[5], aux = {gamma, n[3]}
      roe_flux(x, x + 5, aux + 1, aux[0], y);
      if (xbar && ybar) {
        for (int i = 0; i < 10; ++i) xbar[i] = 0.;
        roe_flux_vjp(x, x + 5, aux + 1, aux[0], ybar, xbar, xbar + 5);
      }
      return DGB_OK;
    }
    case DGB_CHECK_BOUNDARY_STATE: {  // x = UL[5], aux = {btype, n[3], gamma, R, P, Pt, Tt, Ufr[5] (, Tw)}
      DevParams prm{};
      prm.gamma = aux[4];
      prm.R = aux[5];
      prm.P = aux[6];
      prm.Pt = aux[7];
      prm.Tt = aux[8];
      for (int r = 0; r < 5; ++r) prm.Ufr[r] = aux[9 + r];
      const int bt = (int)aux[0];
      if (bt == -8) prm.Tw = aux[14];
      if (boundary_state(bt, x, aux + 1, prm, y)) return DGB_ERR_BOUNDARY;
      if (xbar && ybar) {
        for (int i = 0; i < 5; ++i) xbar[i] = 0.;
        if (boundary_state_vjp(bt, x, aux + 1, prm, ybar, xbar)) return DGB_ERR_UNSUPPORTED;
      }
      return DGB_OK;
    }
    case DGB_CHECK_FACE_MATCH:  // x = {n_own[3], n_nbr[3], fJ_own, fJ_nbr}
      y[0] = face_mismatch(x, x + 3, 1, x[6], x[7]) ? 1. : 0.;
      return DGB_OK;
  }
  return DGB_ERR_ARG;
}
