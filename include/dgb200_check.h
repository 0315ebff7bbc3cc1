/* dgb200 check hooks: the pointwise physics of the residual kernels and its
 * hand-written reverse mode, callable on the host (no GPU) so the adjoint's
 * building blocks can be checked against finite differences.  Not part of the
 * solver interface; the reference has no counterpart (it has no adjoint). */
#ifndef DGB200_CHECK_H
#define DGB200_CHECK_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DGB_CHECK_EULER_FLUX = 0,      /* x = U[5];          aux = {gamma};       y = F[3][5] (flux.cpp:24-48) */
  DGB_CHECK_EULER_FLUX_N = 1,    /* x = U[5];          aux = {gamma, n[3]}; y = F.n[5] */
  DGB_CHECK_VISC_FLUX = 2,       /* x = S[5], G[3][5]; aux = {mu};          y = A(S,G)[3][5] (flux.cpp:156-202) */
  DGB_CHECK_VISC_RANK1 = 3,      /* x = S[5], d[5];    aux = {mu, n[3]};    y = A(S, d n^T)[3][5] */
  DGB_CHECK_VISC_JUMP_N = 4,     /* x = S[5], d[5];    aux = {mu, n[3]};    y = A(S, d n^T).n[5] */
  DGB_CHECK_ROE = 5,             /* x = Ul[5], Ur[5];  aux = {gamma, n[3]}; y = Roe flux[5] (flux.cpp:56-154) */
  DGB_CHECK_BOUNDARY_STATE = 6,  /* x = UL[5]; aux = {btype, n[3], gamma, R, P, Pt, Tt, Ufr[5]}; y = Ub[5]
                                    (bound_states.cpp:24-130); reverse mode for btype -3 .. -8;
                                    btype -8 (isothermal wall) reads Tw from aux[14] */
  /* The viscous forms 2-4 with the optional heat flux kq = mu gamma / Pr
   * in the energy row (an extension: the reference conducts no heat). */
  DGB_CHECK_VISC_FLUX_HEAT = 7,    /* x as 2; aux = {mu, kq} */
  DGB_CHECK_VISC_RANK1_HEAT = 8,   /* x as 3; aux = {mu, n[3], kq} */
  DGB_CHECK_VISC_JUMP_N_HEAT = 9,  /* x as 4; aux = {mu, n[3], kq} */
  /* The face-match test of the geometry builders (host and device): the two
   * sides of an interior face must have opposite unit normals and equal
   * surface Jacobians.  x = {n_own[3], n_nbr[3], fJ_own, fJ_nbr}; aux unused;
   * y[0] = 1 on a mismatch (NaN counts as one), else 0.  No reverse mode. */
  DGB_CHECK_FACE_MATCH = 10
};

/* Evaluates function `which` at x into y; when ybar and xbar are non-NULL
 * also writes xbar = (dy/dx)^T ybar. */
int dgb_check_pointwise(int which, const double* x, const double* ybar, const double* aux, double* y,
                        double* xbar);

#ifdef __cplusplus
}
#endif

#endif /* DGB200_CHECK_H */
