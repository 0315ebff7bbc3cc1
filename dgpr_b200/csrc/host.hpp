// Host-side precompute shared by the C ABI and the CLI driver: 1D operators of
// the tensor-product basis, per-element affine geometry, neighbour table.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dgb200.h"

namespace dgb {

constexpr int kMaxP = 7;  // P = p + 1 supported by the kernels (p <= 6)

// Element geometry record stride in doubles (see ElemGeo layout below).
constexpr int kGeoStride = 36;
// Offsets inside one element record:
//   [0..8]   Jinv, row-major, Jinv[i][c] = d xi_i / d x_c
//   [9]      detJ
//   [10..27] outward unit normal of local face lf at [10 + 3*lf]
//   [28..33] surface Jacobian of local face lf
constexpr int kGeoJinv = 0, kGeoDetJ = 9, kGeoN = 10, kGeoFJ = 28;

// Exact 1D operators of the order-p equispaced Lagrange basis sampled at the
// P = p+1 point Gauss-Legendre rule on [0,1] (quadrature.cpp:187-205,
// basis.cpp:91-148).  All matrices are row-major P x P.
struct Ops1D {
  int p = 0, P = 1;
  std::vector<double> x, w;   // GL nodes / weights
  std::vector<double> B;      // B[q][i]  = l_i(x_q)
  std::vector<double> Bd;     // Bd[q][i] = l_i'(x_q)
  std::vector<double> Dq;     // Dq[q][k] = L_k'(x_q), L_k the Lagrange basis on the GL nodes
  std::vector<double> M1;     // M1[i][j] = sum_q w_q l_i(x_q) l_j(x_q)
  std::vector<double> M1i;    // inverse of M1
  std::vector<double> K;      // K = B M1i B^T  (face lifting factor)
  std::vector<double> E[2];   // E[end][i] = l_i(end), end 0 -> xi=0, 1 -> xi=1
  std::vector<double> D[2];   // D[end][i] = l_i'(end)
  std::vector<double> Wb;     // Wb[i] = sum_q w_q l_i(x_q)
  double cend[2] = {0, 0};    // E[end]^T M1i E[end]
};

int build_ops(int p, Ops1D& ops);

// Gauss-Jordan inverse with partial pivoting, row-major n x n, in place.
int invert_dense(int n, double* A);

double lagrange1d(int i, int p, double x);
double lagrange1d_deriv(int i, int p, double x);
void gauss_legendre(int n, double a, double b, double* x, double* w);

// Affine element geometry + neighbour table for a structured nx*ny*nz mesh.
//   geo[e*kGeoStride + ...]  as documented above
//   nbr[e*6 + lf]            neighbour element (>= 0) or btype code (< 0)
// Returns DGB_ERR_UNSUPPORTED for elements whose Jacobian is not constant
// (curved geometry), DGB_ERR_GEOMETRY for singular Jacobians or mismatched
// periodic sides.
int build_geometry(const dgb_mesh_desc& m, const Ops1D& ops, std::vector<double>& geo,
                   std::vector<int32_t>& nbr, std::string& why);

// Total conditions used by the subsonic inflow state (solve.cpp:167-175).
void total_conditions(const dgb_params& prm, double* Tt, double* Pt);

// Records msg as the calling thread's dgb_last_error_message and returns code.
int set_last_error(int code, const std::string& msg);

}  // namespace dgb
