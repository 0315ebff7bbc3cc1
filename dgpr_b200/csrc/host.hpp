// Host-side precompute shared by the C ABI and the CLI driver: 1D operators of
// the tensor-product basis, per-element affine geometry, neighbour table.
#pragma once

#include <cmath>
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
  std::vector<double> Bi;     // Bi[i][q] = (B^-1)[i][q]: nodal coefficients from values at the GL nodes
  std::vector<double> E[2];   // E[end][i] = l_i(end), end 0 -> xi=0, 1 -> xi=1
  std::vector<double> D[2];   // D[end][i] = l_i'(end)
  std::vector<double> Wb;     // Wb[i] = sum_q w_q l_i(x_q)
  double cend[2] = {0, 0};    // E[end]^T M1i E[end]
  std::vector<double> EL[2];  // EL[end][q] = (E[end] B^-1)[q]: value at xi = end of the
                              // Lagrange polynomial through the GL nodes that is 1 at node q
  std::vector<double> DL[2];  // DL[end][q] = (D[end] B^-1)[q]: its derivative there
};

// Curved (non-affine) elements carry their geometry per point:
//   volume   gv[e][c][P^3]      c < kVolC:  Jinv[9] (row-major d xi_i / d x_c), detJ
//   faces    gf[e][lf][c][P^2]  c < kFaceC: Jinv[9], outward unit normal[3],
//                               surface Jacobian, BR2 lifting scale
// The lifting scale of a face point is the diagonal of the face-restricted
// lifting operator E_f Minv E_f^T times w_t1 w_t2:
//   sum_a EL[end][a]^2 / (w_a detJ(a, t1, t2))   (= cend / detJ when affine).
constexpr int kVolC = 10, kVolDetJ = 9;
constexpr int kFaceC = 14, kFaceN = 9, kFaceFJ = 12, kFaceLift = 13;

// True unless the two sides of an interior face agree: opposite unit normals
// (ng = -nh) and equal surface Jacobians, to 1e-10.  Written as the negation
// of "both within tolerance" so that a NaN normal or surface Jacobian (a
// degenerate face) counts as a mismatch.  sn: stride between the normal's
// components.
__host__ __device__ inline bool face_mismatch(const double* ng, const double* nh, int sn, double fJg, double fJh)
{
  bool ok = true;
  for (int r = 0; r < 3; ++r) ok = ok && (fabs(ng[r * sn] + nh[r * sn]) <= 1e-10);
  return !(ok && fabs(fJg - fJh) / fJg <= 1e-10);
}

int build_ops(int p, Ops1D& ops);

// Gauss-Jordan inverse with partial pivoting, row-major n x n, in place.
int invert_dense(int n, double* A);

double lagrange1d(int i, int p, double x);
double lagrange1d_deriv(int i, int p, double x);
void gauss_legendre(int n, double a, double b, double* x, double* w);

// Element geometry + neighbour table for a structured nx*ny*nz mesh.
//   geo[e*kGeoStride + ...]  affine record as documented above (Jacobian at the
//                            element centre)
//   nbr[e*6 + lf]            neighbour element (>= 0) or btype code (< 0)
// When some element's Jacobian is not constant (curved geometry) `curved` is
// set and gv / gf receive the per-point geometry of every element (layout
// above); otherwise they are left empty.  Returns DGB_ERR_GEOMETRY for
// singular Jacobians or faces that do not match their neighbour's.
int build_geometry(const dgb_mesh_desc& m, const Ops1D& ops, std::vector<double>& geo,
                   std::vector<int32_t>& nbr, std::string& why, bool& curved, std::vector<double>& gv,
                   std::vector<double>& gf);

// The parts of build_geometry that stay on the host in the device build:
// argument checks, and the neighbour table.
int check_mesh(const dgb_mesh_desc& m, std::string& why);
void build_neighbours(const dgb_mesh_desc& m, std::vector<int32_t>& nbr);

// Lagrange values l[m][i] and derivatives d[m][i] (i <= q) of the order-q
// geometry basis at the reference coordinates the geometry is sampled at:
// rows m < P the Gauss points, then 0, 1 and 1/2; with the face-lifting
// weights EL and the Gauss weights.  Built by the host's lagrange1d, so the
// device builder starts from the host builder's numbers.
struct GeoTables {
  double l[kMaxP + 3][8], d[kMaxP + 3][8];
  double EL[2][kMaxP], w[kMaxP];
};
void build_geo_tables(const Ops1D& ops, int q, GeoTables& t);

// build_geometry on the device (geometry.cu), bit-identical to the host
// builder: d_geo (E * kGeoStride doubles, allocated by the caller) receives
// the affine records; when an element is curved, *d_gv and *d_gf are
// allocated and filled with the per-point geometry.  nbr is the host
// neighbour table and d_nbr its device copy.  The same checks in the same
// order, with the same messages; CUDA failures return DGB_ERR_CUDA.
int build_geometry_device(const dgb_mesh_desc& m, const Ops1D& ops, const std::vector<int32_t>& nbr,
                          const int32_t* d_nbr, void* stream, double* d_geo, double** d_gv, double** d_gf,
                          bool& curved, std::string& why);

// Total conditions used by the subsonic inflow state (solve.cpp:167-175).
void total_conditions(const dgb_params& prm, double* Tt, double* Pt);

// Records msg as the calling thread's dgb_last_error_message and returns code.
int set_last_error(int code, const std::string& msg);

}  // namespace dgb
