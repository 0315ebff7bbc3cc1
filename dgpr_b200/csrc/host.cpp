// Host-side precompute: Gauss-Legendre rule, Lagrange basis, 1D tensor-product
// operators, affine element geometry and the structured neighbour table.
#include "host.hpp"

#include <algorithm>
#include <thread>

#include <cmath>
#include <cstdio>
#include <cstring>

namespace dgb {

// Newton iteration on P_n from the Chebyshev-like guess cos(pi (i+3/4)/(n+1/2)),
// P_n and P_n' from the three-term recurrence.  Same rule as the reference's
// gauss_legendre_1d_dbl (quadrature.cpp:84-173); ascending nodes on [a,b].
void gauss_legendre(int n, double a, double b, double* x, double* w)
{
  if (n == 1) {
    x[0] = 0.5 * (a + b);
    w[0] = b - a;
    return;
  }
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; ++i) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5));
    double pn = 0., dpn = 1.;
    for (int it = 0; it < 100; ++it) {
      double pm = 1., pc = z;
      for (int k = 2; k <= n; ++k) {
        double pk = ((2. * k - 1.) * z * pc - (k - 1.) * pm) / k;
        pm = pc;
        pc = pk;
      }
      pn = pc;
      dpn = n * (z * pc - pm) / (z * z - 1.);
      double step = pn / dpn;
      z -= step;
      if (std::fabs(step) < 1e-16) break;
    }
    double pm = 1., pc = z;
    for (int k = 2; k <= n; ++k) {
      double pk = ((2. * k - 1.) * z * pc - (k - 1.) * pm) / k;
      pm = pc;
      pc = pk;
    }
    dpn = n * (z * pc - pm) / (z * z - 1.);
    const int j = n - 1 - i;
    x[j] = a + (b - a) * 0.5 * (z + 1.);
    w[j] = (b - a) / ((1. - z * z) * dpn * dpn);
  }
}

// l_i(x) for equispaced nodes i/p on [0,1] (basis.cpp:91-104); p = 0 is the
// constant 1.
double lagrange1d(int i, int p, double x)
{
  if (p == 0) return 1.;
  const double xi = (double)i / p;
  double v = 1.;
  for (int j = 0; j <= p; ++j)
    if (j != i) v *= (x - (double)j / p) / (xi - (double)j / p);
  return v;
}

// l_i'(x) as a sum over the dropped factor (basis.cpp:125-148).
double lagrange1d_deriv(int i, int p, double x)
{
  if (p == 0) return 0.;
  const double xi = (double)i / p;
  double s = 0.;
  for (int j = 0; j <= p; ++j) {
    if (j == i) continue;
    double m = 1.;
    for (int k = 0; k <= p; ++k)
      if (k != i && k != j) m *= (x - (double)k / p) / (xi - (double)k / p);
    s += m / (xi - (double)j / p);
  }
  return s;
}

int invert_dense(int n, double* A)
{
  std::vector<double> a(2 * (size_t)n * n);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) {
      a[2 * n * r + c] = A[n * r + c];
      a[2 * n * r + n + c] = r == c ? 1. : 0.;
    }
  for (int k = 0; k < n; ++k) {
    int piv = k;
    for (int r = k + 1; r < n; ++r)
      if (std::fabs(a[2 * n * r + k]) > std::fabs(a[2 * n * piv + k])) piv = r;
    if (a[2 * n * piv + k] == 0. || !std::isfinite(a[2 * n * piv + k])) return 1;
    if (piv != k)
      for (int c = 0; c < 2 * n; ++c) std::swap(a[2 * n * k + c], a[2 * n * piv + c]);
    const double d = a[2 * n * k + k];
    for (int c = 0; c < 2 * n; ++c) a[2 * n * k + c] /= d;
    for (int r = 0; r < n; ++r) {
      if (r == k) continue;
      const double f = a[2 * n * r + k];
      if (f == 0.) continue;
      for (int c = 0; c < 2 * n; ++c) a[2 * n * r + c] -= f * a[2 * n * k + c];
    }
  }
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) A[n * r + c] = a[2 * n * r + n + c];
  return 0;
}

int build_ops(int p, Ops1D& o)
{
  if (p < 0 || p + 1 > kMaxP) return DGB_ERR_UNSUPPORTED;
  const int P = p + 1;
  o.p = p;
  o.P = P;
  o.x.assign(P, 0.);
  o.w.assign(P, 0.);
  gauss_legendre(P, 0., 1., o.x.data(), o.w.data());
  o.B.assign(P * P, 0.);
  o.Bd.assign(P * P, 0.);
  o.Dq.assign(P * P, 0.);
  for (int q = 0; q < P; ++q)
    for (int i = 0; i < P; ++i) {
      o.B[P * q + i] = lagrange1d(i, p, o.x[q]);
      o.Bd[P * q + i] = lagrange1d_deriv(i, p, o.x[q]);
    }
  // derivative of the Lagrange interpolant through the GL nodes
  for (int q = 0; q < P; ++q)
    for (int k = 0; k < P; ++k) {
      double s = 0.;
      for (int j = 0; j < P; ++j) {
        if (j == k) continue;
        double m = 1.;
        for (int l = 0; l < P; ++l)
          if (l != k && l != j) m *= (o.x[q] - o.x[l]) / (o.x[k] - o.x[l]);
        s += m / (o.x[k] - o.x[j]);
      }
      o.Dq[P * q + k] = s;
    }
  o.M1.assign(P * P, 0.);
  for (int i = 0; i < P; ++i)
    for (int j = 0; j < P; ++j) {
      double s = 0.;
      for (int q = 0; q < P; ++q) s += o.w[q] * o.B[P * q + i] * o.B[P * q + j];
      o.M1[P * i + j] = s;
    }
  o.M1i = o.M1;
  if (invert_dense(P, o.M1i.data())) return DGB_ERR_GEOMETRY;
  o.Bi = o.B;  // B[q][i] -> Bi[i][q]
  if (invert_dense(P, o.Bi.data())) return DGB_ERR_GEOMETRY;
  for (int e = 0; e < 2; ++e) {
    o.E[e].assign(P, 0.);
    o.D[e].assign(P, 0.);
    for (int i = 0; i < P; ++i) {
      o.E[e][i] = lagrange1d(i, p, (double)e);
      o.D[e][i] = lagrange1d_deriv(i, p, (double)e);
    }
    double s = 0.;
    for (int i = 0; i < P; ++i)
      for (int j = 0; j < P; ++j) s += o.E[e][i] * o.M1i[P * i + j] * o.E[e][j];
    o.cend[e] = s;
    o.EL[e].assign(P, 0.);
    o.DL[e].assign(P, 0.);
    for (int q = 0; q < P; ++q) {
      double v = 0., d = 0.;
      for (int i = 0; i < P; ++i) {
        v += o.E[e][i] * o.Bi[P * i + q];
        d += o.D[e][i] * o.Bi[P * i + q];
      }
      o.EL[e][q] = v;
      o.DL[e][q] = d;
    }
  }
  o.Wb.assign(P, 0.);
  for (int i = 0; i < P; ++i) {
    double s = 0.;
    for (int q = 0; q < P; ++q) s += o.w[q] * o.B[P * q + i];
    o.Wb[i] = s;
  }
  return DGB_OK;
}

namespace {

double det3(const double* m)
{
  return m[0] * m[4] * m[8] + m[1] * m[5] * m[6] + m[2] * m[3] * m[7] - m[2] * m[4] * m[6] -
         m[1] * m[3] * m[8] - m[0] * m[5] * m[7];
}

void inv3(const double* m, double* o)
{
  const double id = 1. / det3(m);
  o[0] = id * (m[4] * m[8] - m[5] * m[7]);
  o[1] = id * (m[2] * m[7] - m[1] * m[8]);
  o[2] = id * (m[1] * m[5] - m[2] * m[4]);
  o[3] = id * (m[5] * m[6] - m[3] * m[8]);
  o[4] = id * (m[0] * m[8] - m[2] * m[6]);
  o[5] = id * (m[2] * m[3] - m[0] * m[5]);
  o[6] = id * (m[3] * m[7] - m[4] * m[6]);
  o[7] = id * (m[1] * m[6] - m[0] * m[7]);
  o[8] = id * (m[0] * m[4] - m[1] * m[3]);
}

void cross(const double* a, const double* b, double* c)
{
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// J[r][c] = d x_r / d xi_c of the order-q isoparametric map at reference point r3
// (geometry_common.cpp:264-290).
void jacobian(const double* X, int q, const double* r3, double* J)
{
  const int Q = q + 1;
  double l[3][8], d[3][8];
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < Q; ++i) {
      l[a][i] = lagrange1d(i, q, r3[a]);
      d[a][i] = lagrange1d_deriv(i, q, r3[a]);
    }
  for (int i = 0; i < 9; ++i) J[i] = 0.;
  for (int k = 0; k < Q; ++k)
    for (int j = 0; j < Q; ++j)
      for (int i = 0; i < Q; ++i) {
        const double* x = X + 3 * (i + Q * (j + Q * k));
        const double g[3] = {d[0][i] * l[1][j] * l[2][k], l[0][i] * d[1][j] * l[2][k],
                             l[0][i] * l[1][j] * d[2][k]};
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) J[3 * r + c] += x[r] * g[c];
      }
}

}  // namespace

namespace {

// face lf, tangential Gauss points (t1, t2) -> reference coordinates
// (tangential axes in axis order: x faces (y,z), y faces (x,z), z faces (x,y))
void face_point(const Ops1D& ops, int lf, int t1, int t2, double* r3)
{
  const int a = lf >> 1;
  const int ax1 = a == 0 ? 1 : 0, ax2 = a == 2 ? 1 : 2;
  r3[a] = (double)(lf & 1);
  r3[ax1] = ops.x[t1];
  r3[ax2] = ops.x[t2];
}

// outward unit normal and surface Jacobian of face lf from the Jacobian at a
// point of it: the face tangents are Jacobian columns, oriented as surf2vol
// (basis.cpp:180-192) and compute_surface_geometry (geometry_common.cpp:416-454):
// x faces (s,t) -> (y,z), y faces -> (z,x), z faces -> (x,y); low faces flipped
void face_normal(const double* J, int lf, double* n, double* fj)
{
  const int a = lf >> 1;
  const int c1 = a == 0 ? 1 : a == 1 ? 2 : 0;
  const int c2 = a == 0 ? 2 : a == 1 ? 0 : 1;
  const double ts[3] = {J[c1], J[3 + c1], J[6 + c1]};
  const double tt[3] = {J[c2], J[3 + c2], J[6 + c2]};
  double c[3];
  cross(ts, tt, c);
  *fj = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  const double sg = (lf & 1) ? 1. : -1.;
  for (int r = 0; r < 3; ++r) n[r] = sg * c[r] / *fj;
}

// per-point geometry of one element (layout in host.hpp)
int curved_element(const double* X, int q, const Ops1D& ops, double* gv, double* gf, long e, std::string& why)
{
  const int P = ops.P, NB = P * P * P, NQF = P * P;
  double J[9], Ji[9];
  for (int k = 0; k < P; ++k)
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i) {
        const int b = i + P * (j + P * k);
        const double r3[3] = {ops.x[i], ops.x[j], ops.x[k]};
        jacobian(X, q, r3, J);
        const double dJ = det3(J);
        if (!(dJ > 0.) || !std::isfinite(dJ)) {
          char buf[120];
          snprintf(buf, sizeof buf, "element %ld has a non-positive Jacobian determinant", e);
          why = buf;
          return DGB_ERR_GEOMETRY;
        }
        inv3(J, Ji);
        for (int c = 0; c < 9; ++c) gv[c * NB + b] = Ji[c];
        gv[kVolDetJ * NB + b] = dJ;
      }
  for (int lf = 0; lf < 6; ++lf) {
    const int a = lf >> 1, end = lf & 1;
    for (int t2 = 0; t2 < P; ++t2)
      for (int t1 = 0; t1 < P; ++t1) {
        const int fq = t1 + P * t2;
        double r3[3], n[3], fj;
        face_point(ops, lf, t1, t2, r3);
        jacobian(X, q, r3, J);
        inv3(J, Ji);
        face_normal(J, lf, n, &fj);
        double* g = gf + (size_t)lf * kFaceC * NQF;
        for (int c = 0; c < 9; ++c) g[c * NQF + fq] = Ji[c];
        for (int c = 0; c < 3; ++c) g[(kFaceN + c) * NQF + fq] = n[c];
        g[kFaceFJ * NQF + fq] = fj;
        double lift = 0.;
        for (int ia = 0; ia < P; ++ia) {
          const int b = a == 0 ? ia + P * (t1 + P * t2) : a == 1 ? t1 + P * (ia + P * t2) : t1 + P * (t2 + P * ia);
          lift += ops.EL[end][ia] * ops.EL[end][ia] / (ops.w[ia] * gv[kVolDetJ * NB + b]);
        }
        g[kFaceLift * NQF + fq] = lift;
      }
  }
  return DGB_OK;
}

}  // namespace

int check_mesh(const dgb_mesh_desc& m, std::string& why)
{
  if (m.nx <= 0 || m.ny <= 0 || m.nz <= 0 || m.q < 1 || m.q > 7 || !m.nodes) {
    why = "mesh sizes must be positive and 1 <= q <= 7";
    return DGB_ERR_ARG;
  }
  if ((long)m.nx * m.ny * m.nz * 6 > 0x7fffffffL) {
    why = "more elements than a 32-bit neighbour table holds";
    return DGB_ERR_ARG;
  }
  for (int s = 0; s < 6; ++s)
    if (m.bounds[s] > -2 || m.bounds[s] < -8) {
      why = "boundary codes must be btype values -2..-7 (or -8, the isothermal wall)";
      return DGB_ERR_ARG;
    }
  for (int a = 0; a < 3; ++a)
    if ((m.bounds[2 * a] == DGB_BT_PERIODIC) != (m.bounds[2 * a + 1] == DGB_BT_PERIODIC)) {
      why = "periodic boundaries are not matching";  // geometry_shared.cpp:123-131
      return DGB_ERR_GEOMETRY;
    }
  return DGB_OK;
}

// neighbours (geometry_common.cpp:397-414 adjacency, periodic wrap as
// geometry_shared.cpp:205-209)
void build_neighbours(const dgb_mesh_desc& m, std::vector<int32_t>& nbr)
{
  const int nx = m.nx, ny = m.ny, nz = m.nz;
  nbr.assign((size_t)nx * ny * nz * 6, 0);
  const int di[6] = {-1, 1, 0, 0, 0, 0}, dj[6] = {0, 0, -1, 1, 0, 0}, dk[6] = {0, 0, 0, 0, -1, 1};
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long e = i + (long)nx * (j + (long)ny * k);
        for (int lf = 0; lf < 6; ++lf) {
          const int ia = i + di[lf], ja = j + dj[lf], ka = k + dk[lf];
          int side = ia < 0 ? 0 : ia >= nx ? 1 : ja < 0 ? 2 : ja >= ny ? 3 : ka < 0 ? 4 : ka >= nz ? 5 : -1;
          if (side < 0 || m.bounds[side] == DGB_BT_PERIODIC) {
            const long en = ((ia + nx) % nx) + (long)nx * (((ja + ny) % ny) + (long)ny * ((ka + nz) % nz));
            nbr[6 * e + lf] = (int32_t)en;
          } else {
            nbr[6 * e + lf] = (int32_t)m.bounds[side];
          }
        }
      }
}

void build_geo_tables(const Ops1D& ops, int q, GeoTables& t)
{
  std::memset(&t, 0, sizeof t);
  const int P = ops.P;
  for (int m = 0; m < P + 3; ++m) {
    const double r = m < P ? ops.x[m] : m == P ? 0. : m == P + 1 ? 1. : 0.5;
    for (int i = 0; i <= q; ++i) {
      t.l[m][i] = lagrange1d(i, q, r);
      t.d[m][i] = lagrange1d_deriv(i, q, r);
    }
  }
  for (int a = 0; a < P; ++a) {
    t.EL[0][a] = ops.EL[0][a];
    t.EL[1][a] = ops.EL[1][a];
    t.w[a] = ops.w[a];
  }
}

int build_geometry(const dgb_mesh_desc& m, const Ops1D& ops, std::vector<double>& geo,
                   std::vector<int32_t>& nbr, std::string& why, bool& curved, std::vector<double>& gv,
                   std::vector<double>& gf)
{
  curved = false;
  gv.clear();
  gf.clear();
  int rc = check_mesh(m, why);
  if (rc) return rc;
  const int q = m.q, P = ops.P;
  const long E = (long)m.nx * m.ny * m.nz;
  const int Q = q + 1, nq = Q * Q * Q;
  geo.assign((size_t)E * kGeoStride, 0.);

  // sample points for the affinity check: all volume quadrature points and the
  // eight element corners
  std::vector<double> pts;
  for (int k = 0; k < P; ++k)
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i) {
        pts.push_back(ops.x[i]);
        pts.push_back(ops.x[j]);
        pts.push_back(ops.x[k]);
      }
  for (int c = 0; c < 8; ++c) {
    pts.push_back(c & 1);
    pts.push_back((c >> 1) & 1);
    pts.push_back((c >> 2) & 1);
  }
  const int npts = (int)pts.size() / 3;

  // the Jacobian is taken at the element centre: for an affine element it is
  // the same everywhere, and there the q = 1 basis gradients are +-1/4, so
  // equal elements get bit-identical Jacobians
  const double centre[3] = {0.5, 0.5, 0.5};
  for (long e = 0; e < E; ++e) {
    const double* X = m.nodes + (size_t)e * nq * 3;
    double J0[9], J[9];
    jacobian(X, q, centre, J0);
    double scale = 0.;
    for (int i = 0; i < 9; ++i) scale = std::fmax(scale, std::fabs(J0[i]));
    for (int s = 0; s < npts && !curved; ++s) {
      jacobian(X, q, &pts[3 * s], J);
      for (int i = 0; i < 9; ++i)
        if (std::fabs(J[i] - J0[i]) > 1e-11 * scale) curved = true;
    }
    double* g = &geo[(size_t)e * kGeoStride];
    const double dJ = det3(J0);
    if (!(std::fabs(dJ) > 0.) || !std::isfinite(dJ)) {
      char buf[120];
      snprintf(buf, sizeof buf, "element %ld has a singular Jacobian", e);
      why = buf;
      return DGB_ERR_GEOMETRY;
    }
    inv3(J0, g + kGeoJinv);
    g[kGeoDetJ] = dJ;
    for (int lf = 0; lf < 6; ++lf) face_normal(J0, lf, g + kGeoN + 3 * lf, g + kGeoFJ + lf);
  }
  if (curved) {  // per-point geometry, elements split over the host's threads
    const int NB = P * P * P, NQF = P * P;
    gv.assign((size_t)E * kVolC * NB, 0.);
    gf.assign((size_t)E * 6 * kFaceC * NQF, 0.);
    const int nth = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<int> rcs(nth, DGB_OK);
    std::vector<long> fails(nth, E);
    std::vector<std::string> whys(nth);
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; ++t)
      pool.emplace_back([&, t]() {
        for (long e = t; e < E && rcs[t] == DGB_OK; e += nth) {
          rcs[t] = curved_element(m.nodes + (size_t)e * nq * 3, q, ops, &gv[(size_t)e * kVolC * NB],
                                  &gf[(size_t)e * 6 * kFaceC * NQF], e, whys[t]);
          if (rcs[t]) fails[t] = e;
        }
      });
    for (auto& th : pool) th.join();
    // the first failing element in element order, whatever the thread split
    int tf = -1;
    for (int t = 0; t < nth; ++t)
      if (rcs[t] && (tf < 0 || fails[t] < fails[tf])) tf = t;
    if (tf >= 0) {
      why = whys[tf];
      return rcs[tf];
    }
  }

  build_neighbours(m, nbr);

  // the two sides of every interior face must see the same face
  for (long e = 0; e < E; ++e)
    for (int lf = 0; lf < 6; ++lf) {
      const int en = nbr[6 * e + lf];
      if (en < 0) continue;
      if (curved) {  // point by point
        const int NQF = P * P;
        const double* g = &gf[((size_t)e * 6 + lf) * kFaceC * NQF];
        const double* h = &gf[((size_t)en * 6 + (lf ^ 1)) * kFaceC * NQF];
        for (int fq = 0; fq < NQF; ++fq) {
          if (face_mismatch(g + kFaceN * NQF + fq, h + kFaceN * NQF + fq, NQF, g[kFaceFJ * NQF + fq],
                            h[kFaceFJ * NQF + fq])) {
            char buf[160];
            snprintf(buf, sizeof buf, "face %d of element %ld does not match its neighbour %d", lf, e, en);
            why = buf;
            return DGB_ERR_GEOMETRY;
          }
        }
        continue;
      }
      const double* g = &geo[(size_t)e * kGeoStride];
      const double* h = &geo[(size_t)en * kGeoStride];
      const int lo = lf ^ 1;
      if (face_mismatch(g + kGeoN + 3 * lf, h + kGeoN + 3 * lo, 1, g[kGeoFJ + lf], h[kGeoFJ + lo])) {
        char buf[160];
        snprintf(buf, sizeof buf, "face %d of element %ld does not match its neighbour %d", lf, e, en);
        why = buf;
        return DGB_ERR_GEOMETRY;
      }
    }
  return DGB_OK;
}

void total_conditions(const dgb_params& prm, double* Tt, double* Pt)
{
  const double u = prm.Ufr[1] / prm.Ufr[0], v = prm.Ufr[2] / prm.Ufr[0], w = prm.Ufr[3] / prm.Ufr[0];
  const double M = std::sqrt(u * u + v * v + w * w) / prm.c;
  const double gm1 = prm.gamma - 1.;
  *Tt = prm.T * (1. + 0.5 * gm1 * M * M);
  *Pt = prm.P * std::pow(*Tt / prm.T, prm.gamma / gm1);
}

}  // namespace dgb
