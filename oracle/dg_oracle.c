/* CPU restatement of the reference's FP64 DG residual and RK time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests compare the
 * CUDA path against; the product never links, loads or calls it.  It is pinned
 * against the reference itself (the unmodified solver compiled in place into
 * oracle/_ref/, and the fixtures under tests/golden/ made from it).
 *
 * It restates, in plain C and dense loops (no sum factorisation, no tensor
 * shortcuts), the algorithm of:
 *   quadrature        quadrature.cpp:84-205   (Gauss-Legendre on [a,b], P=p+1 points)
 *   Lagrange basis    basis.cpp:64-170         (equispaced nodes on [0,1], [z[y[x]]] order)
 *   face mapping      basis.cpp:180-192        (surf2vol)
 *   tables            basis.cpp:351-407        (veval / vgrad / feval / fgrad)
 *   geometry          geometry_common.cpp:264-395 (Jacobian, detJ, Minv by Gauss-Jordan,
 *                                                   physical gradients)
 *   surface geometry  geometry_common.cpp:397-454 (normal, surface Jacobian)
 *   face list         geometry_shared.cpp:156-267 (each face once, periodic wrap)
 *   physics           flux.cpp:24-202, bound_states.cpp:24-130
 *   residual          solve.cpp:150-807 (volume, source, interior faces with BR2
 *                                        lifting and dual consistency, boundary faces,
 *                                        f = -Minv R)
 *   RK4 / TVD-RK3     time_distributed.cpp:46-102, residual norm :23-44
 *   dense math        dgmath.cpp:71-91 (det/inverse 3x3), 143-161 (packed symmetric
 *                                        mat-vec), 311-371 (Gauss-Jordan inverse)
 *
 * The one structural difference from solve.cpp is the periodic face: the
 * reference's single-rank run visits it twice through self-messages, adding
 * only the left side each time (solve.cpp:191,530,607); here it is visited
 * once and both sides are added, which is the same sum up to rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PI_ 3.14159265358979323846

enum { BT_PERIODIC = -2, BT_FREESTREAM = -3, BT_INVISCID_WALL = -4,
       BT_SUBSONIC_INFLOW = -5, BT_SUBSONIC_OUTFLOW = -6, BT_NO_SLIP_WALL = -7 };

/* ---------------------------------------------------------------- quadrature */

/* n-point Gauss-Legendre rule on [a,b] by Newton iteration on P_n with the
 * three-term recurrence (quadrature.cpp:84-173). */
void oracle_gauss_legendre(int n, double a, double b, double* x, double* w)
{
  if (n == 1) { x[0] = 0.5 * (a + b); w[0] = b - a; return; }
  for (int i = 0; i < n; ++i) {
    double z = cos(PI_ * (i + 0.75) / (n + 0.5));
    double dp = 0.;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1., p1 = z;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2. * k - 1.) * z * p1 - (k - 1.) * p0) / k;
        p0 = p1; p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.);
      double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    {
      double p0 = 1., p1 = z;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2. * k - 1.) * z * p1 - (k - 1.) * p0) / k;
        p0 = p1; p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.);
    }
    /* ascending order on [a,b] */
    int j = n - 1 - i;
    x[j] = a + (b - a) * (z + 1.) / 2.;
    w[j] = (b - a) / ((1. - z * z) * dp * dp);
  }
}

/* -------------------------------------------------------------------- basis */

/* basis.cpp:91-104 */
double oracle_lagrange1d(int i, int p, double x)
{
  if (p == 0) return 1.;
  double xi = (double)i / p, v = 1.;
  for (int j = 0; j <= p; ++j)
    if (j != i) v *= (x - (double)j / p) / (xi - (double)j / p);
  return v;
}

/* basis.cpp:125-148 */
double oracle_lagrange1d_deriv(int i, int p, double x)
{
  if (p == 0) return 0.;
  double xi = (double)i / p, s = 0.;
  for (int j = 0; j <= p; ++j) {
    if (j == i) continue;
    double m = 1., xj = (double)j / p;
    for (int k = 0; k <= p; ++k)
      if (k != i && k != j) m *= (x - (double)k / p) / (xi - (double)k / p);
    s += m / (xi - xj);
  }
  return s;
}

static void surf2vol(int face, double s, double t, double* r)
{
  switch (face) {
    case 0: r[0] = 0.; r[1] = s; r[2] = t; break;
    case 1: r[0] = 1.; r[1] = s; r[2] = t; break;
    case 2: r[0] = t; r[1] = 0.; r[2] = s; break;
    case 3: r[0] = t; r[1] = 1.; r[2] = s; break;
    case 4: r[0] = s; r[1] = t; r[2] = 0.; break;
    default: r[0] = s; r[1] = t; r[2] = 1.; break;
  }
}

static void lag3(int bf, int p, const double* r, double* val, double* grad)
{
  int P = p + 1, ix = bf % P, iy = (bf / P) % P, iz = bf / (P * P);
  double lx = oracle_lagrange1d(ix, p, r[0]), ly = oracle_lagrange1d(iy, p, r[1]),
         lz = oracle_lagrange1d(iz, p, r[2]);
  if (val) *val = lx * ly * lz;
  if (grad) {
    grad[0] = oracle_lagrange1d_deriv(ix, p, r[0]) * ly * lz;
    grad[1] = lx * oracle_lagrange1d_deriv(iy, p, r[1]) * lz;
    grad[2] = lx * ly * oracle_lagrange1d_deriv(iz, p, r[2]);
  }
}

/* --------------------------------------------------------------- dense math */

double oracle_det3(const double* m)
{
  return m[0] * m[4] * m[8] + m[1] * m[5] * m[6] + m[2] * m[3] * m[7] -
         m[2] * m[4] * m[6] - m[1] * m[3] * m[8] - m[0] * m[5] * m[7];
}

void oracle_inv3(const double* m, double* o)
{
  double id = 1. / oracle_det3(m);
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

/* in-place inverse of a row-major n x n matrix by Gauss-Jordan elimination
 * with partial pivoting; returns nonzero if a pivot vanishes */
int oracle_invert(int n, double* A)
{
  double* a = (double*)malloc(sizeof(double) * 2 * n * n);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) {
      a[2 * n * r + c] = A[n * r + c];
      a[2 * n * r + n + c] = (r == c) ? 1. : 0.;
    }
  for (int k = 0; k < n; ++k) {
    int piv = k;
    for (int r = k + 1; r < n; ++r)
      if (fabs(a[2 * n * r + k]) > fabs(a[2 * n * piv + k])) piv = r;
    if (a[2 * n * piv + k] == 0.) { free(a); return 1; }
    if (piv != k)
      for (int c = 0; c < 2 * n; ++c) {
        double t = a[2 * n * k + c];
        a[2 * n * k + c] = a[2 * n * piv + c];
        a[2 * n * piv + c] = t;
      }
    double d = a[2 * n * k + k];
    for (int c = 0; c < 2 * n; ++c) a[2 * n * k + c] /= d;
    for (int r = 0; r < n; ++r) {
      if (r == k) continue;
      double f = a[2 * n * r + k];
      if (f == 0.) continue;
      for (int c = 0; c < 2 * n; ++c) a[2 * n * r + c] -= f * a[2 * n * k + c];
    }
  }
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) A[n * r + c] = a[2 * n * r + n + c];
  free(a);
  return 0;
}

/* r = c * M v with M symmetric stored as packed upper triangle, row major
 * (dgmath.cpp:143-161) */
void oracle_symm_packed_mv(int n, const double* M, const double* v, double c, double* r)
{
  int k = 0;
  for (int i = 0; i < n; ++i) r[i] = 0.;
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j, ++k) {
      r[i] += c * M[k] * v[j];
      if (j != i) r[j] += c * M[k] * v[i];
    }
}

/* ------------------------------------------------------------------ physics */

/* flux.cpp:24-48 */
void oracle_analytical_flux(const double* U, double g, double* F)
{
  double r = U[0], u = U[1] / r, v = U[2] / r, w = U[3] / r;
  double p = (g - 1.) * (U[4] - 0.5 * r * (u * u + v * v + w * w));
  double H = (U[4] + p) / r;
  double* Fx = F; double* Fy = F + 5; double* Fz = F + 10;
  Fx[0] = r * u; Fx[1] = r * u * u + p; Fx[2] = r * u * v; Fx[3] = r * u * w; Fx[4] = r * u * H;
  Fy[0] = r * v; Fy[1] = r * u * v; Fy[2] = r * v * v + p; Fy[3] = r * v * w; Fy[4] = r * v * H;
  Fz[0] = r * w; Fz[1] = r * u * w; Fz[2] = r * v * w; Fz[3] = r * w * w + p; Fz[4] = r * w * H;
}

/* Roe flux with the 5%-of-sound-speed entropy fix (flux.cpp:56-154) */
void oracle_roe(const double* Ul, const double* Ur, const double* n, double g,
                double* f, double* smax)
{
  double gm1 = g - 1.;
  double rl = Ul[0], ul = Ul[1] / rl, vl = Ul[2] / rl, wl = Ul[3] / rl;
  double pl = gm1 * (Ul[4] - 0.5 * rl * (ul * ul + vl * vl + wl * wl));
  double Hl = Ul[4] / rl + pl / rl;
  double rr = Ur[0], ur = Ur[1] / rr, vr = Ur[2] / rr, wr = Ur[3] / rr;
  double pr = gm1 * (Ur[4] - 0.5 * rr * (ur * ur + vr * vr + wr * wr));
  double Hr = Ur[4] / rr + pr / rr;
  double sl = sqrt(rl), sr = sqrt(rr), den = sl + sr;
  double u = (sl * ul + sr * ur) / den, v = (sl * vl + sr * vr) / den,
         w = (sl * wl + sr * wr) / den, H = (sl * Hl + sr * Hr) / den;
  double dr = rr - rl, dxm = Ur[1] - Ul[1], dym = Ur[2] - Ul[2], dzm = Ur[3] - Ul[3],
         drE = Ur[4] - Ul[4];
  double q2 = u * u + v * v + w * w;
  double c = sqrt(gm1 * (H - 0.5 * q2));
  double un = u * n[0] + v * n[1] + w * n[2];
  double l1 = un + c, l2 = un - c, l3 = un;
  double a1 = fabs(l1), a2 = fabs(l2), a3 = fabs(l3), eps = 0.05 * c;
  if (a1 < eps) a1 = fabs((eps * eps + l1 * l1) / (2. * eps));
  if (a2 < eps) a2 = fabs((eps * eps + l2 * l2) / (2. * eps));
  if (a3 < eps) a3 = fabs((eps * eps + l3 * l3) / (2. * eps));
  double s1 = 0.5 * (a1 + a2), s2 = 0.5 * (a1 - a2);
  double G1 = gm1 * (0.5 * q2 * dr - (u * dxm + v * dym + w * dzm) + drE);
  double G2 = -un * dr + (dxm * n[0] + dym * n[1] + dzm * n[2]);
  double C1 = (G1 / (c * c)) * (s1 - a3) + (G2 / c) * s2;
  double C2 = (G1 / c) * s2 + (s1 - a3) * G2;
  double unl = ul * n[0] + vl * n[1] + wl * n[2], unr = ur * n[0] + vr * n[1] + wr * n[2];
  f[0] = 0.5 * (rl * unl + rr * unr) - 0.5 * (a3 * dr + C1);
  f[1] = 0.5 * (rl * ul * unl + pl * n[0] + rr * ur * unr + pr * n[0]) - 0.5 * (a3 * dxm + C1 * u + C2 * n[0]);
  f[2] = 0.5 * (rl * vl * unl + pl * n[1] + rr * vr * unr + pr * n[1]) - 0.5 * (a3 * dym + C1 * v + C2 * n[1]);
  f[3] = 0.5 * (rl * wl * unl + pl * n[2] + rr * wr * unr + pr * n[2]) - 0.5 * (a3 * dzm + C1 * w + C2 * n[2]);
  f[4] = 0.5 * (rl * Hl * unl + rr * Hr * unr) - 0.5 * (a3 * drE + C1 * H + C2 * un);
  if (smax) { double m = a1 > a2 ? a1 : a2; *smax = m > a3 ? m : a3; }
}

/* viscous (Stokes, no heat flux) flux A(s, grad s) (flux.cpp:156-202);
 * Q = [Qx(5) Qy(5) Qz(5)] */
void oracle_A(const double* s, const double* sx, const double* sy, const double* sz,
              double mu, double* Q)
{
  double lam = -(2. / 3.) * mu;
  double r = s[0], u = s[1] / r, v = s[2] / r, w = s[3] / r;
  double ux = (sx[1] - sx[0] * u) / r, uy = (sy[1] - sy[0] * u) / r, uz = (sz[1] - sz[0] * u) / r;
  double vx = (sx[2] - sx[0] * v) / r, vy = (sy[2] - sy[0] * v) / r, vz = (sz[2] - sz[0] * v) / r;
  double wx = (sx[3] - sx[0] * w) / r, wy = (sy[3] - sy[0] * w) / r, wz = (sz[3] - sz[0] * w) / r;
  double dv = ux + vy + wz;
  double txx = lam * dv + 2. * mu * ux, tyy = lam * dv + 2. * mu * vy, tzz = lam * dv + 2. * mu * wz;
  double txy = mu * (vx + uy), txz = mu * (uz + wx), tyz = mu * (wy + vz);
  double* Qx = Q; double* Qy = Q + 5; double* Qz = Q + 10;
  Qx[0] = 0.; Qx[1] = txx; Qx[2] = txy; Qx[3] = txz; Qx[4] = u * txx + v * txy + w * txz;
  Qy[0] = 0.; Qy[1] = txy; Qy[2] = tyy; Qy[3] = tyz; Qy[4] = u * txy + v * tyy + w * tyz;
  Qz[0] = 0.; Qz[1] = txz; Qz[2] = tyz; Qz[3] = tzz; Qz[4] = u * txz + v * tyz + w * tzz;
}

/* boundary ghost states (bound_states.cpp:24-130); returns nonzero when the
 * subsonic inflow Mach number has no non-negative root */
int oracle_bc_state(int bt, const double* UL, const double* n, double gamma, double R,
                    double Pt, double Tt, double P, const double* Ufr, double* Ub)
{
  double gm1 = gamma - 1.;
  double u = UL[1] / UL[0], v = UL[2] / UL[0], w = UL[3] / UL[0];
  if (bt == BT_FREESTREAM) { for (int i = 0; i < 5; ++i) Ub[i] = Ufr[i]; return 0; }
  if (bt == BT_INVISCID_WALL) {
    double vn = u * n[0] + v * n[1] + w * n[2];
    Ub[0] = UL[0]; Ub[1] = UL[0] * (u - vn * n[0]); Ub[2] = UL[0] * (v - vn * n[1]);
    Ub[3] = UL[0] * (w - vn * n[2]); Ub[4] = UL[4];
    return 0;
  }
  if (bt == BT_NO_SLIP_WALL) {
    Ub[0] = UL[0]; Ub[1] = 0.; Ub[2] = 0.; Ub[3] = 0.; Ub[4] = UL[4];
    return 0;
  }
  double q2 = u * u + v * v + w * w, pp = gm1 * (UL[4] - 0.5 * UL[0] * q2);
  double unp = u * n[0] + v * n[1] + w * n[2];
  double cp = sqrt(gamma * pp / UL[0]), Jp = unp + 2. * cp / gm1;
  if (bt == BT_SUBSONIC_INFLOW) {
    double a = gamma * R * Tt - 0.5 * gm1 * Jp * Jp;
    double b = -4. * gamma * R * Tt / gm1;
    double c = 4. * gamma * R * Tt / (gm1 * gm1) - Jp * Jp;
    double s0 = (-b + sqrt(b * b - 4. * a * c)) / (2. * a);
    double s1 = (-b - sqrt(b * b - 4. * a * c)) / (2. * a);
    double Mb = 0.;
    int bad = 0;
    if (s0 >= 0. && s1 >= 0.) Mb = s0 < s1 ? s0 : s1;
    else if (s0 >= 0.) Mb = s0;
    else if (s1 >= 0.) Mb = s1;
    else bad = 1;
    double Tb = Tt / (1. + 0.5 * gm1 * Mb * Mb);
    double Pb = Pt * pow(Tb / Tt, gamma / gm1);
    double rb = Pb / (R * Tb), cb = sqrt(gamma * Pb / rb);
    double ub = -Mb * cb * n[0], vb = -Mb * cb * n[1], wb = -Mb * cb * n[2];
    Ub[0] = rb; Ub[1] = rb * ub; Ub[2] = rb * vb; Ub[3] = rb * wb;
    Ub[4] = Pb / gm1 + 0.5 * rb * (ub * ub + vb * vb + wb * wb);
    return bad;
  }
  if (bt == BT_SUBSONIC_OUTFLOW) {
    double Sp = pp / pow(UL[0], gamma);
    double rb = pow(P / Sp, 1. / gamma), cb = sqrt(gamma * P / rb);
    double unb = Jp - 2. * cb / gm1;
    double ub = u - unp * n[0] + unb * n[0], vb = v - unp * n[1] + unb * n[1],
           wb = w - unp * n[2] + unb * n[2];
    Ub[0] = rb; Ub[1] = rb * ub; Ub[2] = rb * vb; Ub[3] = rb * wb;
    Ub[4] = P / gm1 + 0.5 * rb * (ub * ub + vb * vb + wb * wb);
    return 0;
  }
  return 2;
}

/* ------------------------------------------------------------ discretisation */

typedef struct {
  int nx, ny, nz, p, q, P, nb, nqv, nqf, E;
  long long bounds[6];
  const double* nodes;
  /* reference tables */
  double *vw, *fw, *veval, *vgr, *feval, *fgr;
  /* per element */
  double *vJ, *vgrad, *fgrad, *Minv;
  /* faces: [eL, eR(>=0) or btype(<0), lfL, lfR] */
  int nf;
  long long* faces;
  double *fn, *fJ;
} disc;

static void jac(const disc* d, int e, const double* r, double* J)
{
  int Q = d->q + 1, nq = Q * Q * Q;
  for (int i = 0; i < 9; ++i) J[i] = 0.;
  for (int n = 0; n < nq; ++n) {
    double g[3];
    lag3(n, d->q, r, NULL, g);
    const double* x = d->nodes + 3 * ((long)nq * e + n);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) J[3 * a + b] += x[a] * g[b];
  }
}

static void ref2glo(const disc* d, int e, const double* r, double* X)
{
  int Q = d->q + 1, nq = Q * Q * Q;
  X[0] = X[1] = X[2] = 0.;
  for (int n = 0; n < nq; ++n) {
    double v;
    lag3(n, d->q, r, &v, NULL);
    const double* x = d->nodes + 3 * ((long)nq * e + n);
    X[0] += x[0] * v; X[1] += x[1] * v; X[2] += x[2] * v;
  }
}

/* geometry_common.cpp:416-454: tangents from the 2D Lagrange interpolant of the
 * face's geometry nodes; normal flipped on low-side faces so it is outward of
 * the element that owns the face */
static void surface(const disc* d, int e, int lf, double s, double t, double* n, double* fJ)
{
  int Q = d->q + 1;
  double ds[3] = {0, 0, 0}, dt[3] = {0, 0, 0};
  for (int b = 0; b < Q * Q; ++b) {
    int bx = b % Q, by = b / Q;
    double ns = d->q == 0 ? 0. : (double)bx / d->q, nt = d->q == 0 ? 0. : (double)by / d->q;
    double r[3], X[3];
    surf2vol(lf, ns, nt, r);
    ref2glo(d, e, r, X);
    double gs = oracle_lagrange1d_deriv(bx, d->q, s) * oracle_lagrange1d(by, d->q, t);
    double gt = oracle_lagrange1d(bx, d->q, s) * oracle_lagrange1d_deriv(by, d->q, t);
    for (int a = 0; a < 3; ++a) { ds[a] += X[a] * gs; dt[a] += X[a] * gt; }
  }
  n[0] = ds[1] * dt[2] - ds[2] * dt[1];
  n[1] = ds[2] * dt[0] - ds[0] * dt[2];
  n[2] = ds[0] * dt[1] - ds[1] * dt[0];
  *fJ = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  for (int a = 0; a < 3; ++a) n[a] /= *fJ;
  if (lf == 0 || lf == 2 || lf == 4)
    for (int a = 0; a < 3; ++a) n[a] = -n[a];
}

static int build(disc* d, int nx, int ny, int nz, int p, int q, const double* nodes,
                 const long long* bounds)
{
  memset(d, 0, sizeof(*d));
  d->nx = nx; d->ny = ny; d->nz = nz; d->p = p; d->q = q; d->P = p + 1;
  d->nb = d->P * d->P * d->P; d->nqv = d->nb; d->nqf = d->P * d->P;
  d->E = nx * ny * nz; d->nodes = nodes;
  for (int i = 0; i < 6; ++i) d->bounds[i] = bounds[i];
  int P = d->P, nb = d->nb, nqv = d->nqv, nqf = d->nqf, E = d->E;
  double* x1 = (double*)malloc(sizeof(double) * P);
  double* w1 = (double*)malloc(sizeof(double) * P);
  oracle_gauss_legendre(P, 0., 1., x1, w1);
  d->vw = (double*)malloc(sizeof(double) * nqv);
  d->fw = (double*)malloc(sizeof(double) * nqf);
  d->veval = (double*)malloc(sizeof(double) * nqv * nb);
  d->vgr = (double*)malloc(sizeof(double) * nqv * nb * 3);
  d->feval = (double*)malloc(sizeof(double) * 6 * nqf * nb);
  d->fgr = (double*)malloc(sizeof(double) * 6 * nqf * nb * 3);
  for (int k = 0; k < P; ++k)
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i) {
        int qi = i + P * (j + P * k);
        double r[3] = {x1[i], x1[j], x1[k]};
        d->vw[qi] = w1[i] * w1[j] * w1[k];
        for (int b = 0; b < nb; ++b)
          lag3(b, p, r, &d->veval[(long)nb * qi + b], &d->vgr[3 * ((long)nb * qi + b)]);
      }
  for (int j = 0; j < P; ++j)
    for (int i = 0; i < P; ++i) d->fw[i + P * j] = w1[i] * w1[j];
  for (int lf = 0; lf < 6; ++lf)
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i) {
        int qi = i + P * j;
        double r[3];
        surf2vol(lf, x1[i], x1[j], r);
        for (int b = 0; b < nb; ++b)
          lag3(b, p, r, &d->feval[(long)nb * (nqf * lf + qi) + b],
               &d->fgr[3 * ((long)nb * (nqf * lf + qi) + b)]);
      }

  /* per element: detJ, physical gradients, inverse mass matrix */
  d->vJ = (double*)malloc(sizeof(double) * (long)E * nqv);
  d->vgrad = (double*)malloc(sizeof(double) * (long)E * nqv * nb * 3);
  d->fgrad = (double*)malloc(sizeof(double) * (long)E * 6 * nqf * nb * 3);
  d->Minv = (double*)malloc(sizeof(double) * (long)E * nb * nb);
  int err = 0;
  for (int e = 0; e < E; ++e) {
    for (int qi = 0; qi < nqv; ++qi) {
      int i = qi % P, j = (qi / P) % P, k = qi / (P * P);
      double r[3] = {x1[i], x1[j], x1[k]}, J[9], Ji[9];
      jac(d, e, r, J);
      d->vJ[(long)nqv * e + qi] = oracle_det3(J);
      oracle_inv3(J, Ji);
      for (int b = 0; b < nb; ++b) {
        const double* g = &d->vgr[3 * ((long)nb * qi + b)];
        double* o = &d->vgrad[3 * ((long)nb * ((long)nqv * e + qi) + b)];
        for (int c = 0; c < 3; ++c) o[c] = g[0] * Ji[c] + g[1] * Ji[3 + c] + g[2] * Ji[6 + c];
      }
    }
    for (int lf = 0; lf < 6; ++lf)
      for (int qi = 0; qi < nqf; ++qi) {
        int i = qi % P, j = qi / P;
        double r[3], J[9], Ji[9];
        surf2vol(lf, x1[i], x1[j], r);
        jac(d, e, r, J);
        oracle_inv3(J, Ji);
        for (int b = 0; b < nb; ++b) {
          const double* g = &d->fgr[3 * ((long)nb * (nqf * lf + qi) + b)];
          double* o = &d->fgrad[3 * ((long)nb * ((long)nqf * (6L * e + lf) + qi) + b)];
          for (int c = 0; c < 3; ++c) o[c] = g[0] * Ji[c] + g[1] * Ji[3 + c] + g[2] * Ji[6 + c];
        }
      }
    double* M = d->Minv + (long)nb * nb * e;
    for (int t = 0; t < nb; ++t)
      for (int b = t; b < nb; ++b) {
        double s = 0.;
        for (int qi = 0; qi < nqv; ++qi)
          s += d->vJ[(long)nqv * e + qi] * d->vw[qi] * d->veval[(long)nb * qi + t] *
               d->veval[(long)nb * qi + b];
        M[nb * t + b] = s;
        M[nb * b + t] = s;
      }
    if (oracle_invert(nb, M)) err = 1;
  }

  /* faces, enumerated like geometry_shared.cpp:156-267 */
  long maxf = 3L * E + (long)nx * ny + (long)ny * nz + (long)nz * nx;
  d->faces = (long long*)malloc(sizeof(long long) * 4 * maxf);
  d->fn = (double*)malloc(sizeof(double) * 3 * nqf * maxf);
  d->fJ = (double*)malloc(sizeof(double) * nqf * maxf);
  int nf = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int e = i + nx * (j + ny * k);
        int list[6], nl = 0;
        list[nl++] = 1; list[nl++] = 3; list[nl++] = 5;
        if (i == 0) list[nl++] = 0;
        if (j == 0) list[nl++] = 2;
        if (k == 0) list[nl++] = 4;
        for (int li = 0; li < nl; ++li) {
          int lf = list[li];
          if (bounds[1] == BT_PERIODIC && i == nx - 1 && lf == 1) continue;
          if (bounds[3] == BT_PERIODIC && j == ny - 1 && lf == 3) continue;
          if (bounds[5] == BT_PERIODIC && k == nz - 1 && lf == 5) continue;
          int di[6] = {-1, 1, 0, 0, 0, 0}, dj[6] = {0, 0, -1, 1, 0, 0}, dk[6] = {0, 0, 0, 0, -1, 1};
          int ia = i + di[lf], ja = j + dj[lf], ka = k + dk[lf];
          int out = (ia < 0) ? 0 : (ia >= nx) ? 1 : (ja < 0) ? 2 : (ja >= ny) ? 3
                  : (ka < 0) ? 4 : (ka >= nz) ? 5 : -1;
          long long* F = d->faces + 4L * nf;
          F[0] = e; F[2] = lf; F[3] = lf ^ 1;
          if (out < 0 || bounds[out] == BT_PERIODIC)
            F[1] = ((ia + nx) % nx) + nx * (((ja + ny) % ny) + ny * ((ka + nz) % nz));
          else
            F[1] = bounds[out];
          for (int qi = 0; qi < nqf; ++qi)
            surface(d, e, lf, x1[qi % P], x1[qi / P], &d->fn[3 * ((long)nqf * nf + qi)],
                    &d->fJ[(long)nqf * nf + qi]);
          ++nf;
        }
      }
  d->nf = nf;
  free(x1); free(w1);
  return err;
}

static void release(disc* d)
{
  free(d->vw); free(d->fw); free(d->veval); free(d->vgr); free(d->feval); free(d->fgr);
  free(d->vJ); free(d->vgrad); free(d->fgrad); free(d->Minv);
  free(d->faces); free(d->fn); free(d->fJ);
}

typedef struct {
  double gamma, R, mu, c, T, P, Ufr[5], src[5], eta;
} prm;

static prm unpack(const double* a)
{
  prm p;
  p.gamma = a[0]; p.R = a[1]; p.mu = a[2]; p.c = a[3]; p.T = a[4]; p.P = a[5];
  for (int i = 0; i < 5; ++i) { p.Ufr[i] = a[6 + i]; p.src[i] = a[11 + i]; }
  p.eta = a[16];
  return p;
}

#define UIX(e, r, b) ((long)nb * (5L * (e) + (r)) + (b))

/* face trace of value and physical gradient of U on element e at local face lf */
static void trace(const disc* d, const double* U, int e, int lf, int qi, double* S, double* G)
{
  int nb = d->nb, nqf = d->nqf;
  for (int r = 0; r < 5; ++r) { S[r] = 0.; G[r] = G[5 + r] = G[10 + r] = 0.; }
  for (int b = 0; b < nb; ++b) {
    double ph = d->feval[(long)nb * (nqf * lf + qi) + b];
    const double* g = &d->fgrad[3 * ((long)nb * ((long)nqf * (6L * e + lf) + qi) + b)];
    for (int r = 0; r < 5; ++r) {
      double u = U[UIX(e, r, b)];
      S[r] += u * ph;
      G[r] += u * g[0]; G[5 + r] += u * g[1]; G[10 + r] += u * g[2];
    }
  }
}

/* solve.cpp:150-807 */
static int residual(const disc* d, const prm* pp, const double* U, double* R, double* f)
{
  int nb = d->nb, nqv = d->nqv, nqf = d->nqf, E = d->E;
  double gamma = pp->gamma, mu = pp->mu, eta = pp->eta;
  int bad = 0;
  memset(R, 0, sizeof(double) * (long)E * 5 * nb);

  /* boundary total conditions from the freestream (solve.cpp:167-175) */
  double M, Tt, Pt;
  {
    double u = pp->Ufr[1] / pp->Ufr[0], v = pp->Ufr[2] / pp->Ufr[0], w = pp->Ufr[3] / pp->Ufr[0];
    M = sqrt(u * u + v * v + w * w) / pp->c;
    Tt = pp->T * (1. + 0.5 * (gamma - 1.) * M * M);
    Pt = pp->P * pow(Tt / pp->T, gamma / (gamma - 1.));
  }

  /* volume (solve.cpp:276-341) and source (345-360) */
  for (int e = 0; e < E; ++e)
    for (int qi = 0; qi < nqv; ++qi) {
      double S[5] = {0}, Sx[5] = {0}, Sy[5] = {0}, Sz[5] = {0}, F[15], Q[15];
      double wJ = d->vw[qi] * d->vJ[(long)nqv * e + qi];
      for (int b = 0; b < nb; ++b) {
        double ph = d->veval[(long)nb * qi + b];
        const double* g = &d->vgrad[3 * ((long)nb * ((long)nqv * e + qi) + b)];
        for (int r = 0; r < 5; ++r) {
          double u = U[UIX(e, r, b)];
          S[r] += u * ph; Sx[r] += u * g[0]; Sy[r] += u * g[1]; Sz[r] += u * g[2];
        }
      }
      oracle_analytical_flux(S, gamma, F);
      oracle_A(S, Sx, Sy, Sz, mu, Q);
      for (int r = 0; r < 5; ++r)
        for (int t = 0; t < nb; ++t) {
          const double* g = &d->vgrad[3 * ((long)nb * ((long)nqv * e + qi) + t)];
          R[UIX(e, r, t)] += (g[0] * (Q[r] - F[r]) + g[1] * (Q[5 + r] - F[5 + r]) +
                              g[2] * (Q[10 + r] - F[10 + r])) * wJ;
          R[UIX(e, r, t)] -= d->veval[(long)nb * qi + t] * pp->src[r] * wJ;
        }
    }

  double* lift = (double*)malloc(sizeof(double) * 4 * 15 * nb);
  double *RL = lift, *RRv = lift + 15 * nb, *DL = lift + 30 * nb, *DR = lift + 45 * nb;
  double* SLs = (double*)malloc(sizeof(double) * nqf * 40);

  for (int fi = 0; fi < d->nf; ++fi) {
    const long long* F = d->faces + 4L * fi;
    int eL = (int)F[0], lfL = (int)F[2], lfR = (int)F[3];
    int interior = F[1] >= 0;
    int eR = interior ? (int)F[1] : -1;
    int bt = interior ? 0 : (int)F[1];
    const double* fn = d->fn + 3L * nqf * fi;
    const double* fJ = d->fJ + (long)nqf * fi;

    /* traces: SL(5) GL(15) SR/Ub(5) GR(15) per quad point */
    for (int qi = 0; qi < nqf; ++qi) {
      double* s = SLs + 40 * qi;
      trace(d, U, eL, lfL, qi, s, s + 5);
      if (interior) trace(d, U, eR, lfR, qi, s + 20, s + 25);
      else if (oracle_bc_state(bt, s, fn + 3 * qi, gamma, pp->R, Pt, Tt, pp->P, pp->Ufr, s + 20))
        bad = 1;
    }

    /* BR2 lifting right-hand sides (solve.cpp:409-470, 642-682) */
    memset(lift, 0, sizeof(double) * 30 * nb);
    for (int qi = 0; qi < nqf; ++qi) {
      double* s = SLs + 40 * qi;
      const double* n = fn + 3 * qi;
      double wf = fJ[qi] * d->fw[qi];
      double jx[5], jy[5], jz[5], QL[15], QR[15];
      for (int r = 0; r < 5; ++r) {
        double dj = s[r] - s[20 + r];
        jx[r] = dj * n[0]; jy[r] = dj * n[1]; jz[r] = dj * n[2];
      }
      if (interior) {
        oracle_A(s, jx, jy, jz, mu, QL);
        oracle_A(s + 20, jx, jy, jz, mu, QR);
        for (int r = 0; r < 5; ++r)
          for (int t = 0; t < nb; ++t) {
            double pL = d->feval[(long)nb * (nqf * lfL + qi) + t];
            double pR = d->feval[(long)nb * (nqf * lfR + qi) + t];
            for (int c = 0; c < 3; ++c) {
              RL[(long)nb * (5 * c + r) + t] += 0.5 * pL * QL[5 * c + r] * wf;
              RRv[(long)nb * (5 * c + r) + t] += 0.5 * pR * QR[5 * c + r] * wf;
            }
          }
      } else {
        oracle_A(s + 20, jx, jy, jz, mu, QL);
        for (int r = 0; r < 5; ++r)
          for (int t = 0; t < nb; ++t) {
            double pL = d->feval[(long)nb * (nqf * lfL + qi) + t];
            for (int c = 0; c < 3; ++c) RL[(long)nb * (5 * c + r) + t] += pL * QL[5 * c + r] * wf;
          }
      }
    }
    for (int v = 0; v < 15; ++v) {
      const double* ML = d->Minv + (long)nb * nb * eL;
      for (int a = 0; a < nb; ++a) {
        double s = 0.;
        for (int b = 0; b < nb; ++b) s += ML[(long)nb * a + b] * RL[(long)nb * v + b];
        DL[(long)nb * v + a] = s;
      }
      if (interior) {
        const double* MR = d->Minv + (long)nb * nb * eR;
        for (int a = 0; a < nb; ++a) {
          double s = 0.;
          for (int b = 0; b < nb; ++b) s += MR[(long)nb * a + b] * RRv[(long)nb * v + b];
          DR[(long)nb * v + a] = s;
        }
      }
    }

    /* face terms (solve.cpp:484-626, 693-794) */
    for (int qi = 0; qi < nqf; ++qi) {
      double* s = SLs + 40 * qi;
      const double *UL = s, *GL = s + 5, *UR = s + 20, *GR = s + 25;
      const double* n = fn + 3 * qi;
      double wf = fJ[qi] * d->fw[qi];
      double Fh[5], dcL[15], dcR[15], QH[5], QL[15], QR[15];
      if (interior) {
        oracle_roe(UL, UR, n, gamma, Fh, NULL);
      } else {
        double Fb[15];
        oracle_analytical_flux(UR, gamma, Fb);
        for (int r = 0; r < 5; ++r) Fh[r] = Fb[r] * n[0] + Fb[5 + r] * n[1] + Fb[10 + r] * n[2];
      }
      {
        double Uh[5], ax[5], ay[5], az[5];
        for (int r = 0; r < 5; ++r) Uh[r] = interior ? 0.5 * (UL[r] + UR[r]) : UR[r];
        for (int r = 0; r < 5; ++r) {
          double dl = UL[r] - Uh[r];
          ax[r] = dl * n[0]; ay[r] = dl * n[1]; az[r] = dl * n[2];
        }
        oracle_A(UL, ax, ay, az, mu, dcL);
        if (interior) {
          for (int r = 0; r < 5; ++r) {
            double dr = UR[r] - Uh[r];
            ax[r] = dr * -n[0]; ay[r] = dr * -n[1]; az[r] = dr * -n[2];
          }
          oracle_A(UR, ax, ay, az, mu, dcR);
        }
      }
      {
        double dLv[15] = {0}, dRv[15] = {0};
        for (int v = 0; v < 15; ++v)
          for (int b = 0; b < nb; ++b) {
            dLv[v] += d->feval[(long)nb * (nqf * lfL + qi) + b] * DL[(long)nb * v + b];
            if (interior) dRv[v] += d->feval[(long)nb * (nqf * lfR + qi) + b] * DR[(long)nb * v + b];
          }
        oracle_A(UL, GL, GL + 5, GL + 10, mu, QL);
        if (interior) oracle_A(UR, GR, GR + 5, GR + 10, mu, QR);
        for (int r = 0; r < 5; ++r) {
          double qh[3];
          for (int c = 0; c < 3; ++c)
            qh[c] = interior ? 0.5 * (QL[5 * c + r] + QR[5 * c + r]) - eta * 0.5 * (dLv[5 * c + r] + dRv[5 * c + r])
                             : QL[5 * c + r] - eta * dLv[5 * c + r];
          QH[r] = qh[0] * n[0] + qh[1] * n[1] + qh[2] * n[2];
        }
      }
      for (int r = 0; r < 5; ++r)
        for (int t = 0; t < nb; ++t) {
          double pL = d->feval[(long)nb * (nqf * lfL + qi) + t];
          const double* gL = &d->fgrad[3 * ((long)nb * ((long)nqf * (6L * eL + lfL) + qi) + t)];
          R[UIX(eL, r, t)] += (pL * Fh[r] - (gL[0] * dcL[r] + gL[1] * dcL[5 + r] + gL[2] * dcL[10 + r]) -
                               pL * QH[r]) * wf;
          if (interior) {
            double pR = d->feval[(long)nb * (nqf * lfR + qi) + t];
            const double* gR = &d->fgrad[3 * ((long)nb * ((long)nqf * (6L * eR + lfR) + qi) + t)];
            R[UIX(eR, r, t)] += (-(pR * Fh[r]) - (gR[0] * dcR[r] + gR[1] * dcR[5 + r] + gR[2] * dcR[10 + r]) +
                                 pR * QH[r]) * wf;
          }
        }
    }
  }
  free(lift);
  free(SLs);

  /* f = -Minv R (solve.cpp:800-804) */
  for (int e = 0; e < E; ++e) {
    const double* Mi = d->Minv + (long)nb * nb * e;
    for (int r = 0; r < 5; ++r)
      for (int a = 0; a < nb; ++a) {
        double s = 0.;
        for (int b = 0; b < nb; ++b) s += Mi[(long)nb * a + b] * R[UIX(e, r, b)];
        f[UIX(e, r, a)] = -s;
      }
  }
  return bad;
}

/* ------------------------------------------------------------------ exports */

int oracle_residual(int nx, int ny, int nz, int p, int q, const double* nodes,
                    const long long* bounds, const double* params, const double* U,
                    double* R, double* f)
{
  disc d;
  int err = build(&d, nx, ny, nz, p, q, nodes, bounds);
  prm pp = unpack(params);
  long n = (long)d.E * 5 * d.nb;
  double* Rw = R ? R : (double*)malloc(sizeof(double) * n);
  double* fw = f ? f : (double*)malloc(sizeof(double) * n);
  if (!err) err = residual(&d, &pp, U, Rw, fw);
  if (!R) free(Rw);
  if (!f) free(fw);
  release(&d);
  return err;
}

/* time_distributed.cpp:46-102; norms[t] = sqrt(sum R^2 / size) of the first
 * stage of step t (time_distributed.cpp:23-44) */
int oracle_run(int nx, int ny, int nz, int p, int q, const double* nodes,
               const long long* bounds, const double* params, int scheme, double dt,
               int nsteps, double* U, double* norms)
{
  disc d;
  int err = build(&d, nx, ny, nz, p, q, nodes, bounds);
  prm pp = unpack(params);
  long n = (long)d.E * 5 * d.nb;
  double* buf = (double*)malloc(sizeof(double) * n * 8);
  double *R = buf, *U1 = buf + n, *U2 = buf + 2 * n, *U3 = buf + 3 * n, *f1 = buf + 4 * n,
         *f2 = buf + 5 * n, *f3 = buf + 6 * n, *f4 = buf + 7 * n;
  for (int t = 0; t < nsteps && !err; ++t) {
    err |= residual(&d, &pp, U, R, f1);
    if (norms) {
      double s = 0.;
      for (long i = 0; i < n; ++i) s += R[i] * R[i];
      norms[t] = sqrt(s / (double)n);
    }
    if (scheme == 0) {
      for (long i = 0; i < n; ++i) U1[i] = U[i] + dt * f1[i] * 0.5;
      err |= residual(&d, &pp, U1, R, f2);
      for (long i = 0; i < n; ++i) U2[i] = U[i] + dt * f2[i] * 0.5;
      err |= residual(&d, &pp, U2, R, f3);
      for (long i = 0; i < n; ++i) U3[i] = U[i] + dt * f3[i];
      err |= residual(&d, &pp, U3, R, f4);
      for (long i = 0; i < n; ++i)
        U[i] = U[i] + (1. / 6.) * (f1[i] + 2. * f2[i] + 2. * f3[i] + f4[i]) * dt;
    } else {
      for (long i = 0; i < n; ++i) U1[i] = U[i] + dt * f1[i];
      err |= residual(&d, &pp, U1, R, f2);
      for (long i = 0; i < n; ++i) U2[i] = 0.75 * U[i] + 0.25 * U1[i] + 0.25 * dt * f2[i];
      err |= residual(&d, &pp, U2, R, f3);
      for (long i = 0; i < n; ++i) U[i] = (1. / 3.) * U[i] + (2. / 3.) * U2[i] + (2. / 3.) * dt * f3[i];
    }
  }
  free(buf);
  release(&d);
  return err;
}

/* geometry products for known-answer checks: detJ at volume points [E][nqv],
 * dense Minv [E][nb][nb]; returns the number of faces */
int oracle_geometry(int nx, int ny, int nz, int p, int q, const double* nodes,
                    const long long* bounds, double* vJ, double* Minv, double* fJ,
                    double* fn, long long* faces)
{
  disc d;
  build(&d, nx, ny, nz, p, q, nodes, bounds);
  if (vJ) memcpy(vJ, d.vJ, sizeof(double) * (long)d.E * d.nqv);
  if (Minv) memcpy(Minv, d.Minv, sizeof(double) * (long)d.E * d.nb * d.nb);
  if (fJ) memcpy(fJ, d.fJ, sizeof(double) * (long)d.nf * d.nqf);
  if (fn) memcpy(fn, d.fn, sizeof(double) * 3L * d.nf * d.nqf);
  if (faces) memcpy(faces, d.faces, sizeof(long long) * 4L * d.nf);
  int nf = d.nf;
  release(&d);
  return nf;
}

/* box mesh nodes like generate_bump_nodes with no bump and no stretching
 * (geometry_common.cpp:494-552): element (i,j,k) spans [i,i+1]*l/n, nodes
 * equispaced, [z[y[x]]] order */
void oracle_box_nodes(int nx, int ny, int nz, int q, double lx, double ly, double lz,
                      double* nodes)
{
  int Q = q + 1;
  double ex = lx / nx, ey = ly / ny, ez = lz / nz;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        long e = i + nx * (j + (long)ny * k);
        for (int c = 0; c < Q; ++c)
          for (int b = 0; b < Q; ++b)
            for (int a = 0; a < Q; ++a) {
              double* x = nodes + 3 * (Q * Q * Q * e + a + Q * (b + Q * c));
              x[0] = i * ex + (q ? ex / q * a : 0.);
              x[1] = j * ey + (q ? ey / q * b : 0.);
              x[2] = k * ez + (q ? ez / q * c : 0.);
            }
      }
}
