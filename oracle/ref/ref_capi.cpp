/* C entry points into the UNMODIFIED reference FP64 CPU solver, compiled in
 * place from the reference tree (include path set by oracle/Makefile) with the
 * single-rank MPI stand-in in oracle/ref/mpi.h.
 *
 * Test infrastructure only: the parity tests and fixture generator call these
 * to pin the C restatement (oracle/dg_oracle.c) and the CUDA path against the
 * reference's own arithmetic.  Nothing here is part of the product.
 *
 * Every function builds the reference's own objects and calls the reference's
 * own routines:
 *   geometry : distributed_geometry ctor + precompute  (geometry_distributed.cpp:504,386)
 *   residual : residual()                               (solve.cpp:150)
 *   stepping : RK4_distributed / tvdRK3_distributed     (time_distributed.cpp:46,79)
 *   physics  : roe, A, analytical_flux, *_state         (flux.cpp:24-202, bound_states.cpp:24-130)
 *   basis    : basis ctor, gauss_legendre_1d            (basis.cpp:415, quadrature.cpp:187)
 */
#include "io_distributed.cpp"
#include "solver_init.cpp"
#include "time_distributed.cpp"

#include <cstdio>
#include <unistd.h>
#include <fcntl.h>

namespace {

/* params layout shared with the Python side:
 *   [0] gamma [1] R [2] mu [3] c [4] T [5] P [6..10] Ufr [11..15] source [16] eta */
parameters unpack_params(const double* pr)
{
  parameters sp;
  sp.gamma = pr[0];
  sp.R     = pr[1];
  sp.mu    = pr[2];
  sp.c     = pr[3];
  sp.T     = pr[4];
  sp.P     = pr[5];
  for (int i = 0; i < 5; ++i) sp.Ufr[i] = pr[6 + i];
  for (int i = 0; i < 5; ++i) sp.source[i] = pr[11 + i];
  sp.eta = pr[16];
  return sp;
}

distributed_geometry make_geom(int nx, int ny, int nz, int p, int q,
                               const double* nodes, const long long* bounds)
{
  btype b[6];
  for (int i = 0; i < 6; ++i) b[i] = (btype)bounds[i];
  distributed_geometry geom(p, q, nx, ny, nz, b, MPI_COMM_WORLD, 1, 1, 1, 1);
  for (u64 i = 0; i < geom.core.node_size(); ++i) geom.core.node_[i] = nodes[i];
  geom.precompute();
  return geom;
}

/* the reference prints "tstep : norm" on stdout every step
 * (time_distributed.cpp:40); capture those lines into a temporary file */
struct capture_stdout
{
  int saved;
  FILE* tmp;
  capture_stdout()
  {
    fflush(stdout);
    saved = dup(1);
    tmp   = tmpfile();
    dup2(fileno(tmp), 1);
  }
  ~capture_stdout()
  {
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    fclose(tmp);
  }
  int read_norms(double* out, int n)
  {
    fflush(stdout);
    rewind(tmp);
    unsigned long long t;
    double v;
    int k = 0;
    while (k < n && fscanf(tmp, "%llu : %lf", &t, &v) == 2) out[k++] = v;
    return k;
  }
};

}  // namespace

extern "C" {

/* make_reference_state (solver_params.cpp:40) from the raw inputs */
void ref_make_reference_state(double gamma, double gcnst, double mu, double c,
                              double rho, double u, double v, double w,
                              double eta, const double* source, double* out)
{
  solver_inputs in;
  in.gamma = gamma;
  in.gcnst = gcnst;
  in.mu    = mu;
  in.c     = c;
  in.rho   = rho;
  in.u     = u;
  in.v     = v;
  in.w     = w;
  in.eta   = eta;
  for (int i = 0; i < 5; ++i) in.source[i] = source[i];
  parameters sp = make_reference_state(in);
  out[0] = sp.gamma;
  out[1] = sp.R;
  out[2] = sp.mu;
  out[3] = sp.c;
  out[4] = sp.T;
  out[5] = sp.P;
  for (int i = 0; i < 5; ++i) out[6 + i] = sp.Ufr[i];
  for (int i = 0; i < 5; ++i) out[11 + i] = sp.source[i];
  out[16] = sp.eta;
}

/* box nodes from the reference's own generator (generate_bump_nodes,
 * geometry_common.cpp:494) for a non-distributed core geometry */
void ref_bump_nodes(int nx, int ny, int nz, int p, int q, double lx, double ly,
                    double lz, double a, double bh, double bc, double bv,
                    double* nodes)
{
  s64 b[6] = {-2, -2, -2, -2, -2, -2};
  core_geometry core(p, q, nx, ny, nz, b);
  generate_bump_nodes(lx / nx, ly / ny, lz / nz, ly, ny, a, bh, bc, bv, 0, 0, 0,
                      core);
  for (u64 i = 0; i < core.node_size(); ++i) nodes[i] = core.node_[i];
}

/* one residual evaluation: R (un-inverted residual) and f = -Minv R */
int ref_residual(int nx, int ny, int nz, int p, int q, const double* nodes,
                 const long long* bounds, const double* params,
                 const double* U, double* R_out, double* f_out)
{
  distributed_geometry geom = make_geom(nx, ny, nz, p, q, nodes, bounds);
  parameters sp             = unpack_params(params);
  simstate S(geom.core), R(geom.core), f(geom.core);
  for (u64 i = 0; i < S.size(); ++i) S[i] = U[i];
  residual_workspace wsp(geom);
  residual(S, geom, sp, wsp, R, f);
  for (u64 i = 0; i < S.size(); ++i)
  {
    if (R_out) R_out[i] = R[i];
    if (f_out) f_out[i] = f[i];
  }
  geom.free_dtypes();
  return 0;
}

/* nsteps of RK4 (scheme 0) or TVD-RK3 (scheme 1); norms_out[nsteps] gets the
 * residual norm the reference prints at the first stage of each step
 * (time_distributed.cpp:23-44) */
int ref_run(int nx, int ny, int nz, int p, int q, const double* nodes,
            const long long* bounds, const double* params, int scheme,
            double dt, int nsteps, double* U, double* norms_out)
{
  distributed_geometry geom = make_geom(nx, ny, nz, p, q, nodes, bounds);
  parameters sp             = unpack_params(params);
  u64 naux                  = scheme == 0 ? 8 : 4;
  simstate S(geom.core);
  for (u64 i = 0; i < S.size(); ++i) S[i] = U[i];
  simstate* aux = new simstate[naux];
  for (u64 i = 0; i < naux; ++i) aux[i] = simstate(geom.core);
  residual_workspace wsp(geom);
  {
    capture_stdout cap;
    for (int t = 0; t < nsteps; ++t)
    {
      if (scheme == 0)
        RK4_distributed(t, dt, S, aux, geom, sp, wsp);
      else
        tvdRK3_distributed(t, dt, S, aux, geom, sp, wsp);
    }
    if (norms_out) cap.read_norms(norms_out, nsteps);
  }
  for (u64 i = 0; i < S.size(); ++i) U[i] = S[i];
  delete[] aux;
  geom.free_dtypes();
  return 0;
}

/* reference geometry precomputes for one mesh: packed Minv per element,
 * detJ at volume quadrature points, physical basis gradients at volume points */
int ref_geometry(int nx, int ny, int nz, int p, int q, const double* nodes,
                 const long long* bounds, double* Minv_out, double* vJ_out,
                 double* vgrad_out, double* n_out, double* fJ_out,
                 long long* iface_out, long long* bface_out)
{
  distributed_geometry geom = make_geom(nx, ny, nz, p, q, nodes, bounds);
  if (Minv_out)
    for (u64 i = 0; i < geom.core.Minv_size(); ++i) Minv_out[i] = geom.core.Minv_[i];
  if (vJ_out)
    for (u64 i = 0; i < geom.core.vJ_size(); ++i) vJ_out[i] = geom.core.vJ_[i];
  if (vgrad_out)
    for (u64 i = 0; i < geom.core.vgrad_size(); ++i) vgrad_out[i] = geom.core.vgrad_[i];
  if (n_out)
    for (u64 i = 0; i < geom.n_size(); ++i) n_out[i] = geom.n_[i];
  if (fJ_out)
    for (u64 i = 0; i < geom.fJ_size(); ++i) fJ_out[i] = geom.fJ_[i];
  if (iface_out)
    for (u64 i = 0; i < geom.interior_face_list_size(); ++i)
      iface_out[i] = geom.interior_face_list[i];
  if (bface_out)
    for (u64 i = 0; i < geom.boundary_face_list_size(); ++i)
      bface_out[i] = geom.boundary_face_list[i];
  geom.free_dtypes();
  return 0;
}

long long ref_num_faces(int nx, int ny, int nz, int which, const long long* bounds)
{
  btype b[6];
  for (int i = 0; i < 6; ++i) b[i] = (btype)bounds[i];
  distributed_geometry geom(1, 1, nx, ny, nz, b, MPI_COMM_WORLD, 1, 1, 1, 1);
  if (which == 0) return (long long)geom.nface();
  if (which == 1) return (long long)geom.num_interior_faces();
  return (long long)geom.num_boundary_faces();
}

void ref_roe(const double* Ul, const double* Ur, const double* n, double g,
             double* f, double* smax)
{
  real a[5], b[5], nn[3];
  for (int i = 0; i < 5; ++i) { a[i] = Ul[i]; b[i] = Ur[i]; }
  for (int i = 0; i < 3; ++i) nn[i] = n[i];
  roe(a, b, nn, g, f, smax);
}

void ref_A(const double* s, const double* sx, const double* sy,
           const double* sz, double mu, double* Q)
{
  real a[5], bx[5], by[5], bz[5];
  for (int i = 0; i < 5; ++i) { a[i] = s[i]; bx[i] = sx[i]; by[i] = sy[i]; bz[i] = sz[i]; }
  A(a, bx, by, bz, mu, Q, Q + 5, Q + 10);
}

void ref_analytical_flux(const double* U, double g, double* F)
{
  real a[5];
  for (int i = 0; i < 5; ++i) a[i] = U[i];
  analytical_flux(a, g, F, F + 5, F + 10);
}

/* btype codes as boundaries.cpp:26-35 */
void ref_bc_state(long long bt, const double* UL, const double* n, double gamma,
                  double R, double Pt, double Tt, double P, double* Ub)
{
  real a[5], nn[3];
  for (int i = 0; i < 5; ++i) a[i] = UL[i];
  for (int i = 0; i < 3; ++i) nn[i] = n[i];
  switch (bt)
  {
    case inviscid_wall: inviscid_wall_state(a, nn, gamma, Ub); break;
    case no_slip_wall: no_slip_wall_state(a, Ub); break;
    case subsonic_inflow: subsonic_inflow_state(a, nn, gamma, R, Pt, Tt, Ub); break;
    case subsonic_outflow: subsonic_outflow_state(a, nn, gamma, P, Ub); break;
    default: break;
  }
}

void ref_gauss_legendre_1d(int order, double is, double ie, double* x, double* w)
{
  quad r = gauss_legendre_1d(order, is, ie);
  for (u64 i = 0; i < r.n; ++i) { x[i] = r.x[i]; w[i] = r.w[i]; }
}

/* reference basis tables for order p at quadrature order 2p+1 */
void ref_basis_tables(int p, double* veval, double* vgrad, double* feval,
                      double* fgrad)
{
  basis b(p, 2 * p + 1);
  if (veval) for (u64 i = 0; i < b.veval.len; ++i) veval[i] = b.veval[i];
  if (vgrad) for (u64 i = 0; i < b.vgrad.len; ++i) vgrad[i] = b.vgrad[i];
  if (feval) for (u64 i = 0; i < b.feval.len; ++i) feval[i] = b.feval[i];
  if (fgrad) for (u64 i = 0; i < b.fgrad.len; ++i) fgrad[i] = b.fgrad[i];
}

double ref_lagrange1d(int i, int p, double x) { return lagrange1d(i, p, x); }
double ref_lagrange1d_deriv(int i, int p, double x) { return lagrange1d_deriv(i, p, x); }

/* .dg writer/reader from the reference (io.cpp:33,92) for format checks */
int ref_write_state(const char* fname, unsigned long long tstep, int nx, int ny,
                    int nz, int p, int q, const long long* bounds,
                    const double* nodes, int noutput, const char** keys,
                    const double** data)
{
  s64 b[6];
  for (int i = 0; i < 6; ++i) b[i] = bounds[i];
  core_geometry core(p, q, nx, ny, nz, b);
  for (u64 i = 0; i < core.node_size(); ++i) core.node_[i] = nodes[i];
  map<simstate> outs;
  for (int o = 0; o < noutput; ++o)
  {
    simstate& s = outs.add(string(keys[o]), simstate(core));
    for (u64 i = 0; i < s.size(); ++i) s[i] = data[o][i];
  }
  write_state(fname, tstep, core, outs);
  return 0;
}

}  // extern "C"
