// Adjoint entry points of the C ABI (include/dgb200.h): residual VJP, the
// reverse of one RK step, and the recorded forward / backward pair with
// binomial checkpointing.  The reference has no adjoint; these follow its
// forward discretisation (solve.cpp:150-807, time_distributed.cpp:46-110).
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/dgb200.h"
#include "adjoint.hpp"
#include "handle.hpp"

using namespace dgb;

namespace {

#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_status(e_, #call); \
  } while (0)

int fail(int code, const char* msg) { return set_last_error(code, msg); }

int cuda_status_rc(cudaError_t e) { return e == cudaSuccess ? DGB_OK : cuda_status(e, "basis change"); }

// every boundary type has an adjoint (physics_vjp.cuh); kept as the hook for
// inputs the adjoint does not cover
int check_bounds(const dgb_handle*) { return DGB_OK; }

int ensure_adjoint(dgb_handle* h)
{
  if (h->d_adj_ta) return DGB_OK;
  const size_t sb = sizeof(double) * (size_t)h->n;
  const size_t tr = sizeof(double) * (size_t)h->E * 60 * h->NQF;
  cudaError_t e = cudaSuccess;
  for (int b = 0; b < dgb_handle::ADJ_NBUF && e == cudaSuccess; ++b) e = cudaMalloc(&h->d_adj[b], sb);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_adj_tr, tr);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_adj_ta, 2 * tr);
  if (e == cudaSuccess) e = prepare_adjoint(h->P);
  if (e != cudaSuccess) {
    free_adjoint(h);
    return cuda_status(e, "adjoint buffers");
  }
  return DGB_OK;
}

VjpScratch scratch(dgb_handle* h) { return {h->d_adj_tr, h->d_adj_ta, h->d_adj[dgb_handle::ADJ_PART], h->d_flag}; }

VjpArgs vjp(const double* U, double cx, const double* X, double cy = 0., const double* Y = nullptr,
            double cz = 0., const double* Z = nullptr)
{
  VjpArgs v{};  // every pointer not set below (Tr, a_out, acc_in, acc_out) stays null
  v.U = U;
  v.X = X;
  v.Y = Y;
  v.Z = Z;
  v.cx = cx;
  v.cy = cy;
  v.cz = cz;
  return v;
}

// ---- parameter gradient (dgb_backward_params)
// Per element e: part[e][0] = sum W . (F1 - F0) * inv_mu1 (F1 alone when F0
// is null) and
// part[e][1 + r] = sum_b W[r][b], with W = cx X + cy Y + cz Z the adjoint
// weight of one residual VJP; fixed-order block sums.
__global__ void param_dot_kernel(long E, int nb, VjpArgs v, const double* __restrict__ F1,
                                 const double* __restrict__ F0, double inv_mu1, double* __restrict__ part)
{
  __shared__ double red[DGB_NDPARAMS][128];
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  double acc[DGB_NDPARAMS] = {};
  for (int i = tid; i < 5 * nb; i += blockDim.x) {
    const long g = e * 5 * nb + i;
    double w = v.cx * v.X[g];
    if (v.Y) w = fma(v.cy, v.Y[g], w);
    if (v.Z) w = fma(v.cz, v.Z[g], w);
    acc[0] = fma(w, (F0 ? F1[g] - F0[g] : F1[g]) * inv_mu1, acc[0]);
    acc[1 + i / nb] += w;
  }
  for (int k = 0; k < DGB_NDPARAMS; ++k) red[k][tid] = acc[k];
  __syncthreads();
  for (int wdt = blockDim.x / 2; wdt > 0; wdt >>= 1) {
    if (tid < wdt)
      for (int k = 0; k < DGB_NDPARAMS; ++k) red[k][tid] += red[k][tid + wdt];
    __syncthreads();
  }
  if (tid < DGB_NDPARAMS) part[e * DGB_NDPARAMS + tid] = red[tid][0];
}

// dpar[0] += the isothermal-wall points' dJ/dTw terms, which adjA leaves in
// ta[e][lf][10][NQF] of every face with nbr == -8 (the nf faces 6 e + lf of
// wallf); fixed order
__global__ void wall_terms_kernel(long nf, int nqf, const int* __restrict__ wallf, const double* __restrict__ ta,
                                  double* dpar)
{
  __shared__ double red[256];
  const int tid = threadIdx.x;
  double acc = 0.;
  for (long i = tid; i < nf * nqf; i += blockDim.x) {
    const long ef = wallf[i / nqf];
    acc += ta[(ef * 20 + 10) * nqf + i % nqf];
  }
  red[tid] = acc;
  __syncthreads();
  for (int wdt = blockDim.x / 2; wdt > 0; wdt >>= 1) {
    if (tid < wdt) red[tid] += red[tid + wdt];
    __syncthreads();
  }
  if (tid == 0) dpar[0] += red[0];
}

// dpar[k] += sum_e part[e][k], fixed order
__global__ void param_reduce_kernel(long E, const double* __restrict__ part, double* dpar)
{
  __shared__ double red[DGB_NDPARAMS][256];
  const int tid = threadIdx.x;
  double acc[DGB_NDPARAMS] = {};
  for (long e = tid; e < E; e += blockDim.x)
    for (int k = 0; k < DGB_NDPARAMS; ++k) acc[k] += part[e * DGB_NDPARAMS + k];
  for (int k = 0; k < DGB_NDPARAMS; ++k) red[k][tid] = acc[k];
  __syncthreads();
  for (int wdt = blockDim.x / 2; wdt > 0; wdt >>= 1) {
    if (tid < wdt)
      for (int k = 0; k < DGB_NDPARAMS; ++k) red[k][tid] += red[k][tid + wdt];
    __syncthreads();
  }
  if (tid < DGB_NDPARAMS) dpar[tid] += red[tid][0];
}

// d_pg: F1 [n], F0 [n], FP64 traces [E][60][NQF], partials [E][DGB_NDPARAMS],
// the host entry point's device copy of dJ/dparams [DGB_NDPARAMS]
size_t pgrad_doubles(const dgb_handle* h)
{
  return 2 * (size_t)h->n + (size_t)h->E * 60 * h->NQF + (size_t)h->E * DGB_NDPARAMS + DGB_NDPARAMS;
}

int ensure_pgrad(dgb_handle* h)
{
  if (h->d_pg) return DGB_OK;
  CK(cudaMalloc(&h->d_pg, sizeof(double) * pgrad_doubles(h)));
  return DGB_OK;
}

// W^T df/dtheta for one residual VJP v (before it runs: it may overwrite
// v.Y in place), added into dpar.  f is affine in mu (the viscous flux and
// the heat flux at fixed Pr are linear in it), so df/dmu = (f(mu1) - f(0)) /
// mu1, both FP64 residuals of v.U, in the nodal form; the Gauss-point form
// evaluates the viscous terms alone at mu1 (vlaunch_stage_visc), f(mu1) - f(0)
// in one residual.  df/dsource[r] = 1 on variable r.
int enqueue_param_terms(dgb_handle* h, const VjpArgs& v, double* dpar, bool gauss)
{
  KLaunch L = klaunch(h);
  L.precision = DGB_FP64;
  L.ops = L.opsd;
  KLaunch L1 = L, L0 = L;
  const double mu1 = h->dprm.mu != 0. ? h->dprm.mu : 1.;
  if (h->dprm.mu == 0.) {
    dgb_params p1 = h->prm;
    p1.mu = mu1;
    L1.prm = device_params(p1, h->prandtl, h->twall);
  }
  L0.prm.mu = 0.;
  L0.prm.kq = 0.;
  double* F1 = h->d_pg;
  double* F0 = F1 + h->n;
  double* trp = F0 + h->n;
  double* part = trp + (size_t)h->E * 60 * h->NQF;
  if (gauss) {  // f_V's viscous terms alone at mu1, without the source: mu1 df_V/dmu in one residual
    KLaunch Lv = L1;
    for (int r = 0; r < 5; ++r) Lv.prm.src[r] = 0.;
    StageArgs a = stage_args(MODE_RESIDUAL, 0.);
    a.fout = F1;
    a.flag = h->d_flag;
    // the VJP's FP64 traces of v.U are these traces when mu1 is the handle's mu
    const double* tr = v.Tr && h->dprm.mu != 0. ? v.Tr : trp;
    if (tr == trp) CK(launch_vtrace(Lv, v.U, trp, h->stream));
    CK(vlaunch_stage_visc(Lv, v.U, tr, a, h->stream));
    F0 = nullptr;
  } else {
    const KLaunch* Ls[2] = {&L1, &L0};
    double* Fs[2] = {F1, F0};
    for (int k = 0; k < 2; ++k) {  // f(mu1) and f(0)
      StageArgs a = stage_args(MODE_RESIDUAL, 0.);
      a.fout = Fs[k];
      a.flag = h->d_flag;
      CK(launch_trace(*Ls[k], v.U, trp, h->stream));
      CK(launch_stage(*Ls[k], v.U, trp, a, h->stream));
    }
  }
  param_dot_kernel<<<(unsigned)h->E, 128, 0, h->stream>>>(h->E, h->NB, v, F1, F0, 1. / mu1, part);
  CK(cudaGetLastError());
  param_reduce_kernel<<<1, 256, 0, h->stream>>>(h->E, part, dpar);
  CK(cudaGetLastError());
  return DGB_OK;
}

// Reverse of one RK step from U_i (device, unchanged) with lam = adjoint of
// U_{i+1} in, adjoint of U_i out (in place).  The stage states are recomputed
// in the handle's precision, then one residual VJP per stage runs backwards.
// With f = -Minv R, J_s = df/dU at stage state S_s and a_s = J_s^T (...):
//   RK4   U1 = U + dt/2 k1, U2 = U + dt/2 k2, U3 = U + dt k3,
//         U' = U + dt/6 (k1 + 2 k2 + 2 k3 + k4)
//         a3 = J3^T (dt/6 lam)        a2 = J2^T (dt/3 lam + dt a3)
//         a1 = J1^T (dt/3 lam + dt/2 a2)   a0 = J0^T (dt/6 lam + dt/2 a1)
//   TVD   U1 = U + dt f(U), U2 = 3/4 U + 1/4 U1 + dt/4 f(U1),
//         U' = 1/3 U + 2/3 U2 + 2/3 dt f(U2)  (time_distributed.cpp:79-110)
//         a2 = J2^T (2/3 dt lam)      a1 = J1^T (dt/6 lam + dt/4 a2)
//         a0 = J0^T (dt/6 lam + dt/4 a2 + dt a1)
//   and in both  lam_i = lam + a0 + a1 + a2 (+ a3).
// Face traces: an FP64 handle keeps the traces of U_i and of every
// recomputed stage state (the stage epilogues write them) and hands them to
// the VJPs; a mixed-precision handle recomputes the stages in FP32 with
// rotating trace buffers and each VJP takes its own FP64 traces.
// With `stored` (the recorded stage states of this step) nothing is
// recomputed: an FP64 handle takes the traces of the stored states.
// gauss: Ui, lam, the stage states and the result are Gauss-point arrays
// (the Gauss-point form of vspace.cuh, with its stage, trace and VJP
// kernels), else nodal.
int enqueue_reverse_step(dgb_handle* h, int scheme, double dt, const double* Ui, double* lam, long long* nl,
                         double* const* stored = nullptr, double* dpar = nullptr, bool gauss = false)
{
  const KLaunch L = klaunch(h);
  auto trace = [&](const double* U, void* Tout) {
    return gauss ? launch_vtrace(L, U, Tout, h->stream) : launch_trace(L, U, Tout, h->stream);
  };
  double* S[3] = {h->d_adj[dgb_handle::ADJ_S0], h->d_adj[dgb_handle::ADJ_S1], h->d_adj[dgb_handle::ADJ_S2]};
  if (stored)
    for (int s = 0; s < 3; ++s) S[s] = stored[s];
  double* A0 = h->d_adj[dgb_handle::ADJ_A0];
  double* A1 = h->d_adj[dgb_handle::ADJ_A1];
  double* ACC = h->d_adj[dgb_handle::ADJ_ACC];
  const VjpScratch sc = scratch(h);
  const bool f64 = h->precision == DGB_FP64;
  void* const* T = h->d_trace;
  void* TU = f64 ? (void*)h->d_adj_tr : T[0];
  if (f64 || !stored) CK(trace(Ui, TU));
  const int nst = scheme == DGB_RK4 ? 3 : 2;  // recomputed stage states
  const int rk4[3] = {MODE_RK4_0, MODE_RK4_1, MODE_RK4_2}, tvd[2] = {MODE_TVD_0, MODE_TVD_1};
  // trace buffers read / written by the recomputed stages
  const void* tin_f64[3] = {TU, T[0], T[1]};
  void* tout_f64[3] = {T[0], T[1], T[2]};
  const void* tin_mix[3] = {T[0], T[1], T[0]};
  void* tout_mix[3] = {T[1], T[0], nullptr};
  if (scheme != DGB_RK4) tout_mix[1] = nullptr;
  for (int s = 0; s < nst; ++s) {
    if (stored) {  // the stage state is at hand; an FP64 handle still needs its traces
      if (f64) CK(trace(S[s], tout_f64[s]));
      continue;
    }
    StageArgs a = stage_args(scheme == DGB_RK4 ? rk4[s] : tvd[s], dt);
    a.Ubase = Ui;
    a.acc = nullptr;  // the RK4 accumulator only forms the step's end state, which a reverse step does not need
    a.Uout = S[s];
    a.flag = h->d_flag;
    a.Tnext = f64 ? tout_f64[s] : tout_mix[s];
    if (gauss)
      CK(launch_vstage(L, s == 0 ? Ui : S[s - 1], f64 ? tin_f64[s] : tin_mix[s], a, h->stream));
    else
      CK(launch_stage(L, s == 0 ? Ui : S[s - 1], f64 ? tin_f64[s] : tin_mix[s], a, h->stream));
  }
  auto tr = [&](int s) -> const double* {  // FP64 traces of stage state s (-1: U_i)
    if (!f64) return nullptr;
    return (const double*)(s < 0 ? TU : tout_f64[s]);
  };
  int rc;
  auto vjp_launch = [&](const VjpArgs& w) {
    return gauss ? launch_residual_vjp_gauss(L, w, sc, h->stream) : launch_residual_vjp(L, w, sc, h->stream);
  };
  auto run_vjp = [&](const VjpArgs& w0) -> int {
    if (!dpar) {
      CK(vjp_launch(w0));
      return DGB_OK;
    }
    VjpArgs w = w0;
    if (gauss && h->dprm.mu != 0. && !w.Tr) {  // one set of FP64 traces for the parameter terms and the VJP
      KLaunch L64 = klaunch(h);
      L64.precision = DGB_FP64;
      L64.ops = L64.opsd;
      CK(launch_vtrace(L64, w.U, sc.trace, h->stream));
      w.Tr = sc.trace;
    }
    const int r = enqueue_param_terms(h, w, dpar, gauss);
    if (r) return r;
    CK(vjp_launch(w));
    if (h->n_wallf) {  // the VJP left the isothermal walls' dJ/dTw terms in its trace adjoints
      wall_terms_kernel<<<1, 256, 0, h->stream>>>(h->n_wallf, h->NQF, h->d_wallf, sc.ta, dpar + DGB_DPARAM_TWALL);
      CK(cudaGetLastError());
    }
    return DGB_OK;
  };
  VjpArgs v{};
  if (scheme == DGB_RK4) {
    v = vjp(S[2], dt / 6., lam);
    v.Tr = tr(2);
    v.a_out = A0;
    v.acc_in = lam;
    v.acc_out = ACC;
    if ((rc = run_vjp(v))) return rc;
    v = vjp(S[1], dt / 3., lam, dt, A0);
    v.Tr = tr(1);
    v.a_out = A0;
    v.acc_in = ACC;
    v.acc_out = ACC;
    if ((rc = run_vjp(v))) return rc;
    v = vjp(S[0], dt / 3., lam, dt / 2., A0);
    v.Tr = tr(0);
    v.a_out = A0;
    v.acc_in = ACC;
    v.acc_out = ACC;
    if ((rc = run_vjp(v))) return rc;
    v = vjp(Ui, dt / 6., lam, dt / 2., A0);
  } else {
    v = vjp(S[1], 2. * dt / 3., lam);
    v.Tr = tr(1);
    v.a_out = A0;
    v.acc_in = lam;
    v.acc_out = ACC;
    if ((rc = run_vjp(v))) return rc;
    v = vjp(S[0], dt / 6., lam, dt / 4., A0);
    v.Tr = tr(0);
    v.a_out = A1;
    v.acc_in = ACC;
    v.acc_out = ACC;
    if ((rc = run_vjp(v))) return rc;
    v = vjp(Ui, dt / 6., lam, dt / 4., A0, dt, A1);
  }
  v.Tr = tr(-1);
  v.acc_in = ACC;
  v.acc_out = lam;
  if ((rc = run_vjp(v))) return rc;
  if (nl) *nl += (stored && !f64 ? 0 : 1 + nst) + (nst + 1) * ((f64 ? 2 : 3) + (dpar ? 6 : 0));
  return DGB_OK;
}

// The captured graph of one reverse step of the work state d_U with the
// adjoint in ADJ_LAM (the backward sweep's REVERSE operation).
int ensure_rev_graph(dgb_handle* h, int scheme, double dt, bool gauss)
{
  if (h->rev_graph && h->rev_scheme == scheme && h->rev_dt == dt && h->rev_gauss == gauss) return DGB_OK;
  if (h->rev_graph) cudaGraphExecDestroy(h->rev_graph);
  h->rev_graph = nullptr;
  h->rev_scheme = -1;
  cudaGraph_t g;
  long long nl = 0;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_reverse_step(h, scheme, dt, gauss ? h->d_V : h->d_U, h->d_adj[dgb_handle::ADJ_LAM], &nl,
                                nullptr, nullptr, gauss);
  cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
  if (rc) {
    if (ce == cudaSuccess) cudaGraphDestroy(g);
    return rc;
  }
  if (ce != cudaSuccess) return cuda_status(ce, "cudaStreamEndCapture");
  ce = cudaGraphInstantiate(&h->rev_graph, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return cuda_status(ce, "cudaGraphInstantiate");
  h->rev_scheme = scheme;
  h->rev_dt = dt;
  h->rev_gauss = gauss;
  h->rev_launches = nl;
  return DGB_OK;
}

int read_flag(dgb_handle* h)
{
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag & 8) return fail(DGB_ERR_UNSUPPORTED, "boundary state without an adjoint");
  if (flag & 2) return fail(DGB_ERR_BOUNDARY, "subsonic inflow without a non-negative Mach root");
  return DGB_OK;
}

int copy_state(dgb_handle* h, double* dst, const double* src)
{
  if (dst == src) return DGB_OK;
  CK(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToDevice, h->stream));
  return DGB_OK;
}

int check_scheme(int scheme, double dt)
{
  if (scheme != DGB_RK4 && scheme != DGB_TVDRK3) return fail(DGB_ERR_ARG, "unknown time scheme");
  if (!(dt == dt)) return fail(DGB_ERR_ARG, "dt is NaN");
  return DGB_OK;
}

}  // namespace

void dgb::free_adjoint(dgb_handle* h)
{
  if (h->rev_graph) cudaGraphExecDestroy(h->rev_graph);
  h->rev_graph = nullptr;
  h->rev_scheme = -1;
  for (double*& p : h->d_adj) {
    if (p) cudaFree(p);
    p = nullptr;
  }
  if (h->d_adj_tr) cudaFree(h->d_adj_tr);
  if (h->d_adj_ta) cudaFree(h->d_adj_ta);
  h->d_adj_tr = h->d_adj_ta = nullptr;
  if (h->d_pg) cudaFree(h->d_pg);
  h->d_pg = nullptr;
  for (double* p : h->d_slots)
    if (p) cudaFree(p);
  h->d_slots.clear();
  if (h->d_stage_store) cudaFree(h->d_stage_store);
  h->d_stage_store = nullptr;
  h->stage_store_cap = 0;
  h->recorded = false;
}

extern "C" {

int dgb_residual_vjp_device(dgb_handle* h, const double* U_dev, const double* lam_dev, double* Ubar_dev)
{
  if (!h || !U_dev || !lam_dev || !Ubar_dev) return fail(DGB_ERR_ARG, "null argument");
  if (Ubar_dev == U_dev || Ubar_dev == lam_dev) return fail(DGB_ERR_ARG, "Ubar must not alias U or lam");
  int rc = check_bounds(h);
  if (rc) return rc;
  CK(cudaSetDevice(h->device));
  if ((rc = ensure_adjoint(h))) return rc;
  VjpArgs v = vjp(U_dev, 1., lam_dev);
  v.a_out = Ubar_dev;
  CK(launch_residual_vjp(klaunch(h), v, scratch(h), h->stream));
  h->last_launches = 3;
  return DGB_OK;
}

int dgb_residual_vjp(dgb_handle* h, const double* U_host, const double* lam_host, double* Ubar_host)
{
  if (!h || !U_host || !lam_host || !Ubar_host) return fail(DGB_ERR_ARG, "null argument");
  int rc = check_bounds(h);
  if (rc) return rc;
  CK(cudaSetDevice(h->device));
  if ((rc = ensure_adjoint(h))) return rc;
  const size_t sb = sizeof(double) * (size_t)h->n;
  double* in = h->d_adj[dgb_handle::ADJ_IN];
  double* out = h->d_adj[dgb_handle::ADJ_OUT];
  double* lam = h->d_adj[dgb_handle::ADJ_LAM];
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  CK(cudaMemcpyAsync(in, U_host, sb, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(lam, lam_host, sb, cudaMemcpyHostToDevice, h->stream));
  VjpArgs v = vjp(in, 1., lam);
  v.a_out = out;
  CK(launch_residual_vjp(klaunch(h), v, scratch(h), h->stream));
  h->last_launches = 3;
  CK(cudaMemcpyAsync(Ubar_host, out, sb, cudaMemcpyDeviceToHost, h->stream));
  return read_flag(h);
}

int dgb_step_vjp_device(dgb_handle* h, int scheme, double dt, const double* U_dev, double* lam_dev)
{
  if (!h || !U_dev || !lam_dev) return fail(DGB_ERR_ARG, "null argument");
  if ((const double*)lam_dev == U_dev) return fail(DGB_ERR_ARG, "lam must not alias U");
  int rc = check_scheme(scheme, dt);
  if (rc) return rc;
  if ((rc = check_bounds(h))) return rc;
  CK(cudaSetDevice(h->device));
  if ((rc = ensure_adjoint(h))) return rc;
  for (int b = 0; b < dgb_handle::ADJ_NBUF; ++b)
    if (U_dev == h->d_adj[b] || lam_dev == h->d_adj[b]) return fail(DGB_ERR_ARG, "argument aliases scratch");
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  long long nl = 0;
  if (h->gauss_step) {  // the VJP of dgb_step's map U -> B3^-1 Phi_V(B3 U)
    const KLaunch L = klaunch(h);
    double* V = h->d_adj[dgb_handle::ADJ_IN];
    double* lamV = h->d_adj[dgb_handle::ADJ_OUT];
    CK(launch_gauss_basis_mode(L, U_dev, V, GB_TO_GAUSS, h->stream));
    CK(launch_gauss_basis_mode(L, lam_dev, lamV, GB_ADJ_TO_GAUSS, h->stream));
    if ((rc = enqueue_reverse_step(h, scheme, dt, V, lamV, &nl, nullptr, nullptr, true))) return rc;
    CK(launch_gauss_basis_mode(L, lamV, lam_dev, GB_ADJ_TO_NODAL, h->stream));
    nl += 3;
  } else {
    if ((rc = enqueue_reverse_step(h, scheme, dt, U_dev, lam_dev, &nl))) return rc;
  }
  h->last_launches = nl;
  return read_flag(h);
}

int dgb_forward_record(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, int slots,
                       double* norms_host)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  int rc = check_scheme(scheme, dt);
  if (rc) return rc;
  if (nsteps < 1 || slots < 1) return fail(DGB_ERR_ARG, "need nsteps >= 1 and slots >= 1");
  if ((rc = check_bounds(h))) return rc;
  CK(cudaSetDevice(h->device));
  if ((rc = ensure_adjoint(h))) return rc;
  h->recorded = false;
  if (make_checkpoint_plan((long long)nsteps, slots, h->plan)) return fail(DGB_ERR_ARG, "bad checkpoint plan");
  const int need = h->plan.slots;
  while ((int)h->d_slots.size() > need) {
    cudaFree(h->d_slots.back());
    h->d_slots.pop_back();
  }
  while ((int)h->d_slots.size() < need) {
    double* p = nullptr;
    CK(cudaMalloc(&p, sizeof(double) * (size_t)h->n));
    h->d_slots.push_back(p);
  }
  // the run steps in dgb_step's form: on d_V (Gauss points) or on d_U
  const bool gauss = h->gauss_step;
  double* Ures = gauss ? h->d_V : h->d_U;
  if ((rc = ensure_step_graph(h, scheme, dt, nsteps, gauss))) return rc;
  CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  if (gauss && !h->v_current) CK(launch_gauss_basis(klaunch(h), h->d_U, h->d_V, true, h->stream));
  // Between graph replays the face traces of the resident state stay valid
  // (each step's last stage writes them), and storing a checkpoint does not
  // change the state: only the first replay needs the trace kernel.
  bool need_trace = true;
  long long launches = 0;
  for (size_t k = 0; k < h->plan.first_reverse; ++k) {
    const CkOp& op = h->plan.ops[k];
    if (op.kind == CK_STORE) {
      if ((rc = copy_state(h, h->d_slots[op.arg], Ures))) return rc;
    } else if (op.kind == CK_FORWARD) {
      if ((rc = enqueue_steps(h, (unsigned long long)op.arg, need_trace, gauss))) return rc;
      launches += (need_trace ? 1 : 0) + op.arg * h->launches_per_step;
      need_trace = false;
    } else {
      return fail(DGB_ERR_ARG, "checkpoint plan restores during the forward run");
    }
  }
  // work state is U_{N-1}: keep it, take the last step on the resident state
  if ((rc = copy_state(h, h->d_adj[dgb_handle::ADJ_WORK], Ures))) return rc;
  if ((rc = enqueue_steps(h, 1, need_trace, gauss))) return rc;
  launches += (need_trace ? 1 : 0) + h->launches_per_step;
  if ((rc = copy_state(h, h->d_adj[dgb_handle::ADJ_FINAL], Ures))) return rc;
  if (gauss) CK(launch_gauss_basis(klaunch(h), h->d_V, h->d_U, false, h->stream));
  h->v_current = gauss;
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (norms_host)
    CK(cudaMemcpyAsync(norms_host, h->d_norms, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag & 1) return fail(DGB_ERR_NONFINITE, "residual norm became NaN/Inf");
  if (flag & 16) return fail(DGB_ERR_CUDA, "tensor-core stage: a wait for the tensor cores gave up");
  if (flag & 2) return fail(DGB_ERR_BOUNDARY, "subsonic inflow without a non-negative Mach root");
  h->plan_pos = h->plan.first_reverse;
  h->recorded = true;
  h->rec_stages = false;
  h->rec_gauss = gauss;
  h->slots_dirty = false;
  h->rec_scheme = scheme;
  h->rec_dt = dt;
  h->rec_steps = nsteps;
  h->last_launches = launches;
  return DGB_OK;
}

int dgb_forward_record_stages(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, double* norms_host)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  int rc = check_scheme(scheme, dt);
  if (rc) return rc;
  if (nsteps < 1) return fail(DGB_ERR_ARG, "need nsteps >= 1");
  if ((rc = check_bounds(h))) return rc;
  CK(cudaSetDevice(h->device));
  if ((rc = ensure_adjoint(h))) return rc;
  h->recorded = false;
  const int nst = scheme == DGB_RK4 ? 4 : 3;
  // every state U_0 .. U_{N-1} in the slots, every intermediate stage state
  // in one store
  while (h->d_slots.size() > nsteps) {
    cudaFree(h->d_slots.back());
    h->d_slots.pop_back();
  }
  while (h->d_slots.size() < nsteps) {
    double* p = nullptr;
    CK(cudaMalloc(&p, sizeof(double) * (size_t)h->n));
    h->d_slots.push_back(p);
  }
  const size_t need = (size_t)nsteps * (nst - 1) * (size_t)h->n;
  if (need > h->stage_store_cap) {
    if (h->d_stage_store) CK(cudaFree(h->d_stage_store));
    h->d_stage_store = nullptr;
    h->stage_store_cap = 0;
    CK(cudaMalloc(&h->d_stage_store, sizeof(double) * need));
    h->stage_store_cap = need;
  }
  if (nsteps > h->norms_cap) {  // room for every step's norm (ensure_step_graph grows it)
    if ((rc = ensure_step_graph(h, scheme, dt, nsteps))) return rc;
  }
  CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  // the step of enqueue_step (capi.cu) launch by launch, in dgb_step's form,
  // with every stage state written to its own buffer: the same kernels on the
  // same inputs, so the states are those dgb_step computes, bit for bit
  const KLaunch L = klaunch(h);
  const bool gauss = h->gauss_step;
  double* Ures = gauss ? h->d_V : h->d_U;
  if (gauss && !h->v_current) CK(launch_gauss_basis(L, h->d_U, h->d_V, true, h->stream));
  const int rk4[4] = {MODE_RK4_0, MODE_RK4_1, MODE_RK4_2, MODE_RK4_3};
  const int tvd[3] = {MODE_TVD_0, MODE_TVD_1, MODE_TVD_2};
  const int tin4[4] = {0, 1, 0, 1}, tout4[4] = {1, 0, 1, 0};
  const int tin3[3] = {0, 1, 2}, tout3[3] = {1, 2, 0};
  if (gauss)
    CK(launch_vtrace(L, Ures, h->d_trace[0], h->stream));
  else
    CK(launch_trace(L, Ures, h->d_trace[0], h->stream));
  long long launches = 1;
  for (unsigned long long i = 0; i < nsteps; ++i) {
    if ((rc = copy_state(h, h->d_slots[i], Ures))) return rc;
    double* Si = h->d_stage_store + (size_t)i * (nst - 1) * (size_t)h->n;
    for (int st = 0; st < nst; ++st) {
      StageArgs a = stage_args(scheme == DGB_RK4 ? rk4[st] : tvd[st], dt);
      a.Ubase = Ures;
      a.acc = h->d_acc;
      a.Uout = st == nst - 1 ? Ures : Si + (size_t)st * h->n;
      a.part = st == 0 ? h->d_part : nullptr;
      a.flag = h->d_flag;
      a.Tnext = h->d_trace[scheme == DGB_RK4 ? tout4[st] : tout3[st]];
      const double* in = st == 0 ? Ures : Si + (size_t)(st - 1) * h->n;
      const void* tin = h->d_trace[scheme == DGB_RK4 ? tin4[st] : tin3[st]];
      if (gauss)
        CK(launch_vstage(L, in, tin, a, h->stream));
      else
        CK(launch_stage(L, in, tin, a, h->stream));
      ++launches;
      if (st == 0) {
        CK(launch_norm(h->E, h->d_part, 1.0 / (double)h->n, h->d_norms, (long)h->norms_cap, h->d_counter,
                       h->d_flag, h->stream));
        ++launches;
      }
    }
  }
  if ((rc = copy_state(h, h->d_adj[dgb_handle::ADJ_FINAL], Ures))) return rc;
  if (gauss) CK(launch_gauss_basis(L, h->d_V, h->d_U, false, h->stream));
  h->v_current = gauss;
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (norms_host)
    CK(cudaMemcpyAsync(norms_host, h->d_norms, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag & 1) return fail(DGB_ERR_NONFINITE, "residual norm became NaN/Inf");
  if (flag & 16) return fail(DGB_ERR_CUDA, "tensor-core stage: a wait for the tensor cores gave up");
  if (flag & 2) return fail(DGB_ERR_BOUNDARY, "subsonic inflow without a non-negative Mach root");
  h->recorded = true;
  h->rec_stages = true;
  h->rec_gauss = gauss;
  h->rec_scheme = scheme;
  h->rec_dt = dt;
  h->rec_steps = nsteps;
  h->slots_dirty = false;
  h->last_launches = launches;
  return DGB_OK;
}

}  // extern "C"

namespace {

// the backward sweep of dgb_backward_device; with dpar (device,
// DGB_NDPARAMS doubles, zeroed here) also the parameter gradient
int backward_impl(dgb_handle* h, const double* lamN_dev, double* lam0_dev, double* dpar)
{
  if (!h || !lamN_dev || !lam0_dev) return fail(DGB_ERR_ARG, "null argument");
  if (!h->recorded) return fail(DGB_ERR_ARG, "no recorded forward run (dgb_forward_record)");
  CK(cudaSetDevice(h->device));
  // the sweep works in the recorded run's form; adjoint vectors cross the
  // basis change as dJ/dV = B3^-T dJ/dU, dJ/dU = B3^T dJ/dV
  const bool gauss = h->rec_gauss;
  double* Ures = gauss ? h->d_V : h->d_U;
  const KLaunch L = klaunch(h);
  auto lam_in = [&](double* lam) {
    return gauss ? cuda_status_rc(launch_gauss_basis_mode(L, lamN_dev, lam, GB_ADJ_TO_GAUSS, h->stream))
                 : copy_state(h, lam, lamN_dev);
  };
  auto lam_out = [&](const double* lam) {
    return gauss ? cuda_status_rc(launch_gauss_basis_mode(L, lam, lam0_dev, GB_ADJ_TO_NODAL, h->stream))
                 : copy_state(h, lam0_dev, lam);
  };
  if (dpar) {
    const int rc = ensure_pgrad(h);
    if (rc) return rc;
    CK(cudaMemsetAsync(dpar, 0, sizeof(double) * DGB_NDPARAMS, h->stream));
  }
  if (h->rec_stages) {  // every state and stage state was kept: reverse only
    const int nst = h->rec_scheme == DGB_RK4 ? 4 : 3;
    double* lam = h->d_adj[dgb_handle::ADJ_LAM];
    int rc;
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    if ((rc = lam_in(lam))) return rc;
    long long nl = 0;
    for (unsigned long long k = h->rec_steps; k-- > 0;) {
      double* Si = h->d_stage_store + (size_t)k * (nst - 1) * (size_t)h->n;
      double* stored[3] = {Si, Si + (size_t)h->n, nst > 3 ? Si + 2 * (size_t)h->n : nullptr};
      if ((rc = enqueue_reverse_step(h, h->rec_scheme, h->rec_dt, h->d_slots[k], lam, &nl, stored, dpar, gauss)))
        return rc;
    }
    if ((rc = lam_out(lam))) return rc;
    h->last_launches = nl;
    h->adj_forward_steps = 0;
    h->adj_reverse_steps = (long long)h->rec_steps;
    return read_flag(h);
  }
  const int scheme = h->rec_scheme;
  const double dt = h->rec_dt;
  double* lam = h->d_adj[dgb_handle::ADJ_LAM];
  int rc;
  // dgb_step calls since the record may have replaced the step graph
  if ((rc = ensure_step_graph(h, scheme, dt, h->rec_steps, gauss))) return rc;
  if ((rc = ensure_rev_graph(h, scheme, dt, gauss))) return rc;
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  h->v_current = false;  // the sweep moves the resident state
  long long nl = 0, fwd = 0, rev = 0;
  if (h->slots_dirty) {
    // an earlier sweep overwrote checkpoints: rebuild them from U_0 (buffer 0
    // is never overwritten) by replaying the recorded run's part of the plan
    if ((rc = copy_state(h, Ures, h->d_slots[0]))) return rc;
    bool need_trace = true;
    for (size_t k = 1; k < h->plan_pos; ++k) {
      const CkOp& op = h->plan.ops[k];
      if (op.kind == CK_STORE) {
        if ((rc = copy_state(h, h->d_slots[op.arg], Ures))) return rc;
      } else {
        CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
        if ((rc = enqueue_steps(h, (unsigned long long)op.arg, need_trace, gauss))) return rc;
        nl += (need_trace ? 1 : 0) + op.arg * h->launches_per_step;
        need_trace = false;
        fwd += op.arg;
      }
    }
  } else {
    if ((rc = copy_state(h, Ures, h->d_adj[dgb_handle::ADJ_WORK]))) return rc;
  }
  if ((rc = lam_in(lam))) return rc;
  for (size_t k = h->plan_pos; k < h->plan.ops.size(); ++k) {
    const CkOp& op = h->plan.ops[k];
    switch (op.kind) {
      case CK_REVERSE:
        if (dpar) {  // the captured reverse step has no parameter terms
          if ((rc = enqueue_reverse_step(h, scheme, dt, Ures, lam, &nl, nullptr, dpar, gauss))) return rc;
        } else {
          CK(cudaGraphLaunch(h->rev_graph, h->stream));
          nl += h->rev_launches;
        }
        ++rev;
        break;
      case CK_RESTORE:
        if ((rc = copy_state(h, Ures, h->d_slots[op.arg]))) return rc;
        break;
      case CK_STORE:
        if ((rc = copy_state(h, h->d_slots[op.arg], Ures))) return rc;
        h->slots_dirty = true;
        break;
      case CK_FORWARD:
        // the reverse steps reuse the trace buffers: recompute the traces
        CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
        if ((rc = enqueue_steps(h, (unsigned long long)op.arg, true, gauss))) return rc;
        nl += 1 + op.arg * h->launches_per_step;
        fwd += op.arg;
        break;
    }
  }
  if ((rc = lam_out(lam))) return rc;
  if ((rc = copy_state(h, Ures, h->d_adj[dgb_handle::ADJ_FINAL]))) return rc;
  if (gauss) CK(launch_gauss_basis(L, h->d_V, h->d_U, false, h->stream));
  h->v_current = gauss;
  h->last_launches = nl;
  h->adj_forward_steps = fwd;
  h->adj_reverse_steps = rev;
  return read_flag(h);
}

}  // namespace

extern "C" {

int dgb_backward_device(dgb_handle* h, const double* lamN_dev, double* lam0_dev)
{
  return backward_impl(h, lamN_dev, lam0_dev, nullptr);
}

int dgb_backward_params_device(dgb_handle* h, const double* lamN_dev, double* lam0_dev, double* dpar_dev)
{
  if (!dpar_dev) return fail(DGB_ERR_ARG, "null argument");
  return backward_impl(h, lamN_dev, lam0_dev, dpar_dev);
}

int dgb_backward_params(dgb_handle* h, const double* lamN_host, double* lam0_host, double* dpar_host)
{
  if (!h || !lamN_host || !lam0_host || !dpar_host) return fail(DGB_ERR_ARG, "null argument");
  if (!h->recorded) return fail(DGB_ERR_ARG, "no recorded forward run (dgb_forward_record)");
  CK(cudaSetDevice(h->device));
  int rc = ensure_pgrad(h);
  if (rc) return rc;
  const size_t sb = sizeof(double) * (size_t)h->n;
  double* in = h->d_adj[dgb_handle::ADJ_IN];
  double* out = h->d_adj[dgb_handle::ADJ_OUT];
  double* dpar = h->d_pg + pgrad_doubles(h) - DGB_NDPARAMS;
  CK(cudaMemcpyAsync(in, lamN_host, sb, cudaMemcpyHostToDevice, h->stream));
  if ((rc = backward_impl(h, in, out, dpar))) return rc;
  CK(cudaMemcpyAsync(lam0_host, out, sb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(dpar_host, dpar, sizeof(double) * DGB_NDPARAMS, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DGB_OK;
}

int dgb_backward(dgb_handle* h, const double* lamN_host, double* lam0_host)
{
  if (!h || !lamN_host || !lam0_host) return fail(DGB_ERR_ARG, "null argument");
  if (!h->recorded) return fail(DGB_ERR_ARG, "no recorded forward run (dgb_forward_record)");
  CK(cudaSetDevice(h->device));
  const size_t sb = sizeof(double) * (size_t)h->n;
  double* in = h->d_adj[dgb_handle::ADJ_IN];
  double* out = h->d_adj[dgb_handle::ADJ_OUT];
  CK(cudaMemcpyAsync(in, lamN_host, sb, cudaMemcpyHostToDevice, h->stream));
  int rc = dgb_backward_device(h, in, out);
  if (rc) return rc;
  CK(cudaMemcpyAsync(lam0_host, out, sb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DGB_OK;
}

int dgb_adjoint_stats(const dgb_handle* h, long long* forward_steps, long long* reverse_steps,
                      long long* planned_forward_steps)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (forward_steps) *forward_steps = h->adj_forward_steps;
  if (reverse_steps) *reverse_steps = h->adj_reverse_steps;
  if (planned_forward_steps) *planned_forward_steps = h->plan.forward_steps;
  return DGB_OK;
}

}  // extern "C"
