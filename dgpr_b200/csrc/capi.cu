// C ABI (include/dgb200.h): handle life cycle, state transfer, residual,
// CUDA-graph RK stepping, and the host-only helpers.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/dgb200.h"
#include "handle.hpp"
#include "host.hpp"
#include "kernels.hpp"

using namespace dgb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return DGB_ERR_CUDA;
}

#define CK(call)                                 \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

// one residual of Uin (device) into f / R (device), on the handle's stream
int enqueue_residual(dgb_handle* h, const double* Uin, double* R, double* f)
{
  const KLaunch L = klaunch(h);
  CK(launch_trace(L, Uin, h->d_trace[0], h->stream));
  StageArgs a = stage_args(MODE_RESIDUAL, 0.);
  a.fout = f;
  a.Rout = R;
  a.flag = h->d_flag;
  CK(launch_stage(L, Uin, h->d_trace[0], a, h->stream));
  return DGB_OK;
}

// Traces of the resident state, read by the first stage of the next step.
// Every dgb_step call starts with this one launch; later stages and steps get
// their traces from the epilogue of the stage before.
int enqueue_initial_traces(dgb_handle* h, bool gauss)
{
  if (gauss)
    CK(launch_vtrace(klaunch(h), h->d_V, h->d_trace[0], h->stream));
  else
    CK(launch_trace(klaunch(h), h->d_U, h->d_trace[0], h->stream));
  return DGB_OK;
}

// One full RK step as a launch sequence (captured into a graph by dgb_step):
// the stage kernels, plus the residual-norm kernel after the first stage.
// Traces rotate so a stage never writes the buffer it reads:
//   RK4      T0 -> T1 -> T0 -> T1 -> T0
//   TVD-RK3  T0 -> T1 -> T2 -> T0
// With ev != null, ev[i] is recorded before launch i and ev[nlaunch] after the
// last one (per-kernel timing by dgb_profile_step).  gauss: the Gauss-point
// form on d_V (vspace.cuh), else the nodal form on d_U.
// Pieces of the elements, [bound[c], bound[c+1]) (dgb_step_host): a step may
// run its first stage, or its last two, piece by piece so that host copies
// overlap the work.  deps[c] has bit c' set when an element of piece c has a
// neighbour in piece c' (bit c always); a stage's piece reads the previous
// stage's traces of exactly those pieces.
//   in(c)   enqueues what piece c's first-stage input needs (its copy in, its
//           basis change and traces); piece k of the first stage runs as soon
//           as in() has been enqueued for every piece in deps[k]
//   out(c)  is enqueued behind piece c of the last stage; the last two stages
//           run interleaved, piece k of the last one as soon as the one
//           before has run every piece in deps[k]
// The neighbour relation is symmetric, so a last-stage piece also runs only
// after every piece of the stage before that reads its traces: the trace
// buffer the last stage writes may be the one the stage before reads
// (RK4: T0), and no piece reads a trace after it was overwritten.
struct StepPieces {
  int n = 0;
  const long* bound = nullptr;
  const unsigned* deps = nullptr;
  const int* in_order = nullptr;  // the order of in() (null: 0, 1, ...)
  std::function<int(int)> in;   // set: the first stage in pieces
  std::function<int(int)> out;  // set: the last two stages in pieces
};
// Odd stages of a Gauss-point step take the elements in descending order:
// a stage then starts on the elements whose state, accumulator and traces the
// stage before wrote last, which the L2 still holds.  The order changes no
// result (every element's work is independent of it).
#ifndef DGB_ALT_ORDER
#define DGB_ALT_ORDER 1
#endif

int enqueue_step(dgb_handle* h, int scheme, double dt, cudaEvent_t* ev = nullptr, bool gauss = false,
                 const StepPieces* pieces = nullptr, long long* nl = nullptr)
{
  double* Ures = gauss ? h->d_V : h->d_U;
  const KLaunch L = klaunch(h);
  const int nst = scheme == DGB_RK4 ? 4 : 3;
  const int modes4[4] = {MODE_RK4_0, MODE_RK4_1, MODE_RK4_2, MODE_RK4_3};
  const int modes3[3] = {MODE_TVD_0, MODE_TVD_1, MODE_TVD_2};
  const int tin4[4] = {0, 1, 0, 1}, tout4[4] = {1, 0, 1, 0};
  const int tin3[3] = {0, 1, 2}, tout3[3] = {1, 2, 0};
  long long launched = 0;
  auto args = [&](int s) {
    StageArgs a = stage_args(scheme == DGB_RK4 ? modes4[s] : modes3[s], dt);
    a.Ubase = Ures;
    a.acc = h->d_acc;
    a.Uout = s == nst - 1 ? Ures : h->d_Us;
    a.part = s == 0 ? h->d_part : nullptr;
    a.flag = h->d_flag;
    a.Tnext = h->d_trace[scheme == DGB_RK4 ? tout4[s] : tout3[s]];
    a.rev = DGB_ALT_ORDER && gauss && (s & 1);
    return a;
  };
  auto stage_in = [&](int s) -> const double* { return s == 0 ? Ures : h->d_Us; };
  auto stage_tin = [&](int s) -> const void* { return h->d_trace[scheme == DGB_RK4 ? tin4[s] : tin3[s]]; };
  auto piece_launch = [&](int s, StageArgs a, int c) -> cudaError_t {  // piece c of stage s (none if empty)
    if (pieces->bound[c + 1] == pieces->bound[c]) return cudaSuccess;  // (an ecount of 0 would mean all elements)
    a.e0 = pieces->bound[c];
    a.ecount = pieces->bound[c + 1] - pieces->bound[c];
    ++launched;
    return launch_vstage(L, stage_in(s), stage_tin(s), a, h->stream);
  };
  const bool pieced = pieces && gauss;
  int k = 0;
  for (int s = 0; s < nst; ++s) {
    const StageArgs a = args(s);
    if (ev) CK(cudaEventRecord(ev[k++], h->stream));
    if (pieced && pieces->in && s == 0) {
      unsigned have = 0, done = 0;
      for (int i = 0; i < pieces->n; ++i) {
        const int c = pieces->in_order ? pieces->in_order[i] : i;
        if (const int rc = pieces->in(c)) return rc;
        have |= 1u << c;
        for (int q = 0; q < pieces->n; ++q) {
          if (((done >> q) & 1) || (pieces->deps[q] & ~have)) continue;
          done |= 1u << q;
          CK(piece_launch(s, a, q));
        }
      }
    } else if (pieced && pieces->out && s == nst - 2) {
      const StageArgs b = args(s + 1);
      unsigned have = 0, done = 0;
      for (int c = 0; c < pieces->n; ++c) {
        CK(piece_launch(s, a, c));
        have |= 1u << c;
        for (int q = 0; q < pieces->n; ++q) {
          if (((done >> q) & 1) || (pieces->deps[q] & ~have)) continue;
          done |= 1u << q;
          CK(piece_launch(s + 1, b, q));
          if (const int rc = pieces->out(q)) return rc;
        }
      }
      ++s;  // the last stage ran with this one
    } else {
      ++launched;
      if (gauss)
        CK(launch_vstage(L, stage_in(s), stage_tin(s), a, h->stream));
      else
        CK(launch_stage(L, stage_in(s), stage_tin(s), a, h->stream));
    }
    if (s == 0) {
      if (ev) CK(cudaEventRecord(ev[k++], h->stream));
      ++launched;
      CK(launch_norm(h->E, h->d_part, 1.0 / (double)h->n, h->d_norms, (long)h->norms_cap, h->d_counter,
                     h->d_flag, h->stream));
    }
  }
  if (ev) CK(cudaEventRecord(ev[k++], h->stream));
  if (nl) *nl += launched;
  return DGB_OK;
}

long long launches_per_step(const dgb_handle*, int scheme) { return (scheme == DGB_RK4 ? 4 : 3) + 1; }

void free_all(dgb_handle* h)
{
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  if (h->copy_out) cudaStreamSynchronize(h->copy_out);
  drop_step_graphs(h);
  void* ptrs[] = {h->d_ops, h->d_opsf, h->d_geo, h->d_gv, h->d_gf, h->d_nbr, h->d_wallf, h->d_mean, h->d_U, h->d_V, h->d_Us, h->d_acc, h->d_trace[0],
                  h->d_trace[1], h->d_trace[2], h->d_in, h->d_f, h->d_R, h->d_part, h->d_norms,
                  h->d_counter, h->d_flag, h->d_out, h->d_hnorms};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  free_adjoint(h);
  for (cudaEvent_t e : h->host_events) cudaEventDestroy(e);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->copy_out) cudaStreamDestroy(h->copy_out);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace

int dgb::set_last_error(int code, const std::string& msg) { return fail(code, msg); }

DevParams dgb::device_params(const dgb_params& p, double prandtl, double twall)
{
  DevParams d{};
  d.gamma = p.gamma;
  d.R = p.R;
  d.mu = p.mu;
  d.P = p.P;
  d.eta = p.eta;
  total_conditions(p, &d.Tt, &d.Pt);
  for (int r = 0; r < 5; ++r) {
    d.Ufr[r] = p.Ufr[r];
    d.src[r] = p.source[r];
  }
  d.kq = (prandtl == 0. || std::isinf(prandtl)) ? 0. : p.mu * p.gamma / prandtl;
  d.Tw = twall < 0. ? p.T : twall;
  return d;
}

namespace {

// a new DevParams for the handle: captured graphs hold the kernel parameters
// by value, and a recorded forward run was made with the old ones
int replace_device_params(dgb_handle* h, const DevParams& d)
{
  if (!std::memcmp(&d, &h->dprm, sizeof d)) return DGB_OK;
  if (h->tc_step && d.kq != 0.)
    return fail(DGB_ERR_UNSUPPORTED, "the tensor-core step form has no heat flux: select another form first");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  h->dprm = d;
  drop_step_graphs(h);
  if (h->rev_graph) cudaGraphExecDestroy(h->rev_graph);
  h->rev_graph = nullptr;
  h->rev_scheme = -1;
  h->recorded = false;
  return DGB_OK;
}

}  // namespace

void dgb::drop_step_graphs(dgb_handle* h)
{
  for (dgb_handle::StepGraph* g : {&h->graph, &h->ggraph}) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    g->exec = nullptr;
    g->scheme = -1;
  }
}

// The captured graph of one step for (scheme, dt) in the nodal or the
// Gauss-point form, with room for `cap` norms.
int dgb::ensure_step_graph(dgb_handle* h, int scheme, double dt, unsigned long long cap, bool gauss)
{
  if (cap > h->norms_cap) {
    if (h->d_norms) CK(cudaFree(h->d_norms));
    h->d_norms = nullptr;
    CK(cudaMalloc(&h->d_norms, sizeof(double) * cap));
    h->norms_cap = cap;
    drop_step_graphs(h);  // the captured graphs hold the old norms pointer and capacity
  }
  dgb_handle::StepGraph& sg = gauss ? h->ggraph : h->graph;
  if (sg.exec && sg.scheme == scheme && sg.dt == dt) return DGB_OK;
  if (sg.exec) cudaGraphExecDestroy(sg.exec);
  sg.exec = nullptr;
  sg.scheme = -1;
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(h, scheme, dt, nullptr, gauss);
  cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
  if (rc) {
    if (ce == cudaSuccess) cudaGraphDestroy(g);
    return rc;
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
  ce = cudaGraphInstantiate(&sg.exec, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
  sg.scheme = scheme;
  sg.dt = dt;
  h->launches_per_step = launches_per_step(h, scheme);
  return DGB_OK;
}

// k replays of the step graph of the form; with initial_trace the face
// traces of the resident state (d_U, or d_V in the Gauss-point form) are
// computed first (otherwise the last step's epilogue left them in trace
// buffer 0).  Norms go to d_norms[*d_counter ...].
int dgb::enqueue_steps(dgb_handle* h, unsigned long long k, bool initial_trace, bool gauss)
{
  if (initial_trace) {
    int rc = enqueue_initial_traces(h, gauss);
    if (rc) return rc;
  }
  cudaGraphExec_t g = gauss ? h->ggraph.exec : h->graph.exec;
  for (unsigned long long s = 0; s < k; ++s) CK(cudaGraphLaunch(g, h->stream));
  return DGB_OK;
}

extern "C" {

const char* dgb_error_string(int status)
{
  switch (status) {
    case DGB_OK: return "ok";
    case DGB_ERR_ARG: return "invalid argument";
    case DGB_ERR_UNSUPPORTED: return "unsupported input";
    case DGB_ERR_CUDA: return "CUDA error";
    case DGB_ERR_GEOMETRY: return "invalid geometry";
    case DGB_ERR_NONFINITE: return "non-finite residual";
    case DGB_ERR_IO: return "i/o error";
    case DGB_ERR_BOUNDARY: return "no subsonic inflow boundary Mach root";
  }
  return "unknown status";
}

const char* dgb_last_error_message(void) { return g_err.c_str(); }

int dgb_create(const dgb_mesh_desc* mesh, const dgb_params* params, int precision, dgb_handle** out)
{
  if (!mesh || !params || !out) return fail(DGB_ERR_ARG, "null argument");
  *out = nullptr;
  if (precision != DGB_FP64 && precision != DGB_MIXED_FP32) return fail(DGB_ERR_ARG, "unknown precision");
  dgb_handle* h = new dgb_handle();
  h->nx = mesh->nx;
  h->ny = mesh->ny;
  h->nz = mesh->nz;
  h->p = mesh->p;
  h->q = mesh->q;
  h->precision = precision;
  h->prm = *params;
  for (int i = 0; i < 6; ++i) h->bounds[i] = mesh->bounds[i];
  int rc = build_ops(mesh->p, h->ops);
  if (rc) {
    delete h;
    return fail(rc, "solution order outside 0..6");
  }
  h->P = h->ops.P;
  h->NB = h->P * h->P * h->P;
  h->NQF = h->P * h->P;
  h->E = (long)mesh->nx * mesh->ny * mesh->nz;
  h->n = (long long)h->E * 5 * h->NB;
  std::vector<int32_t> nbr;
  std::string why;
  rc = check_mesh(*mesh, why);
  if (rc) {
    delete h;
    return fail(rc, why);
  }
  build_neighbours(*mesh, nbr);
  h->dprm = device_params(*params, 0., -1.);
  for (int s = 0; s < 6; ++s) h->isothermal = h->isothermal || mesh->bounds[s] == DGB_BT_ISOTHERMAL_WALL;

  cudaError_t e = cudaGetDevice(&h->device);
  if (e != cudaSuccess) {
    delete h;
    return cuda_fail(e, "cudaGetDevice");
  }
#define CKF(call)                        \
  do {                                   \
    cudaError_t e_ = (call);             \
    if (e_ != cudaSuccess) {             \
      int rc_ = cuda_fail(e_, #call);    \
      free_all(h);                       \
      delete h;                          \
      return rc_;                        \
    }                                    \
  } while (0)
  CKF(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  h->own_stream = true;
  std::vector<double> table(ops_table_size(h->P));
  pack_ops(h->ops, table.data());
  const size_t sb = sizeof(double) * (size_t)h->n;
  CKF(cudaMalloc(&h->d_ops, sizeof(double) * table.size()));
  CKF(cudaMalloc(&h->d_geo, sizeof(double) * (size_t)h->E * kGeoStride));
  CKF(cudaMalloc(&h->d_nbr, sizeof(int) * nbr.size()));
  CKF(cudaMalloc(&h->d_U, sb));
  CKF(cudaMalloc(&h->d_V, sb));
  CKF(cudaMalloc(&h->d_Us, sb));
  CKF(cudaMalloc(&h->d_acc, sb));
  for (int t = 0; t < 3; ++t)
    CKF(cudaMalloc(&h->d_trace[t], trace_elem_bytes(precision) * (size_t)h->E * 60 * h->NQF));
  CKF(cudaMalloc(&h->d_part, sizeof(double) * (size_t)h->E));
  CKF(cudaMalloc(&h->d_counter, sizeof(int)));
  CKF(cudaMalloc(&h->d_flag, sizeof(int)));
  CKF(cudaMemcpy(h->d_ops, table.data(), sizeof(double) * table.size(), cudaMemcpyHostToDevice));
  CKF(cudaMemcpy(h->d_nbr, nbr.data(), sizeof(int) * nbr.size(), cudaMemcpyHostToDevice));
  {  // the isothermal-wall faces, for the dJ/dTw sum of the adjoint
    std::vector<int> wf;
    for (size_t i = 0; i < nbr.size(); ++i)
      if (nbr[i] == DGB_BT_ISOTHERMAL_WALL) wf.push_back((int)i);
    h->n_wallf = (long)wf.size();
    if (!wf.empty()) {
      CKF(cudaMalloc(&h->d_wallf, sizeof(int) * wf.size()));
      CKF(cudaMemcpy(h->d_wallf, wf.data(), sizeof(int) * wf.size(), cudaMemcpyHostToDevice));
    }
  }
  // element geometry, built on the device (geometry.cu)
  const auto g0 = std::chrono::steady_clock::now();
  rc = build_geometry_device(*mesh, h->ops, nbr, h->d_nbr, h->stream, h->d_geo, &h->d_gv, &h->d_gf, h->curved, why);
  h->geometry_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - g0).count();
  if (rc) {
    fail(rc, why);
    free_all(h);
    delete h;
    return rc;
  }
  CKF(cudaMemset(h->d_U, 0, sb));
  CKF(cudaMemset(h->d_counter, 0, sizeof(int)));
  CKF(cudaMemset(h->d_flag, 0, sizeof(int)));
  if (precision == DGB_MIXED_FP32) {
    std::vector<float> tf(table.begin(), table.end());
    CKF(cudaMalloc(&h->d_opsf, sizeof(float) * tf.size()));
    CKF(cudaMemcpy(h->d_opsf, tf.data(), sizeof(float) * tf.size(), cudaMemcpyHostToDevice));
  }
  CKF(prepare_kernels(h->P, precision));
  CKF(prepare_gauss(h->P, precision));
#undef CKF
  *out = h;
  return DGB_OK;
}

int dgb_get_geometry(dgb_handle* h, int part, double* out, size_t count)
{
  if (!h || !out) return fail(DGB_ERR_ARG, "null argument");
  const double* src = part == DGB_GEO_ELEMENT ? h->d_geo : part == DGB_GEO_VOLUME ? h->d_gv
                      : part == DGB_GEO_FACE  ? h->d_gf
                                              : nullptr;
  const size_t n = part == DGB_GEO_ELEMENT  ? (size_t)h->E * kGeoStride
                   : part == DGB_GEO_VOLUME ? (size_t)h->E * kVolC * h->NB
                                            : (size_t)h->E * 6 * kFaceC * h->NQF;
  if (part < DGB_GEO_ELEMENT || part > DGB_GEO_FACE) return fail(DGB_ERR_ARG, "unknown geometry part");
  if (!src) return fail(DGB_ERR_ARG, "per-point geometry exists only for curved meshes");
  if (count != n) return fail(DGB_ERR_ARG, "count does not match the geometry part's size");
  cudaSetDevice(h->device);
  CK(cudaMemcpyAsync(out, src, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DGB_OK;
}

int dgb_geometry_stats(const dgb_handle* h, int* curved, double* build_seconds)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (curved) *curved = h->curved ? 1 : 0;
  if (build_seconds) *build_seconds = h->geometry_s;
  return DGB_OK;
}

int dgb_destroy(dgb_handle* h)
{
  if (!h) return DGB_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return DGB_OK;
}

int dgb_set_stream(dgb_handle* h, void* stream)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (h->host_pipe) {  // the copies of unsynchronized dgb_step_host_async calls
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    if (h->copy_out) cudaStreamSynchronize(h->copy_out);
  }
  if (h->own_stream && h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  h->own_stream = false;
  h->stream = (cudaStream_t)stream;
  if (!h->stream) {  // graphs need a capturable stream: make our own
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  drop_step_graphs(h);
  return DGB_OK;
}

int dgb_set_prandtl(dgb_handle* h, double prandtl)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (!(prandtl >= 0.)) return fail(DGB_ERR_ARG, "Prandtl number must be >= 0 (0: no heat flux)");
  const int rc = replace_device_params(h, device_params(h->prm, prandtl, h->twall));
  if (rc == DGB_OK) h->prandtl = prandtl;
  return rc;
}

int dgb_set_wall_temperature(dgb_handle* h, double Tw)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (!(Tw > 0.) || std::isinf(Tw)) return fail(DGB_ERR_ARG, "wall temperature must be finite and > 0");
  const int rc = replace_device_params(h, device_params(h->prm, h->prandtl, Tw));
  if (rc == DGB_OK) h->twall = Tw;
  return rc;
}

int dgb_set_params(dgb_handle* h, const dgb_params* params)
{
  if (!h || !params) return fail(DGB_ERR_ARG, "null argument");
  const int rc = replace_device_params(h, device_params(*params, h->prandtl, h->twall));
  if (rc == DGB_OK) h->prm = *params;
  return rc;
}

int dgb_synchronize(dgb_handle* h)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  if (h->copy_stream) CK(cudaStreamSynchronize(h->copy_stream));
  if (h->copy_out) CK(cudaStreamSynchronize(h->copy_out));
  if (!h->host_pipe) return DGB_OK;
  h->host_pipe = false;  // the status of the dgb_step_host_async calls since the last synchronization
  int flag = 0;
  CK(cudaMemcpy(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag & 1) return fail(DGB_ERR_NONFINITE, "residual norm became NaN/Inf");
  if (flag & 16) return fail(DGB_ERR_CUDA, "tensor-core stage: a wait for the tensor cores gave up");
  if (flag & 2) return fail(DGB_ERR_BOUNDARY, "subsonic inflow without a non-negative Mach root");
  return DGB_OK;
}

long long dgb_state_size(const dgb_handle* h) { return h ? h->n : -1; }

long long dgb_last_launch_count(const dgb_handle* h) { return h ? h->last_launches : -1; }

int dgb_set_state(dgb_handle* h, const double* U_host)
{
  if (!h || !U_host) return fail(DGB_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->d_U, U_host, sizeof(double) * (size_t)h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->v_current = false;
  return DGB_OK;
}

int dgb_get_state(dgb_handle* h, double* U_host)
{
  if (!h || !U_host) return fail(DGB_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(U_host, h->d_U, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DGB_OK;
}

int dgb_set_state_device(dgb_handle* h, const double* U_dev)
{
  if (!h || !U_dev) return fail(DGB_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->d_U, U_dev, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->v_current = false;
  return DGB_OK;
}

int dgb_get_state_device(dgb_handle* h, double* U_dev)
{
  if (!h || !U_dev) return fail(DGB_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(U_dev, h->d_U, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DGB_OK;
}

int dgb_mean_update(dgb_handle* h, unsigned long long tstep, unsigned long long mean_start)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (tstep < mean_start) return fail(DGB_ERR_ARG, "tstep before mean_start");
  CK(cudaSetDevice(h->device));
  if (!h->d_mean) {  // a mean that was never set starts from zero
    CK(cudaMalloc(&h->d_mean, sizeof(double) * (size_t)h->n));
    CK(cudaMemsetAsync(h->d_mean, 0, sizeof(double) * (size_t)h->n, h->stream));
  }
  const double old_w = (double)(tstep - mean_start), new_w = (double)(tstep + 1 - mean_start);
  CK(launch_mean_update((long)h->n, h->d_mean, h->d_U, old_w, new_w, tstep == mean_start ? 1 : 0, h->stream));
  return DGB_OK;
}

int dgb_set_mean(dgb_handle* h, const double* mean_host)
{
  if (!h || !mean_host) return fail(DGB_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  if (!h->d_mean) CK(cudaMalloc(&h->d_mean, sizeof(double) * (size_t)h->n));
  CK(cudaMemcpyAsync(h->d_mean, mean_host, sizeof(double) * (size_t)h->n, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DGB_OK;
}

int dgb_get_mean(dgb_handle* h, double* mean_host)
{
  if (!h || !mean_host) return fail(DGB_ERR_ARG, "null argument");
  if (!h->d_mean) return fail(DGB_ERR_ARG, "no running mean (dgb_mean_update / dgb_set_mean)");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(mean_host, h->d_mean, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DGB_OK;
}

int dgb_state_device_ptr(dgb_handle* h, double** U_dev)
{
  if (!h || !U_dev) return fail(DGB_ERR_ARG, "null argument");
  *U_dev = h->d_U;
  h->v_current = false;  // the caller may write through it before the next dgb_step
  return DGB_OK;
}

int dgb_set_step_form(dgb_handle* h, int form)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (form != DGB_STEP_GAUSS && form != DGB_STEP_NODAL && form != DGB_STEP_GAUSS_TC)
    return fail(DGB_ERR_ARG, "unknown step form");
  const bool tc = form == DGB_STEP_GAUSS_TC;
  if (tc) {
    if (h->precision != DGB_MIXED_FP32 || !tc_supported(h->P) || h->d_gv || h->dprm.kq != 0.)
      return fail(DGB_ERR_UNSUPPORTED, "tensor-core stage: mixed precision, p = 3 or 4, affine, no heat flux only");
    CK(cudaSetDevice(h->device));
    CK(vprepare_tc(h->P));
  }
  if (tc != h->tc_step) {  // the captured graphs hold the other stage kernel
    CK(cudaStreamSynchronize(h->stream));
    drop_step_graphs(h);
    if (h->rev_graph) cudaGraphExecDestroy(h->rev_graph);
    h->rev_graph = nullptr;
    h->rev_scheme = -1;
  }
  h->gauss_step = form != DGB_STEP_NODAL;
  h->tc_step = tc;
  h->v_current = false;
  return DGB_OK;
}

int dgb_residual_device(dgb_handle* h, const double* U_dev, double* R_dev, double* f_dev)
{
  if (!h || !U_dev || !f_dev) return fail(DGB_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  int rc = enqueue_residual(h, U_dev, R_dev, f_dev);
  h->last_launches = 2;
  return rc;
}

int dgb_residual(dgb_handle* h, const double* U_host, double* R_host, double* f_host)
{
  if (!h || !U_host || !f_host) return fail(DGB_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  const size_t sb = sizeof(double) * (size_t)h->n;
  if (!h->d_in) {
    CK(cudaMalloc(&h->d_in, sb));
    CK(cudaMalloc(&h->d_f, sb));
    CK(cudaMalloc(&h->d_R, sb));
  }
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  CK(cudaMemcpyAsync(h->d_in, U_host, sb, cudaMemcpyHostToDevice, h->stream));
  int rc = enqueue_residual(h, h->d_in, h->d_R, h->d_f);
  if (rc) return rc;
  h->last_launches = 2;
  CK(cudaMemcpyAsync(f_host, h->d_f, sb, cudaMemcpyDeviceToHost, h->stream));
  if (R_host) CK(cudaMemcpyAsync(R_host, h->d_R, sb, cudaMemcpyDeviceToHost, h->stream));
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag & 2) return fail(DGB_ERR_BOUNDARY, "subsonic inflow without a non-negative Mach root");
  return DGB_OK;
}

int dgb_step(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, double* norms_host)
{
  if (!h) return fail(DGB_ERR_ARG, "null handle");
  if (scheme != DGB_RK4 && scheme != DGB_TVDRK3) return fail(DGB_ERR_ARG, "unknown time scheme");
  if (!(dt == dt)) return fail(DGB_ERR_ARG, "dt is NaN");
  CK(cudaSetDevice(h->device));
  if (nsteps == 0) return DGB_OK;
  const bool gauss = h->gauss_step;
  int rc = ensure_step_graph(h, scheme, dt, nsteps, gauss);
  if (rc) return rc;
  CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  const KLaunch L = klaunch(h);
  const bool convert_in = gauss && !h->v_current;
  if (convert_in) CK(launch_gauss_basis(L, h->d_U, h->d_V, true, h->stream));
  if ((rc = enqueue_steps(h, nsteps, true, gauss))) return rc;
  if (gauss) CK(launch_gauss_basis(L, h->d_V, h->d_U, false, h->stream));
  h->v_current = gauss;
  h->last_launches = 1 + (long long)nsteps * h->launches_per_step + (convert_in ? 1 : 0) + (gauss ? 1 : 0);
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (norms_host)
    CK(cudaMemcpyAsync(norms_host, h->d_norms, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag & 1) return fail(DGB_ERR_NONFINITE, "residual norm became NaN/Inf");
  if (flag & 16) return fail(DGB_ERR_CUDA, "tensor-core stage: a wait for the tensor cores gave up");
  if (flag & 2) return fail(DGB_ERR_BOUNDARY, "subsonic inflow without a non-negative Mach root");
  return DGB_OK;
}

namespace {

__global__ void set_int_kernel(int* p, int v) { *p = v; }

__global__ void copy_doubles_kernel(const double* __restrict__ src, double* __restrict__ dst, long n)
{
  for (long i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// dgb_step_host and dgb_step_host_async.  Asynchronous calls return once the
// work is queued: a call's copy of piece c in waits for the handle's earlier
// work on its stream (the previous call's stepping included) and for the
// previous call's copy of piece c out (U_in may be that call's U_out), but
// not for its other copies out, which read d_out: consecutive calls overlap
// the copies out of one with the copies in of the next.
int step_host(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, const double* U_in, double* U_out,
              double* norms_host, bool async)
{
  if (!h || !U_in || !U_out) return fail(DGB_ERR_ARG, "null argument");
  if (scheme != DGB_RK4 && scheme != DGB_TVDRK3) return fail(DGB_ERR_ARG, "unknown time scheme");
  if (!(dt == dt)) return fail(DGB_ERR_ARG, "dt is NaN");
  CK(cudaSetDevice(h->device));
  int rc;
  if (nsteps == 0 || !h->gauss_step) {  // nothing to overlap: the plain calls
    if (h->host_pipe && (rc = dgb_synchronize(h))) return rc;
    if ((rc = dgb_set_state(h, U_in))) return rc;
    if (nsteps && (rc = dgb_step(h, scheme, dt, nsteps, norms_host))) return rc;
    return dgb_get_state(h, U_out);
  }
  if (!h->d_out) CK(cudaMalloc(&h->d_out, sizeof(double) * (size_t)h->n));
  // pieces of elements with even boundaries (the paired kernels take
  // elements two by two), and which pieces each one's neighbours lie in.
  // 8 pieces measured best for pipelined calls on the 32^3 TGV (1.09e10
  // DOF-updates/s against 1.08 with 6 and 12, 1.04 with 16; one call at a
  // time prefers 12: 1.02e10 against 1.00 with 8)
  constexpr int K = 8;
  long bound[K + 1];
  for (int c = 0; c <= K; ++c) bound[c] = (h->E * c / K) & ~1L;
  bound[K] = h->E;
  if ((long)h->piece_deps.size() != K || h->piece_deps_E != h->E) {
    std::vector<int> nb((size_t)h->E * 6);
    CK(cudaMemcpyAsync(nb.data(), h->d_nbr, sizeof(int) * nb.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->piece_deps.assign(K, 0u);
    for (int c = 0; c < K; ++c) {
      h->piece_deps[c] |= 1u << c;
      for (long e = bound[c]; e < bound[c + 1]; ++e)
        for (int f = 0; f < 6; ++f) {
          const long m = nb[(size_t)e * 6 + f];
          if (m < 0) continue;
          int q = 0;
          while (m >= bound[q + 1]) ++q;
          h->piece_deps[c] |= 1u << q;
        }
    }
    // the order in which the interleaved last two stages release pieces
    // (out), which the copies in follow: a call's copy in of a piece waits
    // for the previous call's copy out of it
    h->piece_order.clear();
    unsigned have = 0, done = 0;
    for (int c = 0; c < K; ++c) {
      have |= 1u << c;
      for (int q = 0; q < K; ++q)
        if (!((done >> q) & 1) && !(h->piece_deps[q] & ~have)) {
          done |= 1u << q;
          h->piece_order.push_back(q);
        }
    }
    h->piece_deps_E = h->E;
  }
  if (!h->copy_stream) CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  if (!h->copy_out) CK(cudaStreamCreateWithFlags(&h->copy_out, cudaStreamNonBlocking));
  while (h->host_events.size() < 3 * K + 2) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    h->host_events.push_back(e);
  }
  cudaEvent_t* ev_in = h->host_events.data();  // piece c landed
  cudaEvent_t* ev_out = ev_in + K;              // piece c's nodal state is in d_out
  cudaEvent_t* ev_done = ev_in + 2 * K;         // piece c copied out (the last call's)
  cudaEvent_t ev_start = ev_in[3 * K];  // (and ev_in[3 K + 1]: the call's norms are staged)
  if ((rc = ensure_step_graph(h, scheme, dt, nsteps, true))) return rc;
  // the call's norms are staged in one half of d_hnorms (alternating between
  // calls) for their copy out, so later work may write d_norms at once
  if (norms_host && h->hnorms_cap < nsteps) {
    CK(cudaStreamSynchronize(h->stream));
    if (h->copy_out) CK(cudaStreamSynchronize(h->copy_out));
    if (h->d_hnorms) CK(cudaFree(h->d_hnorms));
    h->d_hnorms = nullptr;
    CK(cudaMalloc(&h->d_hnorms, sizeof(double) * 2 * nsteps));
    h->hnorms_cap = nsteps;
  }
  set_int_kernel<<<1, 1, 0, h->stream>>>(h->d_counter, 0);  // (a kernel: a memset may queue behind copies)
  CK(cudaGetLastError());
  if (!h->host_pipe)  // (else the status of the unsynchronized calls keeps accumulating)
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  // the copies in start once the handle's earlier work is done with d_U
  CK(cudaEventRecord(ev_start, h->stream));
  CK(cudaStreamWaitEvent(h->copy_stream, ev_start, 0));
  const KLaunch L = klaunch(h);
  const long nbv = 5L * h->NB;  // values per element of a state
  const size_t tb = trace_elem_bytes(h->precision);
  auto piece = [&](long e0, long e1) {  // the launch description of elements [e0, e1): own data only
    KLaunch Lc = L;
    Lc.E = e1 - e0;
    Lc.geo = L.geo + e0 * kGeoStride;
    Lc.gv = L.gv ? L.gv + e0 * (long)kVolC * h->NB : nullptr;
    Lc.gf = L.gf ? L.gf + e0 * 6L * kFaceC * h->NQF : nullptr;
    return Lc;
  };
  long long nl = 1;  // the norm counter set above
  StepPieces sp;
  sp.n = K;
  sp.bound = bound;
  sp.deps = h->piece_deps.data();
  sp.in_order = h->piece_order.data();
  // in: each piece's copy, then its basis change and face traces (element-local work)
  auto in = [&](int c) -> int {
    const long e0 = bound[c], e1 = bound[c + 1];
    if (e1 == e0) return DGB_OK;
    // U_in may be the previous call's U_out: its piece is read once written
    CK(cudaStreamWaitEvent(h->copy_stream, ev_done[c], 0));
    CK(cudaMemcpyAsync(h->d_U + e0 * nbv, U_in + e0 * nbv, sizeof(double) * (size_t)(e1 - e0) * nbv,
                       cudaMemcpyHostToDevice, h->copy_stream));
    CK(cudaEventRecord(ev_in[c], h->copy_stream));
    CK(cudaStreamWaitEvent(h->stream, ev_in[c], 0));
    const KLaunch Lc = piece(e0, e1);
    CK(launch_gauss_basis(Lc, h->d_U + e0 * nbv, h->d_V + e0 * nbv, true, h->stream));
    CK(launch_vtrace(Lc, h->d_V + e0 * nbv, static_cast<char*>(h->d_trace[0]) + (size_t)e0 * 60 * h->NQF * tb,
                     h->stream));
    nl += 2;
    return DGB_OK;
  };
  // out: behind each piece of the last stage of the last step, that piece
  // changed back to nodal values into d_out (once the previous call has copied
  // its piece out) and copied out while the next ones compute; d_U gets the
  // nodal state too, as after dgb_step
  auto out = [&](int c) -> int {
    const long e0 = bound[c], e1 = bound[c + 1];
    if (e1 == e0) return DGB_OK;
    const size_t bytes = sizeof(double) * (size_t)(e1 - e0) * nbv;
    CK(cudaStreamWaitEvent(h->stream, ev_done[c], 0));
    CK(launch_gauss_basis(piece(e0, e1), h->d_V + e0 * nbv, h->d_out + e0 * nbv, false, h->stream,
                          h->d_U + e0 * nbv));
    ++nl;
    CK(cudaEventRecord(ev_out[c], h->stream));
    CK(cudaStreamWaitEvent(h->copy_out, ev_out[c], 0));
    CK(cudaMemcpyAsync(U_out + e0 * nbv, h->d_out + e0 * nbv, bytes, cudaMemcpyDeviceToHost, h->copy_out));
    CK(cudaEventRecord(ev_done[c], h->copy_out));
    return DGB_OK;
  };
  sp.in = in;
  if (nsteps == 1) {
    sp.out = out;
    if ((rc = enqueue_step(h, scheme, dt, nullptr, true, &sp, &nl))) return rc;
  } else {
    if ((rc = enqueue_step(h, scheme, dt, nullptr, true, &sp, &nl))) return rc;
    for (unsigned long long s = 0; s + 2 < nsteps; ++s) CK(cudaGraphLaunch(h->ggraph.exec, h->stream));
    nl += (long long)(nsteps - 2) * h->launches_per_step;
    StepPieces last = sp;
    last.in = nullptr;
    last.out = out;
    if ((rc = enqueue_step(h, scheme, dt, nullptr, true, &last, &nl))) return rc;
  }
  h->v_current = true;
  h->last_launches = nl;
  // the norms go out behind the state, from their staging half: a copy out
  // on the handle's stream would queue behind the state's copies out and
  // hold up the next call's start
  if (norms_host) {
    h->norm_half ^= 1;
    double* stage = h->d_hnorms + (h->norm_half ? h->hnorms_cap : 0);
    copy_doubles_kernel<<<1, 256, 0, h->stream>>>(h->d_norms, stage, (long)nsteps);
    CK(cudaGetLastError());
    ++nl;
    cudaEvent_t ev_norms = ev_in[3 * K + 1];
    CK(cudaEventRecord(ev_norms, h->stream));
    CK(cudaStreamWaitEvent(h->copy_out, ev_norms, 0));
    CK(cudaMemcpyAsync(norms_host, stage, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, h->copy_out));
  }
  h->host_pipe = true;
  return async ? DGB_OK : dgb_synchronize(h);
}

}  // namespace

int dgb_step_host(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, const double* U_in,
                  double* U_out, double* norms_host)
{
  return step_host(h, scheme, dt, nsteps, U_in, U_out, norms_host, false);
}

int dgb_step_host_async(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, const double* U_in,
                        double* U_out, double* norms_host)
{
  return step_host(h, scheme, dt, nsteps, U_in, U_out, norms_host, true);
}

int dgb_profile_step(dgb_handle* h, int scheme, double dt, int reps, double* ms_out, int* nk)
{
  if (!h || !nk || reps < 1) return fail(DGB_ERR_ARG, "bad argument");
  if (scheme != DGB_RK4 && scheme != DGB_TVDRK3) return fail(DGB_ERR_ARG, "unknown time scheme");
  CK(cudaSetDevice(h->device));
  // launch 0 is the initial trace kernel, then one step's launches
  const int nl = 1 + (int)launches_per_step(h, scheme);
  if (*nk < nl || !ms_out) {
    *nk = nl;
    return fail(DGB_ERR_ARG, "ms_out too small");
  }
  *nk = nl;
  if (h->norms_cap < 1) {
    CK(cudaMalloc(&h->d_norms, sizeof(double)));
    h->norms_cap = 1;
  }
  std::vector<cudaEvent_t> ev((size_t)reps * (nl + 1));
  for (auto& e : ev) CK(cudaEventCreate(&e));
  int rc = DGB_OK;
  const bool gauss = h->gauss_step;  // the form dgb_step runs
  if (gauss && !h->v_current) CK(launch_gauss_basis(klaunch(h), h->d_U, h->d_V, true, h->stream));
  for (int r = 0; r < reps && rc == DGB_OK; ++r) {
    cudaEvent_t* er = &ev[(size_t)r * (nl + 1)];
    CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
    CK(cudaEventRecord(er[0], h->stream));
    rc = enqueue_initial_traces(h, gauss);
    if (rc == DGB_OK) rc = enqueue_step(h, scheme, dt, er + 1, gauss);
  }
  if (gauss && rc == DGB_OK) {
    CK(launch_gauss_basis(klaunch(h), h->d_V, h->d_U, false, h->stream));
    h->v_current = true;
  }
  CK(cudaStreamSynchronize(h->stream));
  for (int k = 0; k < nl; ++k) ms_out[k] = 0.;
  for (int r = 0; r < reps && rc == DGB_OK; ++r)
    for (int k = 0; k < nl; ++k) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev[(size_t)r * (nl + 1) + k], ev[(size_t)r * (nl + 1) + k + 1]));
      ms_out[k] += ms / reps;
    }
  for (auto& e : ev) cudaEventDestroy(e);
  h->last_launches = (long long)reps * nl;
  return rc;
}

// ------------------------------------------------------------ host helpers

int dgb_gauss_legendre(int n, double a, double b, double* x, double* w)
{
  if (n < 1 || !x || !w) return fail(DGB_ERR_ARG, "n must be >= 1");
  gauss_legendre(n, a, b, x, w);
  return DGB_OK;
}

int dgb_geometry_host(const dgb_mesh_desc* mesh, int* curved, double* geo, size_t ngeo, double* gv, size_t ngv,
                      double* gf, size_t ngf)
{
  if (!mesh) return fail(DGB_ERR_ARG, "null mesh");
  Ops1D ops;
  if (build_ops(mesh->p, ops)) return fail(DGB_ERR_UNSUPPORTED, "solution order outside 0..6");
  std::vector<double> g, v, f;
  std::vector<int32_t> nbr;
  std::string why;
  bool cv = false;
  const int rc = build_geometry(*mesh, ops, g, nbr, why, cv, v, f);
  if (rc) return fail(rc, why);
  const long E = (long)mesh->nx * mesh->ny * mesh->nz;
  const size_t NB = (size_t)ops.P * ops.P * ops.P, NQF = (size_t)ops.P * ops.P;
  if ((geo && ngeo != (size_t)E * kGeoStride) || (cv && gv && ngv != (size_t)E * kVolC * NB) ||
      (cv && gf && ngf != (size_t)E * 6 * kFaceC * NQF))
    return fail(DGB_ERR_ARG, "geometry output sizes do not match the mesh");
  if (curved) *curved = cv ? 1 : 0;
  if (geo) std::copy(g.begin(), g.end(), geo);
  if (cv && gv) std::copy(v.begin(), v.end(), gv);
  if (cv && gf) std::copy(f.begin(), f.end(), gf);
  return DGB_OK;
}

double dgb_lagrange1d(int i, int p, double x) { return lagrange1d(i, p, x); }
double dgb_lagrange1d_deriv(int i, int p, double x) { return lagrange1d_deriv(i, p, x); }

// generate_bump_nodes (geometry_common.cpp:494-576) for a single domain:
// box elements with optional tanh stretching in y, then the Gaussian bump
// that lifts the lower wall and relaxes linearly to the upper wall.
int dgb_bump_nodes(int nx, int ny, int nz, int q, double lx, double ly, double lz, double a,
                   double bh, double bc, double bv, double* nodes)
{
  if (nx <= 0 || ny <= 0 || nz <= 0 || q < 1 || !nodes) return fail(DGB_ERR_ARG, "bad mesh size");
  const int Q = q + 1;
  const double elx = lx / nx, ely = ly / ny, elz = lz / nz;
  const double nsx = elx / q, nsz = elz / q;
  for (int ez = 0; ez < nz; ++ez)
    for (int ey = 0; ey < ny; ++ey) {
      double esy, eey;
      if (a != 0.) {
        double xi = -1. + 2. * ((double)ey / ny);
        double y = 0.5 * std::tanh(xi * std::atanh(a));
        esy = ly * ((y * (2. / a) + 1.) / 2.);
        xi = -1. + 2. * ((double)(ey + 1.) / ny);
        y = 0.5 * std::tanh(xi * std::atanh(a));
        eey = ly * ((y * (2. / a) + 1.) / 2.);
      } else {
        esy = ey * ely;
        eey = (ey + 1.) * ely;
      }
      const double nsy = (eey - esy) / q;
      for (int ex = 0; ex < nx; ++ex) {
        const long e = ex + (long)nx * (ey + (long)ny * ez);
        for (int k = 0; k < Q; ++k)
          for (int j = 0; j < Q; ++j)
            for (int i = 0; i < Q; ++i) {
              double* x = nodes + 3 * (Q * Q * Q * e + i + Q * (j + Q * k));
              x[0] = ex * elx + nsx * i;
              x[1] = esy + nsy * j;
              x[2] = ez * elz + nsz * k;
              const double f = bh * std::exp(-((x[0] - bc) * (x[0] - bc)) / (2. * bv));
              x[1] = (x[1] / ly) * (ly - f) + f;
            }
      }
    }
  return DGB_OK;
}

int dgb_make_reference_state(double gamma, double gcnst, double mu, double c, double rho, double u,
                             double v, double w, double eta, const double* source, dgb_params* out)
{
  if (!out) return fail(DGB_ERR_ARG, "null output");
  const double P = c * c * (rho / gamma);
  out->gamma = gamma;
  out->R = gcnst;
  out->mu = mu;
  out->c = c;
  out->T = P / (rho * gcnst);
  out->P = P;
  out->eta = eta;
  out->Ufr[0] = rho;
  out->Ufr[1] = rho * u;
  out->Ufr[2] = rho * v;
  out->Ufr[3] = rho * w;
  out->Ufr[4] = P / (gamma - 1.) + 0.5 * rho * (u * u + v * v + w * w);
  for (int i = 0; i < 5; ++i) out->source[i] = source ? source[i] : 0.;
  return DGB_OK;
}

}  // extern "C"
