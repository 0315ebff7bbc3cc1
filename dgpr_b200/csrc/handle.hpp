// The solver handle behind the opaque dgb_handle of the C ABI, shared by the
// forward entry points (capi.cu) and the adjoint ones (adjoint_capi.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/dgb200.h"
#include "checkpoint.hpp"
#include "host.hpp"
#include "kernels.hpp"

struct dgb_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int nx = 0, ny = 0, nz = 0, p = 0, q = 0, P = 0, NB = 0, NQF = 0;
  long E = 0;
  long long n = 0;  // doubles per state array
  long long bounds[6] = {0, 0, 0, 0, 0, 0};
  int precision = DGB_FP64;
  dgb_params prm{};
  dgb::DevParams dprm{};
  double prandtl = 0.;  // heat flux off (0) or its Prandtl number (dgb_set_prandtl)
  double twall = -1.;   // isothermal-wall temperature (dgb_set_wall_temperature); < 0: the parameters' T
  bool isothermal = false;  // the mesh has isothermal-wall sides
  dgb::Ops1D ops;
  double* d_ops = nullptr;
  float* d_opsf = nullptr;    // operator table for the mixed form
  double* d_geo = nullptr;
  bool curved = false;         // per-point geometry (non-affine elements)
  double geometry_s = 0.;      // host wall time of the device geometry build in dgb_create
  double* d_gv = nullptr;      // [E][kVolC][P^3]
  double* d_gf = nullptr;      // [E][6][kFaceC][P^2]
  int* d_nbr = nullptr;
  int* d_wallf = nullptr;  // faces 6 e + lf on isothermal walls (btype -8), in element order
  long n_wallf = 0;
  double* d_U = nullptr;      // resident state
  double* d_Us = nullptr;     // stage state
  double* d_acc = nullptr;    // RK4 accumulator
  void* d_trace[3] = {nullptr, nullptr, nullptr};  // face traces (compute type), rotated between stages
  double* d_in = nullptr;     // residual API input / output
  double* d_f = nullptr;
  double* d_R = nullptr;
  double* d_part = nullptr;
  double* d_mean = nullptr;   // running mean of the state (dgb_mean_update)
  double* d_norms = nullptr;
  int* d_counter = nullptr;
  int* d_flag = nullptr;
  unsigned long long norms_cap = 0;
  // captured RK steps: nodal form (the recorded runs of the adjoint) and
  // Gauss-point form (dgb_step, vspace.cuh), each for one (scheme, dt)
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    int scheme = -1;
    double dt = 0.;
  };
  StepGraph graph, ggraph;
  bool gauss_step = true;    // dgb_step in the Gauss-point form (dgb_set_step_form)
  bool tc_step = false;      // ... with tensor-core volume contractions (mixed precision)
  double* d_V = nullptr;     // Gauss-point values of the state during dgb_step
  // d_V holds the state that d_U is the nodal image of (set by dgb_step,
  // cleared by everything that writes d_U otherwise): consecutive dgb_step
  // calls continue from d_V, so splitting a run into calls changes nothing
  bool v_current = false;
  long long launches_per_step = 0;
  long long last_launches = 0;
  // dgb_step_host: streams for the host copies in (copy_stream) and out
  // (copy_out), the events that order them against the pieces of work on the
  // handle's stream, and the nodal state the copies out read (d_out)
  cudaStream_t copy_stream = nullptr;
  cudaStream_t copy_out = nullptr;
  std::vector<cudaEvent_t> host_events;
  double* d_out = nullptr;
  bool host_pipe = false;  // dgb_step_host_async work not yet synchronized
  double* d_hnorms = nullptr;          // dgb_step_host's norms on their way out: 2 halves
  unsigned long long hnorms_cap = 0;   // doubles per half
  int norm_half = 0;                   // the half the last call staged
  std::vector<unsigned> piece_deps;  // per piece, the pieces its elements' neighbours lie in (bit mask)
  std::vector<int> piece_order;      // the order the interleaved last stages release the pieces
  long piece_deps_E = -1;

  // ---- adjoint (allocated on first use, adjoint_capi.cu)
  // state-sized buffers: stage states S0..S2, stage adjoints A0 A1, the
  // adjoint accumulator, the volume part of a VJP, the adjoint being carried
  // backwards, the state before the last recorded step and after it, and the
  // residual-VJP API's input / output
  enum { ADJ_S0, ADJ_S1, ADJ_S2, ADJ_A0, ADJ_A1, ADJ_ACC, ADJ_PART, ADJ_LAM, ADJ_WORK, ADJ_FINAL, ADJ_IN,
         ADJ_OUT, ADJ_NBUF };
  double* d_adj[ADJ_NBUF] = {};
  double* d_adj_tr = nullptr;  // FP64 face traces [E][6][10][NQF]
  double* d_adj_ta = nullptr;  // face-trace adjoints [E][6][20][NQF]
  double* d_pg = nullptr;      // parameter gradient scratch (adjoint_capi.cu, pgrad_doubles)
  std::vector<double*> d_slots;  // checkpoints
  double* d_stage_store = nullptr;  // recorded stage states [nsteps][stages - 1][n] (dgb_forward_record_stages)
  size_t stage_store_cap = 0;       // doubles
  bool rec_stages = false;          // the recorded run kept its stage states
  dgb::CheckpointPlan plan;    // the recorded forward's plan
  size_t plan_pos = 0;         // first op of the backward part
  bool recorded = false;
  bool slots_dirty = false;    // a backward sweep overwrote checkpoints of the recorded run
  int rec_scheme = DGB_RK4;
  double rec_dt = 0.;
  unsigned long long rec_steps = 0;
  cudaGraphExec_t rev_graph = nullptr;  // one reverse step of d_U with the adjoint in ADJ_LAM
  int rev_scheme = -1;
  double rev_dt = 0.;
  bool rev_gauss = false;  // the captured reverse step's form
  bool rec_gauss = false;  // the recorded run steps the Gauss-point form (on d_V)
  long long rev_launches = 0;
  long long adj_forward_steps = 0;  // steps recomputed by the last dgb_backward
  long long adj_reverse_steps = 0;
};

namespace dgb {

inline KLaunch klaunch(const dgb_handle* h)
{
  KLaunch L{};
  L.P = h->P;
  L.precision = h->precision;
  L.E = h->E;
  L.ops = h->precision == DGB_MIXED_FP32 ? (const void*)h->d_opsf : (const void*)h->d_ops;
  L.opsd = h->d_ops;
  L.geo = h->d_geo;
  L.gv = h->d_gv;
  L.gf = h->d_gf;
  L.nbr = h->d_nbr;
  L.prm = h->dprm;
  L.tc = h->tc_step && h->precision == DGB_MIXED_FP32;
  L.pair = h->E % 2 == 0 && !h->d_gv && !L.tc;
  return L;
}

inline StageArgs stage_args(int mode, double dt)
{
  StageArgs a;
  std::memset(&a, 0, sizeof a);
  a.mode = mode;
  a.dt = dt;
  return a;
}

inline int cuda_status(cudaError_t e, const char* what)
{
  return set_last_error(DGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void free_adjoint(dgb_handle* h);
// DevParams of the reference parameters, with the heat flux of Prandtl number
// `prandtl` (0: none) and isothermal walls at `twall` (< 0: p.T)
DevParams device_params(const dgb_params& p, double prandtl, double twall);
int ensure_step_graph(dgb_handle* h, int scheme, double dt, unsigned long long cap, bool gauss = false);
int enqueue_steps(dgb_handle* h, unsigned long long k, bool initial_trace, bool gauss = false);
void drop_step_graphs(dgb_handle* h);

}  // namespace dgb
