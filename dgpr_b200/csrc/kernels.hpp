// Launch interface between the C ABI (capi.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>

#include "host.hpp"
#include "physics.cuh"

namespace dgb {

// what the stage kernel does with f = -Minv R of its element
enum StageMode {
  MODE_RESIDUAL = 0,  // fout = f, Rout = R
  MODE_RK4_0,         // acc = f;          Uout = Ubase + dt f / 2
  MODE_RK4_1,         // acc += 2 f;       Uout = Ubase + dt f / 2
  MODE_RK4_2,         // acc += 2 f;       Uout = Ubase + dt f
  MODE_RK4_3,         // Uout = Ubase + dt/6 (acc + f)
  MODE_TVD_0,         // Uout = Ubase + dt f
  MODE_TVD_1,         // Uout = 3/4 Ubase + 1/4 Us + dt f / 4
  MODE_TVD_2          // Uout = 1/3 Ubase + 2/3 Us + 2/3 dt f
};

struct StageArgs {
  int mode;
  double dt;
  const double* Ubase;
  double* acc;
  double* Uout;
  double* fout;
  double* Rout;
  double* part;  // per-element sum of R^2 (stage 1 of a step), or null
  int* flag;     // bit 1: non-finite norm, bit 2: inflow without a Mach root
  void* Tnext;   // face traces of Uout for the next stage (compute type), or null
  // Gauss-point stage kernels only: elements [e0, e0 + ecount) (ecount 0: all;
  // both even for the paired kernel), so a stage can run in pieces whose
  // results are copied out while the next piece computes
  long e0, ecount;
  // Gauss-point stage kernels only: 1 takes the elements in descending order,
  // so a stage that follows an ascending one first reads what the L2 still
  // holds of the previous stage's writes
  int rev;
  // set by the launcher from e0, ecount and rev (element_order): CTA b takes
  // element (or, in the paired kernel, pair) ebase + estep * b
  long ebase, estep;
};

// The CTA-to-element map of a Gauss-point stage launch over units of `unit`
// elements (1, or 2 for the paired kernel).
inline StageArgs element_order(StageArgs sa, long E, long unit)
{
  const long cnt = (sa.ecount ? sa.ecount : E) / unit, first = sa.e0 / unit;
  sa.ebase = sa.rev ? first + cnt - 1 : first;
  sa.estep = sa.rev ? -1 : 1;
  return sa;
}

// everything the kernels read that does not change between stages
struct KLaunch {
  int P;
  int precision;       // DGB_FP64 or DGB_MIXED_FP32
  long E;
  const void* ops;     // packed 1D operator table in the compute type (pack_ops)
  const double* opsd;  // the same table in FP64 (inverse mass matrix)
  const double* geo;   // [E][kGeoStride]
  const double* gv;    // curved meshes: per-point volume geometry [E][kVolC][P^3], else null
  const double* gf;    // curved meshes: per-point face geometry [E][6][kFaceC][P^2], else null
  const int* nbr;      // [E][6]
  DevParams prm;
  bool tc;             // mixed Gauss-point stages with tensor-core volume contractions
  // the mixed Gauss-point kernels take elements two by two (FP32x2 pairs):
  // decided once for the whole mesh (even element count, affine, not tc), so
  // a launch over a piece of the elements keeps the mesh's trace layout
  bool pair;
};

int ops_table_size(int P);
void pack_ops(const Ops1D& o, double* table);
size_t trace_elem_bytes(int precision);  // bytes of one trace value

cudaError_t prepare_kernels(int P, int precision);
// face traces T[E][6][10][P*P] of U
cudaError_t launch_trace(const KLaunch& L, const double* U, void* Tout, cudaStream_t st);
// one stage: residual of Us with traces Tin, then sa.mode's update
cudaError_t launch_stage(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                         cudaStream_t st);
// norms[*counter] = sqrt(sum(part) * inv_size) when *counter < cap; ++*counter
cudaError_t launch_norm(long E, const double* part, double inv_size, double* norms, long cap, int* counter,
                        int* flag, cudaStream_t st);

// mean = (mean*old_w + U) / new_w over n values (mean starts at 0 when reset)
cudaError_t launch_mean_update(long n, double* mean, const double* U, double old_w, double new_w, int reset,
                               cudaStream_t st);

// per compute type (kernels_fp64.cu / kernels_fp32.cu)
cudaError_t prepare_fp64(int P);
cudaError_t launch_trace_fp64(const KLaunch& L, const double* U, void* Tout, cudaStream_t st);
cudaError_t launch_stage_fp64(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                              cudaStream_t st);
cudaError_t prepare_fp32(int P);
cudaError_t launch_trace_fp32(const KLaunch& L, const double* U, void* Tout, cudaStream_t st);
cudaError_t launch_stage_fp32(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                              cudaStream_t st);
// the same with the heat flux (kernels_heat_fp64.cu / kernels_heat_fp32.cu)
cudaError_t prepare_fp64_heat(int P);
cudaError_t launch_trace_fp64_heat(const KLaunch& L, const double* U, void* Tout, cudaStream_t st);
cudaError_t launch_stage_fp64_heat(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                                   cudaStream_t st);
cudaError_t prepare_fp32_heat(int P);
cudaError_t launch_trace_fp32_heat(const KLaunch& L, const double* U, void* Tout, cudaStream_t st);
cudaError_t launch_stage_fp32_heat(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                                   cudaStream_t st);

// Gauss-point form of the stage (vspace.cuh), used by dgb_step: states,
// stage states and the RK accumulator are values at the P^3 Gauss points
cudaError_t prepare_gauss(int P, int precision);
cudaError_t launch_vtrace(const KLaunch& L, const double* V, void* Tout, cudaStream_t st);
cudaError_t launch_vstage(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                          cudaStream_t st);
// the basis changes of the Gauss-point form, FP64, per element (vspace.cuh)
enum { GB_TO_GAUSS = 0, GB_TO_NODAL = 1, GB_ADJ_TO_GAUSS = 2, GB_ADJ_TO_NODAL = 3 };
// out2, when given, receives the same values as out
cudaError_t launch_gauss_basis_mode(const KLaunch& L, const double* in, double* out, int mode, cudaStream_t st,
                                    double* out2 = nullptr);
// V = B3 U (to_gauss) or U = B3^-1 V
inline cudaError_t launch_gauss_basis(const KLaunch& L, const double* in, double* out, bool to_gauss,
                                      cudaStream_t st, double* out2 = nullptr)
{
  return launch_gauss_basis_mode(L, in, out, to_gauss ? GB_TO_GAUSS : GB_TO_NODAL, st, out2);
}
// per compute type and heat flag (vspace_*.cu)
cudaError_t vprepare_fp64(int P, bool heat);
cudaError_t vlaunch_trace_fp64(const KLaunch& L, const double* V, void* Tout, cudaStream_t st);
cudaError_t vlaunch_stage_fp64(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                               cudaStream_t st);
cudaError_t vprepare_fp32(int P, bool heat);
cudaError_t vlaunch_trace_fp32(const KLaunch& L, const double* V, void* Tout, cudaStream_t st);
cudaError_t vlaunch_stage_fp32(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                               cudaStream_t st);
cudaError_t vprepare_fp64_heat(int P);
cudaError_t vlaunch_trace_fp64_heat(const KLaunch& L, const double* V, void* Tout, cudaStream_t st);
cudaError_t vlaunch_stage_fp64_heat(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                                    cudaStream_t st);
cudaError_t vprepare_fp32_heat(int P);
cudaError_t vlaunch_trace_fp32_heat(const KLaunch& L, const double* V, void* Tout, cudaStream_t st);
cudaError_t vlaunch_stage_fp32_heat(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                                    cudaStream_t st);
// the viscous terms alone of the FP64 Gauss-point residual (vspace_visc.cu)
cudaError_t vlaunch_stage_visc(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                               cudaStream_t st);
// the mixed stage with tensor-core volume contractions (tc.cuh, vspace_tc.cu)
bool tc_supported(int P);
cudaError_t vprepare_tc(int P);
cudaError_t vlaunch_stage_tc(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                             cudaStream_t st);

}  // namespace dgb
