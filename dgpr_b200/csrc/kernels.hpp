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
  double* part;   // per-element sum of R^2 (stage 1 of a step), or null
  int* flag;      // bit 1: non-finite norm, bit 2: inflow without a Mach root
  double* Tnext;  // face traces of Uout for the next stage, or null
};

// everything the FP64 kernels read that does not change between stages
struct Fp64Launch {
  int P;
  long E;
  const double* ops;   // packed 1D operator table (pack_ops)
  const double* geo;   // [E][kGeoStride]
  const int* nbr;      // [E][6]
  DevParams prm;
};

int ops_table_size(int P);
void pack_ops(const Ops1D& o, double* table);
size_t stage_smem_bytes(int P);

cudaError_t prepare_fp64_kernels(int P);
// face traces T[E][6][10][P*P] of U
cudaError_t launch_trace(const Fp64Launch& L, const double* U, double* Tout, cudaStream_t st);
// one stage: residual of Us with traces Tin, then sa.mode's update
cudaError_t launch_stage(const Fp64Launch& L, const double* Us, const double* Tin, const StageArgs& sa,
                         cudaStream_t st);
cudaError_t launch_norm(long E, const double* part, double inv_size, double* norms, int* counter,
                        int* flag, cudaStream_t st);

}  // namespace dgb
