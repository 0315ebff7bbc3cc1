// Mixed-precision residual path: FP32 contractions and fluxes, FP64 geometry,
// inverse mass and RK accumulation.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "host.hpp"
#include "physics.cuh"

namespace dgb {

struct MixedState;

int mixed_create(MixedState** out, const Ops1D& ops, const std::vector<double>& geo, const double* d_geo,
                 const int* d_nbr, long E, const DevParams& prm);
void mixed_destroy(MixedState* m);
int mixed_residual(MixedState* m, const double* U, double* R, double* f, cudaStream_t st);
int mixed_initial_traces(MixedState* m, const double* U, cudaStream_t st);
int mixed_step(MixedState* m, int scheme, double dt, double* U, double* Us, double* acc, double* part,
               double* norms, int* counter, int* flag, cudaStream_t st, cudaEvent_t* ev);
long long mixed_launches_per_step(const MixedState* m, int nstages);

}  // namespace dgb
