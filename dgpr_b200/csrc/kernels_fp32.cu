// FP32 instantiation of the residual / stage kernels: the mixed form.
// Contractions, traces and pointwise fluxes run in FP32; the kernels keep the
// state, the inverse mass matrix and the RK update in FP64 (kernels.cuh).
#include "kernels.cuh"

namespace dgb {

cudaError_t prepare_fp32(int P)
{
  switch (P) {
    case 1: return prepare_p<1, float>();
    case 2: return prepare_p<2, float>();
    case 3: return prepare_p<3, float>();
    case 4: return prepare_p<4, float>();
    case 5: return prepare_p<5, float>();
    case 6: return prepare_p<6, float>();
    case 7: return prepare_p<7, float>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_trace_fp32(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_trace_p<1, float>(L, U, Tout, st);
    case 2: return launch_trace_p<2, float>(L, U, Tout, st);
    case 3: return launch_trace_p<3, float>(L, U, Tout, st);
    case 4: return launch_trace_p<4, float>(L, U, Tout, st);
    case 5: return launch_trace_p<5, float>(L, U, Tout, st);
    case 6: return launch_trace_p<6, float>(L, U, Tout, st);
    case 7: return launch_trace_p<7, float>(L, U, Tout, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage_fp32(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                              cudaStream_t st)
{
  switch (L.P) {
    case 1: return launch_stage_p<1, float>(L, Us, Tin, sa, st);
    case 2: return launch_stage_p<2, float>(L, Us, Tin, sa, st);
    case 3: return launch_stage_p<3, float>(L, Us, Tin, sa, st);
    case 4: return launch_stage_p<4, float>(L, Us, Tin, sa, st);
    case 5: return launch_stage_p<5, float>(L, Us, Tin, sa, st);
    case 6: return launch_stage_p<6, float>(L, Us, Tin, sa, st);
    case 7: return launch_stage_p<7, float>(L, Us, Tin, sa, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dgb
