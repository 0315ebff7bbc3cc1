// FP32 (mixed form) residual / stage kernels with the heat flux: the
// kernels of kernels.cuh instantiated with HT = true, compiled apart from the
// plain ones so that both build in parallel.
#include "kernels.cuh"

namespace dgb {

cudaError_t prepare_fp32_heat(int P) { return prepare_t<float, true>(P); }

cudaError_t launch_trace_fp32_heat(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  return launch_trace_t<float, true>(L, U, Tout, st);
}

cudaError_t launch_stage_fp32_heat(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                                   cudaStream_t st)
{
  return launch_stage_t<float, true>(L, Us, Tin, sa, st);
}

}  // namespace dgb
