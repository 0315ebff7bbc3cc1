// FP64 residual / stage kernels with the heat flux: the
// kernels of kernels.cuh instantiated with HT = true, compiled apart from the
// plain ones so that both build in parallel.
#include "kernels.cuh"

namespace dgb {

cudaError_t prepare_fp64_heat(int P) { return prepare_t<double, true>(P); }

cudaError_t launch_trace_fp64_heat(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  return launch_trace_t<double, true>(L, U, Tout, st);
}

cudaError_t launch_stage_fp64_heat(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                                   cudaStream_t st)
{
  return launch_stage_t<double, true>(L, Us, Tin, sa, st);
}

}  // namespace dgb
