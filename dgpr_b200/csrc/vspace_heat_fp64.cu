// Gauss-point stage kernels (vspace.cuh) in FP64 with the heat flux (HT = true).
#include "vspace.cuh"

namespace dgb {

cudaError_t vprepare_fp64_heat(int P) { return vprepare_t<double, true>(P); }

cudaError_t vlaunch_trace_fp64_heat(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  return vlaunch_trace_t<double, true>(L, V, Tout, st);
}

cudaError_t vlaunch_stage_fp64_heat(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                                    cudaStream_t st)
{
  return vlaunch_stage_t<double, true>(L, Vs, Tin, sa, st);
}

}  // namespace dgb
