// Gauss-point stage kernels (vspace.cuh) in FP32 with the heat flux (HT = true).
#include "vspace.cuh"

namespace dgb {

cudaError_t vprepare_fp32_heat(int P)
{
  cudaError_t e = vprepare_t<float, true>(P);
  return e == cudaSuccess ? vprepare2_t<true>(P) : e;
}

cudaError_t vlaunch_trace_fp32_heat(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  return use_pair(L) ? vlaunch_trace2_t<true>(L, V, Tout, st) : vlaunch_trace_t<float, true>(L, V, Tout, st);
}

cudaError_t vlaunch_stage_fp32_heat(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                                    cudaStream_t st)
{
  return use_pair(L) ? vlaunch_stage2_t<true>(L, Vs, Tin, sa, st) : vlaunch_stage_t<float, true>(L, Vs, Tin, sa, st);
}

}  // namespace dgb
