// Gauss-point stage kernels (vspace.cuh) in FP32 (the mixed form) without
// the heat flux: the paired kernels where they apply, else one element per CTA.
#include "vspace.cuh"

namespace dgb {

cudaError_t vprepare_fp32(int P, bool heat)
{
  cudaError_t e = vprepare_t<float, false>(P);
  if (e == cudaSuccess) e = vprepare2_t<false>(P);
  return e == cudaSuccess && heat ? vprepare_fp32_heat(P) : e;
}

cudaError_t vlaunch_trace_fp32(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  if (L.prm.kq != 0.) return vlaunch_trace_fp32_heat(L, V, Tout, st);
  return use_pair(L) ? vlaunch_trace2_t<false>(L, V, Tout, st) : vlaunch_trace_t<float, false>(L, V, Tout, st);
}

cudaError_t vlaunch_stage_fp32(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                               cudaStream_t st)
{
  if (L.tc) return vlaunch_stage_tc(L, Vs, Tin, sa, st);
  if (L.prm.kq != 0.) return vlaunch_stage_fp32_heat(L, Vs, Tin, sa, st);
  return use_pair(L) ? vlaunch_stage2_t<false>(L, Vs, Tin, sa, st) : vlaunch_stage_t<float, false>(L, Vs, Tin, sa, st);
}

}  // namespace dgb
