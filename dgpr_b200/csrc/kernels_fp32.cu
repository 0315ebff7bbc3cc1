// FP32 instantiation of the residual / stage kernels: the mixed form.
// Contractions, traces and pointwise fluxes run in FP32; the kernels keep the
// state, the inverse mass matrix and the RK update in FP64 (kernels.cuh).
#include "kernels.cuh"

namespace dgb {

cudaError_t prepare_fp32(int P)
{
  cudaError_t e = prepare_t<float, false>(P);
  return e == cudaSuccess ? prepare_fp32_heat(P) : e;
}

cudaError_t launch_trace_fp32(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  return L.prm.kq != 0. ? launch_trace_fp32_heat(L, U, Tout, st) : launch_trace_t<float, false>(L, U, Tout, st);
}

cudaError_t launch_stage_fp32(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                              cudaStream_t st)
{
  return L.prm.kq != 0. ? launch_stage_fp32_heat(L, Us, Tin, sa, st)
                        : launch_stage_t<float, false>(L, Us, Tin, sa, st);
}

}  // namespace dgb
