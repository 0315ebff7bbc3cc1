// Discrete adjoint of the FP64 residual: the kernels of adjoint_kernels.cuh
// without the heat flux, and the dispatch to the heat-conducting ones
// (adjoint_heat.cu) when the handle has one.
#include "adjoint_kernels.cuh"

namespace dgb {

cudaError_t prepare_adjoint(int P)
{
  cudaError_t e = prepare_fp64(P);  // the FP64 trace kernel, also on mixed-precision handles
  if (e == cudaSuccess) e = prepare_adj_t<false>(P);
  return e == cudaSuccess ? prepare_adjoint_heat(P) : e;
}

cudaError_t launch_residual_vjp(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st)
{
  return L.prm.kq != 0. ? launch_residual_vjp_heat(L, v, s, st) : launch_vjp_t<false>(L, v, s, st);
}

}  // namespace dgb
