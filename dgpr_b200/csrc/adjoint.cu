// Discrete adjoint of the FP64 residual: the nodal kernels of
// adjoint_kernels.cuh without the heat flux, and the dispatch to the
// heat-conducting ones (adjoint_heat.cu) and to the Gauss-point form
// (adjoint_gauss.cu, adjoint_gauss_heat.cu).
#include "adjoint_kernels.cuh"

namespace dgb {

cudaError_t prepare_adjoint(int P)
{
  cudaError_t e = prepare_fp64(P);  // the FP64 trace kernel, also on mixed-precision handles
  if (e == cudaSuccess) e = vprepare_fp64(P, true);  // FP64 Gauss-point traces, also on mixed handles
  if (e == cudaSuccess) e = prepare_adj_t<false, false>(P);
  if (e == cudaSuccess) e = prepare_adjoint_heat(P);
  return e == cudaSuccess ? prepare_adjoint_gauss(P) : e;
}

cudaError_t launch_residual_vjp(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st)
{
  return L.prm.kq != 0. ? launch_residual_vjp_heat(L, v, s, st) : launch_vjp_t<false, false>(L, v, s, st);
}

cudaError_t launch_residual_vjp_gauss(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st)
{
  return L.prm.kq != 0. ? launch_residual_vjp_gauss_heat(L, v, s, st) : launch_vjp_gauss_plain(L, v, s, st);
}

}  // namespace dgb
