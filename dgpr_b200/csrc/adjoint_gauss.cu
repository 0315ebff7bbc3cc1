// Discrete adjoint of the FP64 residual in the Gauss-point form (the VJP of
// f_V, vspace.cuh), without the heat flux: the kernels of adjoint_kernels.cuh
// instantiated with GS = true, compiled apart so that the forms build in
// parallel.
#include "adjoint_kernels.cuh"

namespace dgb {

cudaError_t prepare_adjoint_gauss(int P)
{
  cudaError_t e = prepare_adj_t<false, true>(P);
  return e == cudaSuccess ? prepare_adj_t_gauss_heat(P) : e;
}

cudaError_t launch_vjp_gauss_plain(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st)
{
  return launch_vjp_t<false, true>(L, v, s, st);
}

}  // namespace dgb
