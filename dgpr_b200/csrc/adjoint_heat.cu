// Discrete adjoint of the FP64 residual with the heat flux: the kernels of
// adjoint_kernels.cuh instantiated with HT = true, compiled apart from the
// plain ones so that both build in parallel.
#include "adjoint_kernels.cuh"

namespace dgb {

cudaError_t prepare_adjoint_heat(int P) { return prepare_adj_t<true, false>(P); }

cudaError_t launch_residual_vjp_heat(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st)
{
  return launch_vjp_t<true, false>(L, v, s, st);
}

}  // namespace dgb
