// Discrete adjoint of the FP64 residual in the Gauss-point form with the heat
// flux: the kernels of adjoint_kernels.cuh instantiated with HT = GS = true.
#include "adjoint_kernels.cuh"

namespace dgb {

cudaError_t prepare_adj_t_gauss_heat(int P) { return prepare_adj_t<true, true>(P); }

cudaError_t launch_residual_vjp_gauss_heat(const KLaunch& L, const VjpArgs& v, const VjpScratch& s,
                                           cudaStream_t st)
{
  return launch_vjp_t<true, true>(L, v, s, st);
}

}  // namespace dgb
