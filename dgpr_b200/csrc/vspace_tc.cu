// The mixed form's Gauss-point stage with tensor-core volume contractions
// (tc.cuh): p = 3 and 4, affine elements, no heat flux.
#include "tc.cuh"

namespace dgb {

template <int P>
static cudaError_t tc_prepare_p()
{
  return cudaFuncSetAttribute(vstage_tc_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcSmem<P>::TOTAL);
}

bool tc_supported(int P) { return P == 4 || P == 5; }

cudaError_t vprepare_tc(int P)
{
  switch (P) {
    case 4: return tc_prepare_p<4>();
    case 5: return tc_prepare_p<5>();
  }
  return cudaErrorNotSupported;
}

template <int P>
static cudaError_t tc_launch_p(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                               cudaStream_t st)
{
  const unsigned grid = (unsigned)(sa.ecount ? sa.ecount : L.E);
  vstage_tc_kernel<P><<<grid, kTcThreads, TcSmem<P>::TOTAL, st>>>(
      L.E, Vs, reinterpret_cast<const float*>(Tin), reinterpret_cast<const float*>(L.ops), L.opsd, L.geo, L.nbr,
      L.prm, element_order(sa, L.E, 1));
  return cudaGetLastError();
}

cudaError_t vlaunch_stage_tc(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                             cudaStream_t st)
{
  if (L.gv || L.prm.kq != 0.) return cudaErrorNotSupported;  // curved elements, heat flux: not built
  switch (L.P) {
    case 4: return tc_launch_p<4>(L, Vs, Tin, sa, st);
    case 5: return tc_launch_p<5>(L, Vs, Tin, sa, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace dgb
