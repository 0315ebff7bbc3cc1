// The viscous terms of the FP64 Gauss-point residual alone (vstage_kernel
// with VO): the derivative of the residual in the viscosity, for the
// parameter gradients of the adjoint sweep.
#include "../../include/dgb200.h"
#include "vspace.cuh"

namespace dgb {

template <int P, bool CV, bool HT>
static cudaError_t visc_launch_k(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                                 cudaStream_t st)
{
  using K = VStageSmem<P, double>;
  cudaError_t e = cudaFuncSetAttribute(vstage_kernel<P, double, CV, HT, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, K::TOTAL);
  if (e != cudaSuccess) return e;
  vstage_kernel<P, double, CV, HT, true><<<(unsigned)L.E, Cfg<P>::NTS, K::TOTAL, st>>>(
      L.E, Vs, reinterpret_cast<const double*>(Tin), reinterpret_cast<const double*>(L.ops), L.opsd, L.geo,
      CV ? L.gv : nullptr, CV ? L.gf : nullptr, L.nbr, L.prm, element_order(sa, L.E, 1));
  return cudaGetLastError();
}

template <int P>
static cudaError_t visc_launch_p(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                                 cudaStream_t st)
{
  const bool heat = L.prm.kq != 0.;
  if (L.gv)
    return heat ? visc_launch_k<P, true, true>(L, Vs, Tin, sa, st) : visc_launch_k<P, true, false>(L, Vs, Tin, sa, st);
  return heat ? visc_launch_k<P, false, true>(L, Vs, Tin, sa, st) : visc_launch_k<P, false, false>(L, Vs, Tin, sa, st);
}

cudaError_t vlaunch_stage_visc(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                               cudaStream_t st)
{
  if (L.precision != DGB_FP64 || sa.mode != MODE_RESIDUAL || sa.ecount) return cudaErrorInvalidValue;
  switch (L.P) {
    case 1: return visc_launch_p<1>(L, Vs, Tin, sa, st);
    case 2: return visc_launch_p<2>(L, Vs, Tin, sa, st);
    case 3: return visc_launch_p<3>(L, Vs, Tin, sa, st);
    case 4: return visc_launch_p<4>(L, Vs, Tin, sa, st);
    case 5: return visc_launch_p<5>(L, Vs, Tin, sa, st);
    case 6: return visc_launch_p<6>(L, Vs, Tin, sa, st);
    case 7: return visc_launch_p<7>(L, Vs, Tin, sa, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dgb
