// Gauss-point stage kernels (vspace.cuh) in FP64 without the heat flux, the
// basis change, and the dispatch of the Gauss-point form on compute type and
// heat flag (dgb_step).
#include "../../include/dgb200.h"
#include "vspace.cuh"

namespace dgb {

cudaError_t vprepare_fp64(int P, bool heat)
{
  cudaError_t e = vprepare_t<double, false>(P);
  return e == cudaSuccess && heat ? vprepare_fp64_heat(P) : e;
}

cudaError_t vlaunch_trace_fp64(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  return L.prm.kq != 0. ? vlaunch_trace_fp64_heat(L, V, Tout, st) : vlaunch_trace_t<double, false>(L, V, Tout, st);
}

cudaError_t vlaunch_stage_fp64(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa,
                               cudaStream_t st)
{
  return L.prm.kq != 0. ? vlaunch_stage_fp64_heat(L, Vs, Tin, sa, st)
                        : vlaunch_stage_t<double, false>(L, Vs, Tin, sa, st);
}

cudaError_t prepare_gauss(int P, int precision)
{
  cudaError_t e = precision == DGB_MIXED_FP32 ? vprepare_fp32(P, true) : vprepare_fp64(P, true);
  return e;
}

cudaError_t launch_vtrace(const KLaunch& L, const double* V, void* Tout, cudaStream_t st)
{
  return L.precision == DGB_MIXED_FP32 ? vlaunch_trace_fp32(L, V, Tout, st) : vlaunch_trace_fp64(L, V, Tout, st);
}

cudaError_t launch_vstage(const KLaunch& L, const double* Vs, const void* Tin, const StageArgs& sa, cudaStream_t st)
{
  return L.precision == DGB_MIXED_FP32 ? vlaunch_stage_fp32(L, Vs, Tin, sa, st)
                                       : vlaunch_stage_fp64(L, Vs, Tin, sa, st);
}

template <int P>
static cudaError_t gauss_basis_p(const KLaunch& L, const double* in, double* out, int mode, cudaStream_t st,
                                 double* out2)
{
  const unsigned g = (unsigned)L.E;
  switch (mode) {
    case GB_TO_GAUSS: gauss_basis_kernel<P, GB_TO_GAUSS><<<g, Cfg<P>::NT, 0, st>>>(L.E, in, out, L.opsd, out2); break;
    case GB_TO_NODAL: gauss_basis_kernel<P, GB_TO_NODAL><<<g, Cfg<P>::NT, 0, st>>>(L.E, in, out, L.opsd, out2); break;
    case GB_ADJ_TO_GAUSS:
      gauss_basis_kernel<P, GB_ADJ_TO_GAUSS><<<g, Cfg<P>::NT, 0, st>>>(L.E, in, out, L.opsd, out2);
      break;
    case GB_ADJ_TO_NODAL:
      gauss_basis_kernel<P, GB_ADJ_TO_NODAL><<<g, Cfg<P>::NT, 0, st>>>(L.E, in, out, L.opsd, out2);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_gauss_basis_mode(const KLaunch& L, const double* in, double* out, int mode, cudaStream_t st,
                                    double* out2)
{
  switch (L.P) {
    case 1: return gauss_basis_p<1>(L, in, out, mode, st, out2);
    case 2: return gauss_basis_p<2>(L, in, out, mode, st, out2);
    case 3: return gauss_basis_p<3>(L, in, out, mode, st, out2);
    case 4: return gauss_basis_p<4>(L, in, out, mode, st, out2);
    case 5: return gauss_basis_p<5>(L, in, out, mode, st, out2);
    case 6: return gauss_basis_p<6>(L, in, out, mode, st, out2);
    case 7: return gauss_basis_p<7>(L, in, out, mode, st, out2);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dgb
