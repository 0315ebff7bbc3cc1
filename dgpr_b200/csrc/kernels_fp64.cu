// FP64 instantiation of the residual / stage kernels (the plain form), plus
// the pieces shared by both compute types: operator-table packing, the
// residual-norm reduction and the dispatch on the precision.
#include "../../include/dgb200.h"
#include "kernels.cuh"

namespace dgb {

int ops_table_size(int P) { return 5 * P * P + 10 * P + 2; }

void pack_ops(const Ops1D& o, double* t)
{
  const int P = o.P, PP = P * P;
  for (int i = 0; i < PP; ++i) {
    t[i] = o.B[i];
    t[PP + i] = o.Bd[i];
    t[2 * PP + i] = o.Dq[i];
    t[3 * PP + i] = o.M1i[i];
    t[4 * PP + i] = o.Bi[i];
  }
  const int oE = 5 * PP, oD = oE + 2 * P, oWb = oD + 2 * P, oW = oWb + P, oC = oW + P;
  for (int i = 0; i < P; ++i) {
    t[oE + i] = o.E[0][i];
    t[oE + P + i] = o.E[1][i];
    t[oD + i] = o.D[0][i];
    t[oD + P + i] = o.D[1][i];
    t[oWb + i] = o.Wb[i];
    t[oW + i] = o.w[i];
  }
  t[oC] = o.cend[0];
  t[oC + 1] = o.cend[1];
  const int oEh = oC + 2, oDh = oEh + 2 * P;
  for (int q = 0; q < P; ++q) {
    t[oEh + q] = o.EL[0][q];
    t[oEh + P + q] = o.EL[1][q];
    t[oDh + q] = o.DL[0][q];
    t[oDh + P + q] = o.DL[1][q];
  }
}

size_t trace_elem_bytes(int precision) { return precision == DGB_MIXED_FP32 ? sizeof(float) : sizeof(double); }

// sqrt(sum(part) / size) into norms[*counter], deterministic fixed-order sum
__global__ void norm_kernel(long E, const double* __restrict__ part, double inv_size, double* norms, long cap,
                            int* counter, int* flag)
{
  __shared__ double red[1024];
  const int tid = threadIdx.x;
  double s = 0.;
  for (long i = tid; i < E; i += blockDim.x) s += part[i];
  red[tid] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (tid < w) red[tid] += red[tid + w];
    __syncthreads();
  }
  if (tid == 0) {
    const int c = *counter;
    const double v = sqrt(red[0] * inv_size);
    if (c >= 0 && c < cap) norms[c] = v;
    if (!isfinite(v)) *flag |= 1;
    *counter = c + 1;
  }
}

cudaError_t launch_norm(long E, const double* part, double inv_size, double* norms, long cap, int* counter,
                        int* flag, cudaStream_t st)
{
  norm_kernel<<<1, 1024, 0, st>>>(E, part, inv_size, norms, cap, counter, flag);
  return cudaGetLastError();
}

// running mean of the state (output.cpp:39-49): mean = (mean*old + U) / new,
// unfused like the reference's expression; `reset` starts from zero
__global__ void mean_update_kernel(long n, double* __restrict__ mean, const double* __restrict__ U, double old_w,
                                   double new_w, int reset)
{
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double m = reset ? 0. : mean[i];
    mean[i] = __ddiv_rn(__dadd_rn(__dmul_rn(m, old_w), U[i]), new_w);
  }
}

cudaError_t launch_mean_update(long n, double* mean, const double* U, double old_w, double new_w, int reset,
                               cudaStream_t st)
{
  mean_update_kernel<<<148 * 8, 256, 0, st>>>(n, mean, U, old_w, new_w, reset);
  return cudaGetLastError();
}

// the heat-conducting kernels (kernels_heat_fp64.cu) are prepared with the
// plain ones and launched when the handle has a heat flux
cudaError_t prepare_fp64(int P)
{
  cudaError_t e = prepare_t<double, false>(P);
  return e == cudaSuccess ? prepare_fp64_heat(P) : e;
}

cudaError_t launch_trace_fp64(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  return L.prm.kq != 0. ? launch_trace_fp64_heat(L, U, Tout, st) : launch_trace_t<double, false>(L, U, Tout, st);
}

cudaError_t launch_stage_fp64(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa,
                              cudaStream_t st)
{
  return L.prm.kq != 0. ? launch_stage_fp64_heat(L, Us, Tin, sa, st)
                        : launch_stage_t<double, false>(L, Us, Tin, sa, st);
}

cudaError_t prepare_kernels(int P, int precision)
{
  return precision == DGB_MIXED_FP32 ? prepare_fp32(P) : prepare_fp64(P);
}

cudaError_t launch_trace(const KLaunch& L, const double* U, void* Tout, cudaStream_t st)
{
  return L.precision == DGB_MIXED_FP32 ? launch_trace_fp32(L, U, Tout, st) : launch_trace_fp64(L, U, Tout, st);
}

cudaError_t launch_stage(const KLaunch& L, const double* Us, const void* Tin, const StageArgs& sa, cudaStream_t st)
{
  return L.precision == DGB_MIXED_FP32 ? launch_stage_fp32(L, Us, Tin, sa, st)
                                       : launch_stage_fp64(L, Us, Tin, sa, st);
}

}  // namespace dgb
