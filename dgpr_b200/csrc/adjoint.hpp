// Launch interface of the adjoint (residual VJP) kernels, adjoint.cu.
#pragma once

#include <cuda_runtime.h>

#include "kernels.hpp"

namespace dgb {

// One residual VJP: with lam = cx X + cy Y + cz Z (Y, Z may be null) it
// computes a = (df/dU)^T lam at U, f = -Minv R(U), and writes
//   a_out = a                (if a_out)
//   acc_out = acc_in + a     (if acc_out; acc_in may be null, or alias acc_out)
// a_out may alias Y or Z (they are read before it is written); acc_out may
// alias X, Y or Z likewise.
struct VjpArgs {
  const double* U;
  const double* Tr;  // FP64 face traces of U [E][6][10][P*P], or null: computed into the scratch
  const double* X;
  const double* Y;
  const double* Z;
  double cx, cy, cz;
  double* a_out;
  const double* acc_in;
  double* acc_out;
};

// per-handle scratch of a VJP
struct VjpScratch {
  double* trace;  // FP64 face traces [E][6][10][P*P]
  double* ta;     // face-trace adjoints [E][6][20][P*P]; an isothermal-wall face keeps its points'
                  // dJ/dTw terms in [10][P*P]
  double* part;   // volume part of a, [E][5][P^3]
  int* flag;      // bit 3: a boundary type without an adjoint
};

cudaError_t prepare_adjoint(int P);
// [trace_kernel (FP64)] + adjA + adjB on stream st; L.opsd is the operator table
cudaError_t launch_residual_vjp(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st);
// the heat-conducting kernels (adjoint_heat.cu); launch_residual_vjp picks them when L.prm.kq != 0
cudaError_t prepare_adjoint_heat(int P);
cudaError_t launch_residual_vjp_heat(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st);
// The Gauss-point form (U, lam and the result at the Gauss points: the VJP of
// f_V, vspace.cuh), for the reverse steps of recorded runs in that form
// (adjoint_gauss.cu, adjoint_gauss_heat.cu); prepared by prepare_adjoint
cudaError_t launch_residual_vjp_gauss(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st);
cudaError_t prepare_adjoint_gauss(int P);
cudaError_t prepare_adj_t_gauss_heat(int P);
cudaError_t launch_vjp_gauss_plain(const KLaunch& L, const VjpArgs& v, const VjpScratch& s, cudaStream_t st);
cudaError_t launch_residual_vjp_gauss_heat(const KLaunch& L, const VjpArgs& v, const VjpScratch& s,
                                           cudaStream_t st);

}  // namespace dgb
