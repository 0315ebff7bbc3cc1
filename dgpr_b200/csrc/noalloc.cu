// dgb_residual_noalloc: one FP64 residual evaluation that allocates no device
// memory.
//
// Who needs it: callers that are not allowed to allocate GPU memory at the
// point where they need a residual.  Examples: a host application that owns
// the device memory pool and hands libraries only pointers it manages, or a
// solver loop that has reserved all HBM for its own state before this library
// is called.  dgb_create allocates per-mesh buffers with cudaMalloc; this entry
// point instead keeps every intermediate it needs in one fixed-size array that
// is part of the library image itself (file-scope `static __device__`), so the
// call only copies data and launches kernels.
//
// Costs of that choice:
//  * every GPU that loads the library reserves the array (kNoallocScratchBytes)
//    for the life of the process, whether or not this entry point is used;
//  * all calls share the one array, so two calls whose work overlaps on the GPU
//    (different streams, or different host threads) race and give wrong
//    results: callers must order them (same stream, or synchronise between);
//  * the array keeps the previous call's contents; everything the kernels read
//    is rewritten at the start of each call, and the status word is cleared;
//  * a call cannot be captured into a CUDA graph: it copies from pageable host
//    memory and synchronises the stream before it returns.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/dgb200.h"
#include "host.hpp"
#include "kernels.hpp"

namespace {

// 32 MiB: operator table, element geometry, neighbour table, face traces and a
// status word.  At p = 3 one element needs about 8 KB, so meshes up to about
// 4,000 elements (e.g. 16^3) fit.
constexpr size_t kNoallocScratchBytes = 32u << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" int dgb_residual_noalloc(const dgb_mesh_desc* mesh, const dgb_params* params, const double* U_dev,
                                    double* f_dev, void* stream)
{
  using namespace dgb;
  if (!mesh || !params || !U_dev || !f_dev) return set_last_error(DGB_ERR_ARG, "null argument");
  Ops1D ops;
  int rc = build_ops(mesh->p, ops);
  if (rc) return set_last_error(rc, "solution order outside 0..6");
  if (mesh->nx <= 0 || mesh->ny <= 0 || mesh->nz <= 0) return set_last_error(DGB_ERR_ARG, "empty mesh");
  {  // the affine layout is a lower bound on the scratch any mesh of this size
     // needs: reject far-too-large meshes before building their geometry
    const double E = (double)mesh->nx * mesh->ny * mesh->nz, NQF = (double)ops.P * ops.P;
    const double lower = E * (60. * NQF * sizeof(double) + kGeoStride * sizeof(double) + 6. * sizeof(int32_t));
    if (lower > (double)kNoallocScratchBytes)
      return set_last_error(DGB_ERR_ARG, "mesh needs at least " + std::to_string((long long)lower) +
                                             " bytes of scratch; the static array holds " +
                                             std::to_string(kNoallocScratchBytes) + " bytes (32 MiB)");
  }
  std::vector<double> geo, gv, gf;
  std::vector<int32_t> nbr;
  std::string why;
  bool curved = false;
  rc = build_geometry(*mesh, ops, geo, nbr, why, curved, gv, gf);
  if (rc) return set_last_error(rc, why);
  const int P = ops.P, NQF = P * P;
  const long E = (long)mesh->nx * mesh->ny * mesh->nz;
  std::vector<double> table(ops_table_size(P));
  pack_ops(ops, table.data());

  // layout inside the static array
  const size_t oOps = 0;
  const size_t oGeo = oOps + round256(sizeof(double) * table.size());
  const size_t oNbr = oGeo + round256(sizeof(double) * geo.size());
  const size_t oTr = oNbr + round256(sizeof(int32_t) * nbr.size());
  const size_t oGv = oTr + round256(sizeof(double) * (size_t)E * 60 * NQF);  // curved meshes: per-point geometry
  const size_t oGf = oGv + round256(sizeof(double) * gv.size());
  const size_t oFlag = oGf + round256(sizeof(double) * gf.size());
  const size_t need = oFlag + 256;
  if (need > kNoallocScratchBytes)
    return set_last_error(DGB_ERR_ARG, "mesh needs " + std::to_string(need) +
                                           " bytes of scratch; the static array holds " +
                                           std::to_string(kNoallocScratchBytes) + " bytes (32 MiB)");

  // the array's device address on the current device, looked up on every
  // call (a lookup, no allocation): the host-side symbol is not a device
  // pointer, and an address kept from an earlier call would be stale after
  // the context was torn down and made again
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_last_error(DGB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int sdev = dev;
  e = cudaStreamGetDevice(st, &sdev);
  if (e != cudaSuccess)
    return set_last_error(DGB_ERR_CUDA, std::string("cudaStreamGetDevice: ") + cudaGetErrorString(e));
  if (sdev != dev)
    return set_last_error(DGB_ERR_ARG, "stream belongs to device " + std::to_string(sdev) +
                                           ", but the current device is " + std::to_string(dev));
  unsigned char* base = nullptr;
  {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return set_last_error(DGB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    base = static_cast<unsigned char*>(p);
  }
  // shared-memory attributes of the kernel instances for this order (no allocation)
  e = prepare_kernels(P, DGB_FP64);
  if (e != cudaSuccess) return set_last_error(DGB_ERR_CUDA, std::string("kernel set-up: ") + cudaGetErrorString(e));

  int* flag = reinterpret_cast<int*>(base + oFlag);
#define NA_CK(call)                                                                                \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return set_last_error(DGB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
  NA_CK(cudaMemcpyAsync(base + oOps, table.data(), sizeof(double) * table.size(), cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(base + oGeo, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice, st));
  if (curved) {
    NA_CK(cudaMemcpyAsync(base + oGv, gv.data(), sizeof(double) * gv.size(), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + oGf, gf.data(), sizeof(double) * gf.size(), cudaMemcpyHostToDevice, st));
  }
  NA_CK(cudaMemcpyAsync(base + oNbr, nbr.data(), sizeof(int32_t) * nbr.size(), cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemsetAsync(flag, 0, sizeof(int), st));  // status word must start at zero

  KLaunch L{};
  L.P = P;
  L.precision = DGB_FP64;
  L.E = E;
  L.ops = base + oOps;
  L.opsd = reinterpret_cast<const double*>(base + oOps);
  L.geo = reinterpret_cast<const double*>(base + oGeo);
  L.nbr = reinterpret_cast<const int*>(base + oNbr);
  L.gv = curved ? reinterpret_cast<const double*>(base + oGv) : nullptr;
  L.gf = curved ? reinterpret_cast<const double*>(base + oGf) : nullptr;
  L.prm.gamma = params->gamma;
  L.prm.R = params->R;
  L.prm.mu = params->mu;
  L.prm.P = params->P;
  L.prm.eta = params->eta;
  L.prm.Tw = params->T;  // isothermal walls at the reference temperature
  total_conditions(*params, &L.prm.Tt, &L.prm.Pt);
  for (int r = 0; r < 5; ++r) {
    L.prm.Ufr[r] = params->Ufr[r];
    L.prm.src[r] = params->source[r];
  }
  void* traces = base + oTr;  // fully rewritten by the trace kernel before it is read
  NA_CK(launch_trace(L, U_dev, traces, st));
  StageArgs a;
  memset(&a, 0, sizeof a);
  a.mode = MODE_RESIDUAL;
  a.fout = f_dev;
  a.flag = flag;
  NA_CK(launch_stage(L, U_dev, traces, a, st));
  int hflag = 0;
  NA_CK(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
#undef NA_CK
  if (hflag & 2) return set_last_error(DGB_ERR_BOUNDARY, "subsonic inflow without a non-negative Mach root");
  return DGB_OK;
}
