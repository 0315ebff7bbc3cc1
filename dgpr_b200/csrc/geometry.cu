// Element geometry on the device: the precompute of build_geometry (host.cpp)
// as kernels, one thread per element, sample point, or face point.  The
// reference does this on the host, element by element
// (core_geometry::precompute, geometry_common.cpp:292-395, with the face
// geometry of geometry_common.cpp:416-454 and geometry_shared.cpp:156-267).
//
// The results are bit-identical to the host builder's: the kernels start
// from the host's 1D Lagrange tables (GeoTables) and repeat its operations in
// its order, with the _rn intrinsics, which the compiler does not contract
// into fused multiply-adds.  Division and square root are IEEE-rounded on
// both sides.
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>

#include "host.hpp"

namespace dgb {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// J[r][c] = d x_r / d xi_c at the reference point whose coordinates are the
// table rows (ma, mb, mc); loop and operation order of host.cpp's jacobian
__device__ void jacobian_at(const double* X, int q, const GeoTables& t, int ma, int mb, int mc, double* J)
{
  const int Q = q + 1;
#pragma unroll
  for (int i = 0; i < 9; ++i) J[i] = 0.;
  for (int k = 0; k < Q; ++k)
    for (int j = 0; j < Q; ++j)
      for (int i = 0; i < Q; ++i) {
        const double* x = X + 3 * (i + Q * (j + Q * k));
        const double g[3] = {mul(mul(t.d[ma][i], t.l[mb][j]), t.l[mc][k]),
                             mul(mul(t.l[ma][i], t.d[mb][j]), t.l[mc][k]),
                             mul(mul(t.l[ma][i], t.l[mb][j]), t.d[mc][k])};
        const double xr[3] = {x[0], x[1], x[2]};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) J[3 * r + c] = add(J[3 * r + c], mul(xr[r], g[c]));
      }
}

__device__ double det3_rn(const double* m)
{
  double s = mul(mul(m[0], m[4]), m[8]);
  s = add(s, mul(mul(m[1], m[5]), m[6]));
  s = add(s, mul(mul(m[2], m[3]), m[7]));
  s = sub(s, mul(mul(m[2], m[4]), m[6]));
  s = sub(s, mul(mul(m[1], m[3]), m[8]));
  return sub(s, mul(mul(m[0], m[5]), m[7]));
}

__device__ void inv3_rn(const double* m, double* o)
{
  const double id = __ddiv_rn(1., det3_rn(m));
  o[0] = mul(id, sub(mul(m[4], m[8]), mul(m[5], m[7])));
  o[1] = mul(id, sub(mul(m[2], m[7]), mul(m[1], m[8])));
  o[2] = mul(id, sub(mul(m[1], m[5]), mul(m[2], m[4])));
  o[3] = mul(id, sub(mul(m[5], m[6]), mul(m[3], m[8])));
  o[4] = mul(id, sub(mul(m[0], m[8]), mul(m[2], m[6])));
  o[5] = mul(id, sub(mul(m[2], m[3]), mul(m[0], m[5])));
  o[6] = mul(id, sub(mul(m[3], m[7]), mul(m[4], m[6])));
  o[7] = mul(id, sub(mul(m[1], m[6]), mul(m[0], m[7])));
  o[8] = mul(id, sub(mul(m[0], m[4]), mul(m[1], m[3])));
}

// outward unit normal and surface Jacobian of face lf (host.cpp's face_normal:
// tangents are Jacobian columns, x faces (y,z), y faces (z,x), z faces (x,y),
// low faces flipped)
__device__ void face_normal_rn(const double* J, int lf, double* n, double* fj)
{
  const int a = lf >> 1;
  const int c1 = a == 0 ? 1 : a == 1 ? 2 : 0;
  const int c2 = a == 0 ? 2 : a == 1 ? 0 : 1;
  const double ts[3] = {J[c1], J[3 + c1], J[6 + c1]};
  const double tt[3] = {J[c2], J[3 + c2], J[6 + c2]};
  const double c[3] = {sub(mul(ts[1], tt[2]), mul(ts[2], tt[1])), sub(mul(ts[2], tt[0]), mul(ts[0], tt[2])),
                       sub(mul(ts[0], tt[1]), mul(ts[1], tt[0]))};
  const double f = __dsqrt_rn(add(add(mul(c[0], c[0]), mul(c[1], c[1])), mul(c[2], c[2])));
  *fj = f;
  const double sg = (lf & 1) ? 1. : -1.;
#pragma unroll
  for (int r = 0; r < 3; ++r) n[r] = __ddiv_rn(mul(sg, c[r]), f);
}

struct GeoStatus {
  int singular;  // first element whose centre Jacobian is singular
  int curved;    // some element's Jacobian is not constant
  int nonpos;    // first element with a non-positive determinant at a volume point
  int face;      // first 6 e + lf whose face does not match its neighbour's
};

// every block copies the 1D tables (about 1.5 KB) into shared memory
__device__ void load_tables(const GeoTables* __restrict__ g, GeoTables& s)
{
  const double* src = reinterpret_cast<const double*>(g);
  double* dst = reinterpret_cast<double*>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(GeoTables) / sizeof(double)); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// The affine record of each element (Jacobian at the centre, table row P + 2)
// and the singular check.
__global__ void geo_element_kernel(const double* __restrict__ nodes, int q, int P, long E, const GeoTables* __restrict__ tab,
                                   double* __restrict__ geo, GeoStatus* st)
{
  __shared__ GeoTables t;
  load_tables(tab, t);
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= E) return;
  const int Q = q + 1;
  const double* X = nodes + (size_t)e * Q * Q * Q * 3;
  double J0[9];
  jacobian_at(X, q, t, P + 2, P + 2, P + 2, J0);
  double* g = geo + (size_t)e * kGeoStride;
  const double dJ = det3_rn(J0);
  if (!(fabs(dJ) > 0.) || !isfinite(dJ)) atomicMin(&st->singular, (int)e);
  inv3_rn(J0, g + kGeoJinv);
  g[kGeoDetJ] = dJ;
  for (int lf = 0; lf < 6; ++lf) face_normal_rn(J0, lf, g + kGeoN + 3 * lf, g + kGeoFJ + lf);
  for (int c = kGeoFJ + 6; c < kGeoStride; ++c) g[c] = 0.;
}

// The affinity check: the Jacobian at every volume point and corner against
// the centre's, relative to the centre's largest entry.
__global__ void geo_affinity_kernel(const double* __restrict__ nodes, int q, int P, long E, const GeoTables* __restrict__ tab,
                                    GeoStatus* st)
{
  __shared__ GeoTables t;
  load_tables(tab, t);
  const int NB = P * P * P, npts = NB + 8;
  const long id = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (id >= E * npts) return;
  const long e = id / npts;
  const int s = (int)(id - e * npts);
  const int Q = q + 1;
  const double* X = nodes + (size_t)e * Q * Q * Q * 3;
  int ma, mb, mc;
  if (s < NB) {
    ma = s % P;
    mb = (s / P) % P;
    mc = s / (P * P);
  } else {
    const int c = s - NB;
    ma = P + (c & 1);
    mb = P + ((c >> 1) & 1);
    mc = P + ((c >> 2) & 1);
  }
  double J0[9], J[9];
  jacobian_at(X, q, t, P + 2, P + 2, P + 2, J0);
  double scale = 0.;
  for (int i = 0; i < 9; ++i) scale = fmax(scale, fabs(J0[i]));
  jacobian_at(X, q, t, ma, mb, mc, J);
  bool bent = false;
  for (int i = 0; i < 9; ++i) bent = bent || fabs(J[i] - J0[i]) > 1e-11 * scale;
  if (bent) atomicExch(&st->curved, 1);
}

// Per-point volume geometry of curved elements (host.cpp's curved_element).
__global__ void geo_volume_kernel(const double* __restrict__ nodes, int q, int P, long E, const GeoTables* __restrict__ tab,
                                  double* __restrict__ gv, GeoStatus* st)
{
  __shared__ GeoTables t;
  load_tables(tab, t);
  const int NB = P * P * P;
  const long id = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (id >= E * NB) return;
  const long e = id / NB;
  const int b = (int)(id - e * NB);
  const int Q = q + 1;
  const double* X = nodes + (size_t)e * Q * Q * Q * 3;
  double J[9], Ji[9];
  jacobian_at(X, q, t, b % P, (b / P) % P, b / (P * P), J);
  const double dJ = det3_rn(J);
  if (!(dJ > 0.) || !isfinite(dJ)) atomicMin(&st->nonpos, (int)e);
  inv3_rn(J, Ji);
  double* g = gv + (size_t)e * kVolC * NB;
  for (int c = 0; c < 9; ++c) g[c * NB + b] = Ji[c];
  g[kVolDetJ * NB + b] = dJ;
}

// Per-point face geometry of curved elements; the lifting scale reads the
// volume determinants geo_volume_kernel wrote.
__global__ void geo_face_kernel(const double* __restrict__ nodes, int q, int P, long E, const GeoTables* __restrict__ tab,
                                const double* __restrict__ gv, double* __restrict__ gf)
{
  __shared__ GeoTables t;
  load_tables(tab, t);
  const int NB = P * P * P, NQF = P * P;
  const long id = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (id >= E * 6 * NQF) return;
  const long ef = id / NQF;  // 6 e + lf
  const int fq = (int)(id - ef * NQF);
  const long e = ef / 6;
  const int lf = (int)(ef - 6 * e);
  const int a = lf >> 1, end = lf & 1, t1 = fq % P, t2 = fq / P;
  int m[3];
  m[a] = P + end;
  m[a == 0 ? 1 : 0] = t1;
  m[a == 2 ? 1 : 2] = t2;
  const int Q = q + 1;
  const double* X = nodes + (size_t)e * Q * Q * Q * 3;
  double J[9], Ji[9], n[3], fj;
  jacobian_at(X, q, t, m[0], m[1], m[2], J);
  inv3_rn(J, Ji);
  face_normal_rn(J, lf, n, &fj);
  double* g = gf + (size_t)ef * kFaceC * NQF;
  for (int c = 0; c < 9; ++c) g[c * NQF + fq] = Ji[c];
  for (int c = 0; c < 3; ++c) g[(kFaceN + c) * NQF + fq] = n[c];
  g[kFaceFJ * NQF + fq] = fj;
  const double* dJ = gv + ((size_t)e * kVolC + kVolDetJ) * NB;
  double lift = 0.;
  for (int ia = 0; ia < P; ++ia) {
    const int b = a == 0 ? ia + P * (t1 + P * t2) : a == 1 ? t1 + P * (ia + P * t2) : t1 + P * (t2 + P * ia);
    lift = add(lift, __ddiv_rn(mul(t.EL[end][ia], t.EL[end][ia]), mul(t.w[ia], dJ[b])));
  }
  g[kFaceLift * NQF + fq] = lift;
}

// The two sides of every interior face see the same face: opposite unit
// normals and equal surface Jacobians, per element (affine) or per point.
__global__ void geo_match_kernel(const int32_t* __restrict__ nbr, long E, int NQF, const double* __restrict__ geo,
                                 const double* __restrict__ gf, GeoStatus* st)
{
  const int per = gf ? NQF : 1;
  const long id = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (id >= E * 6 * per) return;
  const long ef = id / per;
  const int fq = (int)(id - ef * per);
  const int en = nbr[ef];
  if (en < 0) return;
  const long e = ef / 6;
  const int lf = (int)(ef - 6 * e), lo = lf ^ 1;
  bool bad;
  if (gf) {
    const double* g = gf + (size_t)ef * kFaceC * NQF;
    const double* h = gf + ((size_t)en * 6 + lo) * kFaceC * NQF;
    bad = face_mismatch(g + kFaceN * NQF + fq, h + kFaceN * NQF + fq, NQF, g[kFaceFJ * NQF + fq],
                        h[kFaceFJ * NQF + fq]);
  } else {
    const double* g = geo + (size_t)e * kGeoStride;
    const double* h = geo + (size_t)en * kGeoStride;
    bad = face_mismatch(g + kGeoN + 3 * lf, h + kGeoN + 3 * lo, 1, g[kGeoFJ + lf], h[kGeoFJ + lo]);
  }
  if (bad) atomicMin(&st->face, (int)ef);
}

unsigned blocks(long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

int build_geometry_device(const dgb_mesh_desc& m, const Ops1D& ops, const std::vector<int32_t>& nbr,
                          const int32_t* d_nbr, void* stream, double* d_geo, double** d_gv, double** d_gf,
                          bool& curved, std::string& why)
{
  curved = false;
  int rc = check_mesh(m, why);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int q = m.q, P = ops.P, Q = q + 1, NB = P * P * P, NQF = P * P;
  const long E = (long)m.nx * m.ny * m.nz;
  const size_t nodes_bytes = sizeof(double) * (size_t)E * Q * Q * Q * 3;
  GeoTables t;
  build_geo_tables(ops, q, t);
  double* d_nodes = nullptr;
  GeoStatus* d_st = nullptr;
  GeoTables* d_t = nullptr;
  GeoStatus hs = {INT_MAX, 0, INT_MAX, INT_MAX};
  const int TB = 128;
  cudaError_t e = cudaSuccess;
  const char* what = "";
#define GEO_CK(call)      \
  do {                    \
    e = (call);           \
    if (e != cudaSuccess) { \
      what = #call;       \
      goto done;          \
    }                     \
  } while (0)
  GEO_CK(cudaMalloc(&d_nodes, nodes_bytes));
  GEO_CK(cudaMalloc(&d_st, sizeof(GeoStatus)));
  GEO_CK(cudaMalloc(&d_t, sizeof(GeoTables)));
  GEO_CK(cudaMemcpyAsync(d_t, &t, sizeof t, cudaMemcpyHostToDevice, st));
  GEO_CK(cudaMemcpyAsync(d_nodes, m.nodes, nodes_bytes, cudaMemcpyHostToDevice, st));
  GEO_CK(cudaMemcpyAsync(d_st, &hs, sizeof hs, cudaMemcpyHostToDevice, st));
  geo_element_kernel<<<blocks(E, TB), TB, 0, st>>>(d_nodes, q, P, E, d_t, d_geo, d_st);
  GEO_CK(cudaGetLastError());
  geo_affinity_kernel<<<blocks(E * (NB + 8), TB), TB, 0, st>>>(d_nodes, q, P, E, d_t, d_st);
  GEO_CK(cudaGetLastError());
  GEO_CK(cudaMemcpyAsync(&hs, d_st, sizeof hs, cudaMemcpyDeviceToHost, st));
  GEO_CK(cudaStreamSynchronize(st));
  if (hs.singular != INT_MAX) {
    char buf[120];
    snprintf(buf, sizeof buf, "element %d has a singular Jacobian", hs.singular);
    why = buf;
    rc = DGB_ERR_GEOMETRY;
    goto done;
  }
  curved = hs.curved != 0;
  if (curved) {
    GEO_CK(cudaMalloc(d_gv, sizeof(double) * (size_t)E * kVolC * NB));
    GEO_CK(cudaMalloc(d_gf, sizeof(double) * (size_t)E * 6 * kFaceC * NQF));
    geo_volume_kernel<<<blocks(E * NB, TB), TB, 0, st>>>(d_nodes, q, P, E, d_t, *d_gv, d_st);
    GEO_CK(cudaGetLastError());
    geo_face_kernel<<<blocks(E * 6 * NQF, TB), TB, 0, st>>>(d_nodes, q, P, E, d_t, *d_gv, *d_gf);
    GEO_CK(cudaGetLastError());
  }
  geo_match_kernel<<<blocks(E * 6 * (curved ? NQF : 1), TB), TB, 0, st>>>(d_nbr, E, NQF, d_geo,
                                                                          curved ? *d_gf : nullptr, d_st);
  GEO_CK(cudaGetLastError());
  GEO_CK(cudaMemcpyAsync(&hs, d_st, sizeof hs, cudaMemcpyDeviceToHost, st));
  GEO_CK(cudaStreamSynchronize(st));
  if (hs.nonpos != INT_MAX) {
    char buf[120];
    snprintf(buf, sizeof buf, "element %d has a non-positive Jacobian determinant", hs.nonpos);
    why = buf;
    rc = DGB_ERR_GEOMETRY;
  } else if (hs.face != INT_MAX) {
    char buf[160];
    snprintf(buf, sizeof buf, "face %d of element %d does not match its neighbour %d", hs.face % 6, hs.face / 6,
             nbr[hs.face]);
    why = buf;
    rc = DGB_ERR_GEOMETRY;
  }
done:
#undef GEO_CK
  if (d_nodes) cudaFree(d_nodes);
  if (d_st) cudaFree(d_st);
  if (d_t) cudaFree(d_t);
  if (e != cudaSuccess) {
    why = std::string(what) + ": " + cudaGetErrorString(e);
    return DGB_ERR_CUDA;
  }
  return rc;
}

}  // namespace dgb
