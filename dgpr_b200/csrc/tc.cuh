// The mixed form's Gauss-point stage with its volume contractions on the
// 5th-generation tensor cores (tcgen05, kind::tf32, accumulators in tensor
// memory).  Everything else (the pointwise volume flux, the face phase, the
// norm, the FP64 RK update and the next stage's traces) is the FP32 stage
// kernel's own code (vspace.cuh), so the two differ only in how the six
// sum-factorised contractions of the volume integral are computed.
//
// The contractions (solve_cuda.cu:344-491 computes them as dense products
// with the reference's vgrad tables; the Gauss-point form has them as 1D
// operators along each axis):
//   gradient   G_d[r][o] = sum_k Dq[a_d(o)][k]  V[r][o + (k - a_d(o)) S_d]
//   test       Y  [r][o] = sum_d sum_k Dq[k][a_d(o)] Ghat_d[r][o + (k - a_d(o)) S_d]
// For direction d each is one matrix product D = A B with the rows
// m = r P^2 + (the other two coordinates of the point), K = the coordinate
// along d (P <= 8 of the instruction's 8) and N = the P outputs along d
// (padded to 16): M = 5 P^2 <= 128 rows, so one M = 128 instruction per
// direction and precision term.  FP32 accuracy comes from three TF32
// products per contraction (hi/lo split of both operands, the lo x lo term
// dropped: relative error about 2^-21 per product), accumulated in FP32.
//
// Shared-memory operands are in the canonical K-major layout without
// swizzle: 8-row by 16-byte core matrices, rows 16 bytes apart, 8-row blocks
// 128 bytes apart (the descriptor's stride offset) and the two 16-byte K
// chunks of an instruction `lbo` apart (its leading offset).  With P <= 4 the
// second chunk of every A tile is the one shared zero chunk.  One thread
// issues the 9 instructions of a contraction (3 directions x 3 terms) and a
// commit to an mbarrier; the CTA's four warps wait on it (bounded: a wait
// that gives up sets bit 16 of the status word) and read the accumulator rows
// of their lane quadrant with tcgen05.ld.  CTAs have 128 threads, as the
// four lane quadrants of an M = 128 accumulator need.
#pragma once

#include <cstdint>

#include "vspace.cuh"

namespace dgb {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// round to TF32 (10 explicit mantissa bits), nearest with ties away from zero
__device__ __forceinline__ float tf32(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// shared-memory matrix descriptor: no swizzle, byte offsets lbo (between the
// K chunks) and sbo (between 8-row blocks), descriptor version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), A
// and B TF32 (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4
// at bit 24
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_tf32()
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void alloc(uint32_t* dst, uint32_t ncols)  // one whole warp
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols)  // the warp that allocated
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes of shared memory made visible to the tensor core's reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on the mbarrier when every tcgen05.mma this thread issued has completed
__device__ __forceinline__ void commit(uint64_t* bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// wait for the completion of the mbarrier phase of this parity, at most
// `limit` polls; false when it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long limit)
{
  const uint32_t a = smem_addr(bar);
  for (long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 4 or 8 consecutive FP32 accumulator columns of this thread's lane; the
// wait inside takes the values as operands so nothing reads them before it
template <int X>
__device__ __forceinline__ void ld_cols(uint32_t taddr, float* v)
{
  uint32_t r[8];
  if constexpr (X == 4) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])::"memory");
  } else {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])::"memory");
  }
#pragma unroll
  for (int i = 0; i < X; ++i) v[i] = __uint_as_float(r[i]);
}

// byte offset of element (row m, k) in a K-major tile of 8-row blocks 128
// bytes apart and K chunks `lbo` apart
__device__ __forceinline__ int kmajor_off(int m, int k, int lbo)
{
  return (m >> 3) * 128 + (k >> 2) * lbo + (m & 7) * 16 + (k & 3) * 4;
}

// the row and K index of variable r at Gauss point o in direction d's
// contraction: rows r P^2 + (the two other coordinates, lower axis fastest)
template <int P>
__device__ __forceinline__ void row_of(int d, int r, int o, int& m, int& k)
{
  const int x = o % P, y = (o / P) % P, z = o / (P * P);
  m = r * P * P + (d == 0 ? y + P * z : d == 1 ? x + P * z : x + P * y);
  k = d == 0 ? x : d == 1 ? y : z;
}

// the Gauss point of row m's output column a in direction d
template <int P>
__device__ __forceinline__ int point_of(int d, int m, int a)
{
  const int j = m % (P * P), c1 = j % P, c2 = j / P;
  return d == 0 ? a + P * c1 + P * P * c2 : d == 1 ? c1 + P * a + P * P * c2 : c1 + P * c2 + P * P * a;
}

}  // namespace tc

constexpr int kTcThreads = 128;
constexpr int kTcCols = 64;       // tensor-memory columns: 3 directions x 16
constexpr long kTcWaitLimit = 1L << 22;
constexpr int kTcTimeoutFlag = 16;

template <int P>
struct TcSmem {
  using S = VStageSmem<P, float, kTcThreads>;
  static constexpr int NCH = (P + 3) / 4;  // 16-byte K chunks holding data
  static constexpr int CHUNK = 2048;       // one K chunk of 128 rows
  static constexpr int TILE = NCH * CHUNK;
  static constexpr int oT = (S::TOTAL + 127) & ~127;  // A tiles [direction][hi, lo]
  static constexpr int oZ = oT + 6 * TILE;            // the zero chunk (P <= 4)
  static constexpr int oB = oZ + (NCH == 1 ? CHUNK : 0);  // B tiles: gradient hi, lo; test hi, lo
  static constexpr int BT = 512;                          // 16 rows x 2 chunks
  static constexpr int oBar = oB + 4 * BT;                // mbarrier, tensor-memory address
  static constexpr int TOTAL = oBar + 16;
  // resident CTAs the shared memory allows (228 KB per SM, 1 KB reserved per
  // CTA), at most 8: 8 x 64 tensor-memory columns fill the SM's 512
  static constexpr int BY_SMEM = 228 * 1024 / (TOTAL + 1024);
  static constexpr int MIN_BLOCKS = BY_SMEM > 8 ? 8 : BY_SMEM;
  static_assert(5 * P * P <= 128 && P <= 8, "one M = 128 instruction per direction");
};

// The FP32 Gauss-point stage (vstage_kernel<P, float, false, false>: affine
// elements, no heat flux) with the tensor-core volume contractions.
template <int P>
__global__ void __launch_bounds__(kTcThreads, TcSmem<P>::MIN_BLOCKS)
vstage_tc_kernel(long E, const double* Vs, const float* __restrict__ Tr, const float* __restrict__ opsg,
                 const double* __restrict__ opsd, const double* __restrict__ geo, const int* __restrict__ nbr,
                 DevParams prm, StageArgs sa)
{
  using T = float;
  using C = Cfg<P>;
  using TL = TcSmem<P>;
  using L = typename TL::S;
  constexpr int NB = C::NB, NQF = C::NQF, NX = P <= 4 ? 4 : 8;
  constexpr int TILE = TL::TILE;
  constexpr uint32_t IDESC = tc::idesc_tf32<128, 16>();
  extern __shared__ __align__(16) unsigned char smraw[];
  T* so = reinterpret_cast<T*>(smraw + L::oOps);
  T* sg = reinterpret_cast<T*>(smraw + L::oGeo);
  unsigned char* sXb = smraw + L::oX;
  T* sX = reinterpret_cast<T*>(sXb);
  unsigned char* tiles = smraw + TL::oT;
  unsigned char* btiles = smraw + TL::oB;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw + TL::oBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smraw + TL::oBar + 8);
  const long e = sa.ebase + sa.estep * (long)blockIdx.x;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool node = tid < NB;
  const int qx = tid % P, qy = (tid / P) % P, qz = tid / (P * P);

  T* V1 = sX;
  T* G = sX + 5 * NB;
  if (DGB_PREFETCH_L2_F32) {
    prefetch_range(Tr + e * 60 * NQF, 60L * NQF * sizeof(T), tid, kTcThreads);
    if (tid < 6) {
      const int nb = nbr[e * 6 + tid];
      if (nb >= 0) prefetch_range(Tr + ((long)nb * 6 + (tid ^ 1)) * 10 * NQF, 10L * NQF * sizeof(T), 0, 1);
    }
    if (sa.Ubase) prefetch_range(sa.Ubase + e * 5 * NB, 40L * NB, tid, kTcThreads);
    if (sa.acc && sa.mode >= MODE_RK4_1 && sa.mode <= MODE_RK4_3)
      prefetch_range(sa.acc + e * 5 * NB, 40L * NB, tid, kTcThreads);
  }
  if (warp == 0) tc::alloc(tslot, kTcCols);
  if (tid == 0) tc::mbar_init(bar, 1);
  for (int i = tid; i < C::OPS; i += kTcThreads) so[i] = opsg[i];
  for (int i = tid; i < kGeoStride; i += kTcThreads) sg[i] = T(geo[e * kGeoStride + i]);
  const double* Ve = Vs + e * 5 * NB;
  for (int i = tid; i < 5 * NB; i += kTcThreads) V1[i] = T(Ve[i]);
  {  // zero the tiles: rows past 5 P^2, K past P, the zero chunk, the B padding
    float4* z = reinterpret_cast<float4*>(tiles);
    for (int i = tid; i < (TL::oBar - TL::oT) / 16; i += kTcThreads) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  // B operands, K-major (row n = output, K = input): gradient Dq[n][k], test Dq[k][n]
  for (int i = tid; i < P * P; i += kTcThreads) {
    const int n = i / P, k = i % P;
    const float g = so[C::oDq + n * P + k], t = so[C::oDq + k * P + n];
    const float gh = tc::tf32(g), th = tc::tf32(t);
    const int off = tc::kmajor_off(n, k, 256);
    *reinterpret_cast<float*>(btiles + 0 * TL::BT + off) = gh;
    *reinterpret_cast<float*>(btiles + 1 * TL::BT + off) = tc::tf32(g - gh);
    *reinterpret_cast<float*>(btiles + 2 * TL::BT + off) = th;
    *reinterpret_cast<float*>(btiles + 3 * TL::BT + off) = tc::tf32(t - th);
  }
  // A operands of the gradient: V split into hi and lo, one row layout per direction
  for (int i = tid; i < 5 * NB; i += kTcThreads) {
    const int r = i / NB, o = i % NB;
    const float v = V1[i], hi = tc::tf32(v), lo = tc::tf32(v - hi);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int m, k;
      tc::row_of<P>(d, r, o, m, k);
      const int off = tc::kmajor_off(m, k, TL::CHUNK);
      *reinterpret_cast<float*>(tiles + (2 * d) * TILE + off) = hi;
      *reinterpret_cast<float*>(tiles + (2 * d + 1) * TILE + off) = lo;
    }
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t a0 = tc::smem_addr(tiles), b0 = tc::smem_addr(btiles);
  // leading offset of A tile t: the zero chunk (P <= 4) or the tile's own second chunk
  auto lbo_a = [&](int t) -> uint32_t {
    return TL::NCH == 1 ? (uint32_t)(TL::oZ - TL::oT - t * TILE) : (uint32_t)TL::CHUNK;
  };
  auto issue = [&](int bsel) {  // 3 directions x (lo hi + hi lo + hi hi)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const uint32_t dcol = tmem + 16u * d;
      const uint64_t ahi = tc::sdesc(a0 + (2 * d) * TILE, lbo_a(2 * d), 128);
      const uint64_t alo = tc::sdesc(a0 + (2 * d + 1) * TILE, lbo_a(2 * d + 1), 128);
      const uint64_t bhi = tc::sdesc(b0 + (2 * bsel) * TL::BT, 256, 128);
      const uint64_t blo = tc::sdesc(b0 + (2 * bsel + 1) * TL::BT, 256, 128);
      tc::mma(dcol, alo, bhi, IDESC, 0);
      tc::mma(dcol, ahi, blo, IDESC, 1);
      tc::mma(dcol, ahi, bhi, IDESC, 1);
    }
    tc::commit(bar);
  };
  const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's lane quadrant
  const int m = 32 * warp + lane;                                // the accumulator row of this thread
  bool ok = true;

  // ---------------- reference gradients on the tensor cores
  if (tid == 0) issue(0);
  ok = tc::mbar_wait(bar, 0, kTcWaitLimit);
  tc::fence_after();
  {
    float g[3][NX];
#pragma unroll
    for (int d = 0; d < 3; ++d) tc::ld_cols<NX>(trow + 16u * d, g[d]);
    if (m < 5 * P * P) {
      const int r = m / (P * P);
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < P; ++a) G[d * 5 * NB + r * NB + tc::point_of<P>(d, m, a)] = g[d][a];
    }
  }
  tc::fence_before();
  __syncthreads();

  // ---------------- pointwise flux, written as the test contraction's A operands
  const T* Ji = sg + kGeoJinv;
  const T detJ = sg[kGeoDetJ];
  const T gamma = T(prm.gamma), mu = T(prm.mu), kq = T(0);
  T wJq = T(0);
  if (node)
    wJq = vpoint_flux<P, T, false, false>(so, V1, G, Ji, detJ, nullptr, gamma, mu, kq, tid, [&](int i, int r, T v) {
      int mm, k;
      tc::row_of<P>(i, r, tid, mm, k);
      const int off = tc::kmajor_off(mm, k, TL::CHUNK);
      const float hi = tc::tf32(v);
      *reinterpret_cast<float*>(tiles + (2 * i) * TILE + off) = hi;
      *reinterpret_cast<float*>(tiles + (2 * i + 1) * TILE + off) = tc::tf32(v - hi);
    });
  tc::fence_async_smem();
  __syncthreads();
  tc::fence_after();

  // ---------------- Y = sum_i Dq_i^T Ghat_i on the tensor cores
  if (tid == 0) issue(1);
  ok = tc::mbar_wait(bar, 1, kTcWaitLimit) && ok;
  tc::fence_after();
  T* Yd = G;  // [3][5][NB]: the gradients are no longer read
  {
    float y[3][NX];
#pragma unroll
    for (int d = 0; d < 3; ++d) tc::ld_cols<NX>(trow + 16u * d, y[d]);
    if (m < 5 * P * P) {
      const int r = m / (P * P);
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < P; ++a) Yd[d * 5 * NB + r * NB + tc::point_of<P>(d, m, a)] = y[d][a];
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::dealloc(tmem, kTcCols);
  }
  if (!ok && lane == 0) atomicOr(sa.flag, kTcTimeoutFlag);
  T Rv[5] = {T(0), T(0), T(0), T(0), T(0)};
  if (node) {  // the same association as the FP32 stage kernel: (Y_0 + Y_1) + Y_2 - source
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      Rv[r] = Yd[r * NB + tid];
      Rv[r] += Yd[5 * NB + r * NB + tid];
      Rv[r] = Rv[r] + Yd[10 * NB + r * NB + tid] - T(prm.src[r]) * wJq;
    }
  }
  __syncthreads();

  const double detJd = geo[e * kGeoStride + kGeoDetJ];
  vstage_faces<P, T, false>(e, Tr, nbr, so, sg, sX, geo, nullptr, nullptr, prm, gamma, mu, kq, detJ, Ji, sa.flag,
                            node, qx, qy, qz, Rv);
  vstage_finish<P, T, false, L>(e, sa, Rv, Ve, nullptr, detJd, sXb, so, sg, opsd, mu, kq, nullptr, node, qx, qy, qz);
}

}  // namespace dgb
