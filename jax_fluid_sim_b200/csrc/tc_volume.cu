// Inviscid volume integrals of prism and tetrahedron blocks on the 5th-generation tensor cores
// (tcgen05, kind::tf32 with a three-term split: about float32 accuracy).
//
// The reference evaluates the volume term of every element as two dense contractions against
// the block's shared basis tables (hybrid/spatial.py:47-72):
//   U_q   = sum_i B[q][i] U_i                                   (nodes -> volume points)
//   R_i   = sum_q sum_r dB[q][i][r] G_r(q),  G_r = w|J| sum_d J^-1[r][d] (F_d(U_q) - F_d(anchor))
// Both are GEMMs with one constant operand shared by all elements of the block and a streamed
// operand with one column per (element, variable).  Here a CTA works on tiles of Te elements:
//   GEMM 1: D1 (128 points x Te*NV) = A1 (128 points x Np) . X (Np x Te*NV), X = U - anchor;
//   the flux at each point is evaluated from D1 (TMEM lane q = point q) on the CUDA cores and
//   contracted with the metrics into G_r (r = 0, 1, 2);
//   GEMM 2: D2 (Np nodes x Te*NV) += A2_r (Np x 128 points) . G_r (128 points x Te*NV).
// Every operand is split hi + lo (hi = the value rounded to tf32, lo = the remainder rounded to tf32)
// and each product is summed as hi.hi + hi.lo + lo.hi in float32, which gives about 2^-21 relative
// error per product (3xTF32), against 2^-24 for float32 arithmetic.
//
// Data movement: the constant A1/A2 images (packed once per plan by k_tc_pack) and each tile's
// element states (Te consecutive elements are one contiguous run of the state) are copied into
// shared memory by the bulk-copy engine (cp.async.bulk with mbarrier transaction counts); the
// tensor cores read the operands from shared memory and accumulate in tensor memory; the epilogue
// reads TMEM with tcgen05.ld.  Only this GPU's own memory is read (no cluster multicast).
//
// Shared-memory operand layouts (canonical, no swizzle):
//   A (K-major): core matrices of 8 rows x 4 values (128 B), [k/4][row/8][row%8][k%4];
//                LBO = stride between k/4 blocks, SBO = 128 B between row groups.
//   B (K-major as well): core matrices of 8 columns x 4 k, [k/4][col/8][col%8][k%4];
//                LBO = stride between k/4 blocks, SBO = 128 B between column groups.
// (An MN-major B with no swizzle read as zeros on this hardware; both operands are K-major.)
// A2 holds only the ceil(Np/8) real row groups of each k/4 block; the MMA's rows beyond them read
// the next block's data (in bounds: the B region follows A2) and land in TMEM lanes that are
// never read.
//
// Every wait on an mbarrier is bounded; on a time-out the CTA records DGB_DEVICE_TIMEOUT in the
// error word, waits (bounded) for its own operations in flight, frees its TMEM and returns.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dg_kernels.cuh"
#include "tc_volume.h"

namespace dgb {

namespace {

constexpr int kTcThreads = 256;          // 8 warps: lane quarter = warp % 4, element half = warp / 4
constexpr int kTcTe = 8;                 // elements per tile
constexpr int kTcNV = 5;                 // conserved variables (flow only)
constexpr long long kWaitCycles = 4000000000LL;   // about 2 s at the boost clock

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// true once the phase of parity `parity` has completed; false after about kWaitCycles
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// smem matrix descriptor, no swizzle (layout type 0), descriptor version 1 at bits 46-48
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// D[tmem] (+)= A . B, kind::tf32, M = 128, A and B K-major, f32 accumulate
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float* v) {
  uint32_t r0, r1, r2, r3;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(taddr));
  v[0] = __uint_as_float(r0);
  v[1] = __uint_as_float(r1);
  v[2] = __uint_as_float(r2);
  v[3] = __uint_as_float(r3);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x rounded to the nearest tf32 value (10 explicit mantissa bits; ties away from zero): add half
// of the dropped unit, then clear the 13 low bits
__device__ __forceinline__ float tf32_round(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
// the two tf32 terms of x: hi = round(x), lo = round(x - hi) (x - hi is exact in float32); hi + lo
// represents x to about 2^-22 relative
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
  hi = tf32_round(x);
  lo = tf32_round(x - hi);
}

__host__ __device__ inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

}  // namespace

TcShape tc_shape(int Np, int Nq, int nv) {
  TcShape s{};
  s.Np = Np;
  s.Nq = Nq;
  s.Te = kTcTe;
  s.Kp1 = round_up(Np, 8);
  s.Kq = round_up(Nq, 8);
  s.G8 = (Np + 7) / 8;
  s.N1 = round_up(kTcNV * kTcTe, 16);
  s.a1_floats = 128 * s.Kp1;
  s.a2_floats = 8 * s.Kq * s.G8;
  s.image_floats = 2 * s.a1_floats + 6 * s.a2_floats;
  const size_t b1 = sizeof(float) * 2 * (size_t)s.N1 * s.Kp1;
  const size_t stage = sizeof(double) * (size_t)kTcTe * Np * kTcNV;
  const size_t b2 = sizeof(float) * 2 * (size_t)s.N1 * s.Kq;
  s.b_offset = sizeof(float) * s.image_floats;
  s.stage_offset = s.b_offset + b1;
  const size_t bregion = b2 > b1 + stage ? b2 : b1 + stage;
  s.smem = s.b_offset + bregion;
  // the A2 rows past Np read up to (16 - G8) row groups of 128 B beyond the last A2 buffer
  s.eligible = nv == kTcNV && Np % 2 == 0 && Np <= 40 && Nq <= 128 && bregion >= (size_t)(16 - s.G8) * 128 &&
               s.smem + 2048 <= 227 * 1024;   // static shared memory of the kernel: about 1.2 KB
  return s;
}

// Packs A1 (basis at the volume points, rows q) and A2_r (derivatives, rows i) hi/lo for one block.
__global__ void k_tc_pack(const double* __restrict__ B, const double* __restrict__ dB, TcShape s, float* image) {
  const int total = s.image_floats;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int part, off;
    if (t < 2 * s.a1_floats) {
      part = t / s.a1_floats;          // 0 hi, 1 lo
      off = t % s.a1_floats;
      // off = ((k/4) * 16 + m/8) * 32 + (m%8) * 4 + k%4
      const int core = off / 32, in = off % 32;
      const int kb = core / 16, g = core % 16;
      const int m = g * 8 + in / 4, k = kb * 4 + in % 4;
      const float x = (m < s.Nq && k < s.Np) ? (float)B[(size_t)m * s.Np + k] : 0.0f;
      float hi, lo;
      tf32_split(x, hi, lo);
      image[t] = part == 0 ? hi : lo;
    } else {
      const int u = t - 2 * s.a1_floats;
      const int buf = u / s.a2_floats;  // r * 2 + (0 hi, 1 lo)
      const int r = buf / 2;
      part = buf % 2;
      off = u % s.a2_floats;
      // off = ((k/4) * G8 + m/8) * 32 + (m%8) * 4 + k%4
      const int core = off / 32, in = off % 32;
      const int kb = core / s.G8, g = core % s.G8;
      const int m = g * 8 + in / 4, k = kb * 4 + in % 4;
      const float x = (m < s.Np && k < s.Nq) ? (float)dB[((size_t)k * s.Np + m) * 3 + r] : 0.0f;
      float hi, lo;
      tf32_split(x, hi, lo);
      image[t] = part == 0 ? hi : lo;
    }
  }
}

// Inviscid volume residuals of one block (precision mode 1), written to B.Rinv [E][Np][NV].
__global__ void __launch_bounds__(kTcThreads, 1) k_tc_volume(const DevPlan P, const StatePtrs S, int b, TcShape s,
                                                            const float* __restrict__ image, int* err) {
  constexpr int NV = kTcNV, Te = kTcTe, HALF = Te / 2;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t bar_tma, bar_mma;
  __shared__ uint32_t tmem_base;
  __shared__ double anchor[Te][NV];
  __shared__ float fa[Te][3][NV];
  __shared__ float ajac[Te][10];          // affine: J^-1 (9) and |det J|
  __shared__ int aff[Te];
  const BlockDev& B = P.blk[b];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, half = warp >> 2;
  const int Np = s.Np, Nq = s.Nq, N1 = s.N1;
  const int ntiles = (B.E + Te - 1) / Te;
  float* A1 = reinterpret_cast<float*>(tc_smem);
  float* A2 = A1 + 2 * s.a1_floats;
  float* Bm = reinterpret_cast<float*>(tc_smem + s.b_offset);
  const double* stage = reinterpret_cast<const double*>(tc_smem + s.stage_offset);
  const uint32_t ncols = 2 * N1 <= 32 ? 32 : (2 * N1 <= 64 ? 64 : (2 * N1 <= 128 ? 128 : 256));
  if (tid == 0) {
    mbar_init(&bar_tma, 1);
    mbar_init(&bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_base;
  const uint32_t d1 = tbase, d2 = tbase + ncols / 2;
  // instruction descriptor: f32 accumulate, tf32 A and B, both K-major, N = N1, M = 128
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N1 >> 3) << 17) |
                         ((uint32_t)(128 >> 4) << 24);
  const uint32_t a1_lbo = 16 * 128, a2_lbo = (uint32_t)s.G8 * 128, b_lbo = (uint32_t)(N1 / 8) * 128;
  uint32_t tma_phase = 0, mma_phase = 0;
  if (tid == 0) {
    mbar_expect_tx(&bar_tma, (uint32_t)(sizeof(float) * s.image_floats));
    bulk_g2s(A1, image, (uint32_t)(sizeof(float) * s.image_floats), &bar_tma);
  }
  bool ok = mbar_wait(&bar_tma, tma_phase);
  tma_phase ^= 1;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int e0 = tile * Te;
    const int ne = B.E - e0 < Te ? B.E - e0 : Te;
    const double* Ug = S.b[b] + (size_t)e0 * Np * NV;
    if (tid == 0) {
      const uint32_t bytes = (uint32_t)(sizeof(double) * (size_t)ne * Np * NV);
      mbar_expect_tx(&bar_tma, bytes);
      bulk_g2s(const_cast<double*>(stage), Ug, bytes, &bar_tma);
    }
    // per-element constants: anchor (node 0), anchor fluxes, affine metrics
    if (tid < Te) {
      const int e = tid;
      if (e < ne) {
        const size_t ee = (size_t)e0 + e;
        float a[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          anchor[e][v] = Ug[(size_t)e * Np * NV + v];
          a[v] = (float)anchor[e][v];
        }
        const float ex[3] = {1.f, 0.f, 0.f}, ey[3] = {0.f, 1.f, 0.f}, ez[3] = {0.f, 0.f, 1.f};
        normal_flux<NV>(P.ph, a, ex, fa[e][0]);
        normal_flux<NV>(P.ph, a, ey, fa[e][1]);
        normal_flux<NV>(P.ph, a, ez, fa[e][2]);
        const int af = (B.affine != nullptr && B.affine[ee]) ? 1 : 0;
        aff[e] = af;
        if (af) {
#pragma unroll
          for (int k = 0; k < 9; ++k) ajac[e][k] = (float)B.ajinv[ee * 9 + k];
          ajac[e][9] = (float)B.adet[ee];
        }
      } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) anchor[e][v] = 0.0;
        aff[e] = 1;
        for (int k = 0; k < 10; ++k) ajac[e][k] = 0.f;
        for (int d = 0; d < 3; ++d)
          for (int v = 0; v < NV; ++v) fa[e][d][v] = 0.f;
      }
    }
    ok = mbar_wait(&bar_tma, tma_phase);
    tma_phase ^= 1;
    __syncthreads();
    // X = U - anchor (float64 difference, then float32) into B1 hi/lo, K-major; column n = v*Te + e
    {
      float* B1h = Bm;
      float* B1l = Bm + N1 * s.Kp1;
      const int kquads = s.Kp1 / 4;
      for (int t = tid; t < kquads * N1; t += kTcThreads) {
        const int n = t % N1, kb = t / N1;          // column n, nodes 4kb..4kb+3
        const int v = n / Te, e = n % Te;
        float hp[4], lp[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int k = kb * 4 + c;
          float x = 0.f;
          if (v < NV && e < ne && k < Np) x = (float)(stage[((size_t)e * Np + k) * NV + v] - anchor[e][v]);
          tf32_split(x, hp[c], lp[c]);
        }
        const int off = (kb * (N1 / 8) + n / 8) * 32 + (n % 8) * 4;
        *reinterpret_cast<float4*>(B1h + off) = make_float4(hp[0], hp[1], hp[2], hp[3]);
        *reinterpret_cast<float4*>(B1l + off) = make_float4(lp[0], lp[1], lp[2], lp[3]);
      }
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0 && ok) {
      tc_fence_after();
      const uint32_t a1h = smem_u32(A1), a1l = a1h + sizeof(float) * s.a1_floats;
      const uint32_t b1h = smem_u32(Bm), b1l = b1h + sizeof(float) * N1 * s.Kp1;
      for (int ks = 0; ks < s.Kp1 / 8; ++ks) {
        const uint32_t ao = ks * 2 * a1_lbo, bo = ks * 2 * b_lbo;
        mma_tf32(d1, smem_desc(a1h + ao, a1_lbo, 128), smem_desc(b1h + bo, b_lbo, 128), idesc, ks > 0);
        mma_tf32(d1, smem_desc(a1h + ao, a1_lbo, 128), smem_desc(b1l + bo, b_lbo, 128), idesc, 1);
        mma_tf32(d1, smem_desc(a1l + ao, a1_lbo, 128), smem_desc(b1h + bo, b_lbo, 128), idesc, 1);
      }
      mma_commit(&bar_mma);
    }
    ok = ok && mbar_wait(&bar_mma, mma_phase);
    mma_phase ^= 1;
    tc_fence_after();
    // this thread: volume point q (TMEM lane), elements half*HALF .. +HALF-1
    const int q = quarter * 32 + lane;
    float G[3][HALF][NV];
    {
      float uq[NV][HALF];
#pragma unroll
      for (int v = 0; v < NV; ++v)
        tmem_ld4(d1 + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(v * Te + half * HALF), uq[v]);
      tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < HALF; ++j) {
        const int e = half * HALF + j;
        float J[9], wq = 0.f;
        const bool live = q < Nq && e < ne;
        if (live) {
          if (aff[e]) {
#pragma unroll
            for (int k = 0; k < 9; ++k) J[k] = ajac[e][k];
            wq = (float)(B.wref[q] * (double)ajac[e][9]);
          } else {
            const size_t pq = ((size_t)e0 + e) * Nq + q;
#pragma unroll
            for (int k = 0; k < 9; ++k) J[k] = (float)B.jinv[pq * 9 + k];
            wq = (float)B.wdet[pq];
          }
        } else {
#pragma unroll
          for (int k = 0; k < 9; ++k) J[k] = 0.f;
        }
        float U[NV], F[3][NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) U[v] = (float)(anchor[e][v] + (double)uq[v][j]);
        const float ex[3] = {1.f, 0.f, 0.f}, ey[3] = {0.f, 1.f, 0.f}, ez[3] = {0.f, 0.f, 1.f};
        normal_flux<NV>(P.ph, U, ex, F[0]);
        normal_flux<NV>(P.ph, U, ey, F[1]);
        normal_flux<NV>(P.ph, U, ez, F[2]);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int v = 0; v < NV; ++v)
            G[r][j][v] = live ? (J[r * 3 + 0] * (F[0][v] - fa[e][0][v]) + J[r * 3 + 1] * (F[1][v] - fa[e][1][v]) +
                                 J[r * 3 + 2] * (F[2][v] - fa[e][2][v])) * wq
                              : 0.f;
      }
    }
    const int Kq = s.Kq;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      if (r > 0) {
        // the previous GEMM 2 pass still reads B2
        ok = ok && mbar_wait(&bar_mma, mma_phase);
        mma_phase ^= 1;
      }
      if (q < Kq) {
        // K-major: element (n, k = q) at ((q/4) * N1/8 + n/8) * 32 + (n%8) * 4 + q%4
        float* B2h = Bm;
        float* B2l = Bm + N1 * Kq;
        const int kb = (q / 4) * (N1 / 8) * 32 + q % 4;
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int j = 0; j < HALF; ++j) {
            const int n = v * Te + half * HALF + j;
            float hi, lo;
            tf32_split(G[r][j][v], hi, lo);
            B2h[kb + (n / 8) * 32 + (n % 8) * 4] = hi;
            B2l[kb + (n / 8) * 32 + (n % 8) * 4] = lo;
          }
        if (half == 0)
          for (int n = NV * Te; n < N1; ++n) {
            B2h[kb + (n / 8) * 32 + (n % 8) * 4] = 0.f;
            B2l[kb + (n / 8) * 32 + (n % 8) * 4] = 0.f;
          }
      }
      fence_async_smem();
      __syncthreads();
      if (tid == 0 && ok) {
        tc_fence_after();
        const uint32_t a2h = smem_u32(A2) + (uint32_t)(sizeof(float) * (2 * r) * s.a2_floats);
        const uint32_t a2l = a2h + (uint32_t)(sizeof(float) * s.a2_floats);
        const uint32_t b2h = smem_u32(Bm), b2l = b2h + (uint32_t)(sizeof(float) * N1 * Kq);
        for (int ks = 0; ks < Kq / 8; ++ks) {
          const uint32_t ao = ks * 2 * a2_lbo, bo = ks * 2 * b_lbo;
          mma_tf32(d2, smem_desc(a2h + ao, a2_lbo, 128), smem_desc(b2h + bo, b_lbo, 128), idesc, (r > 0 || ks > 0));
          mma_tf32(d2, smem_desc(a2h + ao, a2_lbo, 128), smem_desc(b2l + bo, b_lbo, 128), idesc, 1);
          mma_tf32(d2, smem_desc(a2l + ao, a2_lbo, 128), smem_desc(b2h + bo, b_lbo, 128), idesc, 1);
        }
        mma_commit(&bar_mma);
      }
    }
    ok = ok && mbar_wait(&bar_mma, mma_phase);
    mma_phase ^= 1;
    tc_fence_after();
    // epilogue: node i = TMEM lane, this half's elements
    {
      const int i = quarter * 32 + lane;
      float rv[NV][HALF];
#pragma unroll
      for (int v = 0; v < NV; ++v)
        tmem_ld4(d2 + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(v * Te + half * HALF), rv[v]);
      tmem_wait_ld();
      if (i < Np && ok) {
#pragma unroll
        for (int j = 0; j < HALF; ++j) {
          const int e = half * HALF + j;
          if (e < ne) {
            double* Ri = B.Rinv + (((size_t)e0 + e) * Np + i) * NV;
#pragma unroll
            for (int v = 0; v < NV; ++v) Ri[v] = (double)rv[v][j];
          }
        }
      }
    }
    tc_fence_before();
    if (__syncthreads_or(!ok)) ok = false;
    tc_fence_after();
  }
  if (!ok) {
    if (tid == 0) {
      atomicOr(err, DGB_DEVICE_TIMEOUT);
    }
    // let operations in flight drain (bounded) before the tensor memory is released
    mbar_wait(&bar_mma, mma_phase);
    mbar_wait(&bar_tma, tma_phase);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(ncols));
  }
}

int tc_pack(const BlockDev& B, const TcShape& s, float* image, cudaStream_t st) {
  const int threads = 256, blocks = (s.image_floats + threads - 1) / threads;
  k_tc_pack<<<blocks, threads, 0, st>>>(B.B, B.dB, s, image);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

cudaError_t tc_volume(const DevPlan& P, const StatePtrs& S, int b, const TcShape& s, const float* image, int* err,
                      int sm_count, cudaStream_t st) {
  const int E = P.blk[b].E;
  if (E == 0) return cudaSuccess;
  const int ntiles = (E + kTcTe - 1) / kTcTe;
  const int grid = ntiles < sm_count ? ntiles : sm_count;
  // at least 60 KB of shared memory per CTA keeps at most three CTAs on an SM, so their tensor
  // memory (at most 128 columns each) always fits in the SM's 512 columns: no CTA waits in
  // tcgen05.alloc.  The attribute is the dynamic size of this launch (static shared memory comes
  // on top of it within the 227 KB limit).
  const size_t smem = s.smem > 60 * 1024 ? s.smem : 60 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k_tc_volume, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_tc_volume<<<grid, kTcThreads, smem, st>>>(P, S, b, s, image, err);
  return cudaGetLastError();
}

}  // namespace dgb
