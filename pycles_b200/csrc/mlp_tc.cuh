// Refresh of the learned seed on the 5th-generation tensor cores (tcgen05).
//
// The network (mlp.cuh) evaluated for tiles of 128 cells: layer 1 (the
// inputs split into BF16 high and low parts and two constant-one columns
// that carry the split bias, K = 16) and layer 2 (K = 64, four MMAs) are
// tcgen05.mma kind::f16 products, BF16 operands in shared memory, FP32
// accumulators in tensor memory (TMEM).  Row m of a tile is TMEM lane m, so thread m
// (warp m/32 reads lanes 32(m/32) .. +31) reads its own sample's 64
// pre-activations with tcgen05.ld, applies the bias and the SiLU (the packed
// BF16 form of mlp.cuh, as training uses) and writes the activations back
// as the next product's A operand; layer 3 (64 -> 1) is a dot product in
// registers.  z1 and z2 share the 64 allocated columns: layer 2's product is
// issued once every thread has read z1 out.  One elected thread issues the
// MMAs and commits them to an mbarrier; every wait is bounded.
//
// Operand layout: the canonical K-major layout without swizzling, 8-row x
// 16-byte core matrices; element (row, k) of a tile with K columns lives at
// byte (row/8)*SBO + (k/8)*128 + (row%8)*16 + (k%8)*2, SBO = K/8 * 128 (the
// core matrices of one 8-row group are adjacent along K, 128 bytes apart).
//
// Resident blocks per SM are held to 6 by the shared-memory request (6 x 64
// TMEM columns of the 512), so a block's allocation never waits; the
// per-tile chain (two products, two epilogues) is latency-bound, so the
// blocks of an SM overlap each other's.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "mlp.cuh"
#include "tma.cuh"

namespace mlptc {

constexpr int kM = 128;             // samples per tile, one per thread
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 64;
constexpr int kScanBatch = 4;       // cells per thread per scan round
constexpr int kQueue = kM * (kScanBatch + 1);
constexpr size_t kSmemRequest = 36 * 1024;  // <= 6 resident blocks per SM

struct alignas(128) SmemTc {
  alignas(128) uint8_t a1[kM * 16 * 2];    // layer-1 A: 128 x 16 BF16
  alignas(128) uint8_t b1[64 * 16 * 2];    // layer-1 B: 64 x 16 BF16 (row n: unit n's weights over k)
  alignas(128) uint8_t a2[kM * 64 * 2];    // layer-2 A: 128 x 64 BF16
  alignas(128) uint8_t b2[64 * 64 * 2];    // layer-2 B: 64 x 64 BF16 (row n: w2[n][:])
  float b2f[64];
  float w3f[64];                           // BF16 weights as FP32
  float b3;
  int queue[kQueue];
  int count;
  uint32_t tmem;
  alignas(8) uint64_t bar;
};

__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int sbo) {
  return (uint32_t)((row >> 3) * sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start, leading (K) and stride (8-row)
// byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major,
// N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, int accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   pbtma::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct RefreshTcArgs {
  const __nv_bfloat16* w1;
  const float* b1;
  const __nv_bfloat16* w2;
  const float* b2;
  const __nv_bfloat16* w3;
  const float* b3;
  float lo[3], hi[3];
  const double* p0;  // per level (n2)
  const double* s;
  const double* qt;
  const double* ql;  // the previous update's condensate: the flag
  float* y;
  long long npg;
  int n2;
  unsigned int* err;
};

__device__ __forceinline__ void stage_weights_tc(SmemTc& sm, const RefreshTcArgs& a) {
  const int t = threadIdx.x;
  // B1 row n, k: w1[n][k % 3] for k < 6 (the inputs' high and low parts),
  // the bias split into BF16 high (k = 6) and low (k = 7) parts, then zeros
  for (int e = t; e < 64 * 16; e += kThreads) {
    const int n = e >> 4, k = e & 15;
    __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
    if (k < 6) {
      v = a.w1[n * 3 + k % 3];
    } else if (k < 8) {
      const __nv_bfloat16 hi = __float2bfloat16_rn(a.b1[n]);
      v = (k == 6) ? hi : __float2bfloat16_rn(a.b1[n] - __bfloat162float(hi));
    }
    *reinterpret_cast<__nv_bfloat16*>(sm.b1 + kmajor_off(n, k, 256)) = v;
  }
  for (int e = t; e < 64 * 64; e += kThreads) {
    const int n = e >> 6, k = e & 63;
    *reinterpret_cast<__nv_bfloat16*>(sm.b2 + kmajor_off(n, k, 1024)) = a.w2[n * 64 + k];
  }
  if (t < 64) {
    sm.b2f[t] = a.b2[t];
    sm.w3f[t] = __bfloat162float(a.w3[t]);
  }
  if (t == 0) sm.b3 = a.b3[0];
}

// One tile of n <= 128 queued cells.
__device__ __forceinline__ void tile_tc(SmemTc& sm, const RefreshTcArgs& a, const int* q, int n, uint32_t& phase) {
  const int t = threadIdx.x;
  const int w = t >> 5;
  const int cell = t < n ? q[t] : -1;
  // layer-1 A row t: [x_hi (3), x_lo (3), 1, 1, 0 x 8]
  {
    float x[3] = {0.0f, 0.0f, 0.0f};
    if (cell >= 0) {
      x[0] = mlpk::norm_in(a.p0[cell % a.n2], a.lo[0], a.hi[0]);
      x[1] = mlpk::norm_in(a.s[cell], a.lo[1], a.hi[1]);
      x[2] = mlpk::norm_in(a.qt[cell], a.lo[2], a.hi[2]);
    }
    float v[8];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      v[i] = __bfloat162float(__float2bfloat16_rn(x[i]));
      v[3 + i] = x[i] - v[i];
    }
    v[6] = v[7] = (cell >= 0) ? 1.0f : 0.0f;
    uint4 lo4, hi4;
    lo4.x = mlpk::pack_bf16(v[0], v[1]);
    lo4.y = mlpk::pack_bf16(v[2], v[3]);
    lo4.z = mlpk::pack_bf16(v[4], v[5]);
    lo4.w = mlpk::pack_bf16(v[6], v[7]);
    hi4 = make_uint4(0u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(sm.a1 + kmajor_off(t, 0, 256)) = lo4;
    *reinterpret_cast<uint4*>(sm.a1 + kmajor_off(t, 8, 256)) = hi4;
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  if (t == 0) {
    fence_after();
    mma(sm.tmem, smem_desc(pbtma::smem_u32(sm.a1), 128, 256), smem_desc(pbtma::smem_u32(sm.b1), 128, 256), 0);
    commit(&sm.bar);
  }
  pbtma::mbar_wait(&sm.bar, phase, a.err);
  phase ^= 1u;
  fence_after();
  const uint32_t lane_addr = sm.tmem + ((uint32_t)(w * 32) << 16);
  // layer-1 activations -> layer-2 A row t
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float z[16];
    tmem_ld16(lane_addr + 16 * q, z);
#pragma unroll
    for (int c8 = 0; c8 < 2; ++c8) {
      uint4 h;
      h.x = mlpk::silu_bf16x2(z[8 * c8 + 0], z[8 * c8 + 1]);
      h.y = mlpk::silu_bf16x2(z[8 * c8 + 2], z[8 * c8 + 3]);
      h.z = mlpk::silu_bf16x2(z[8 * c8 + 4], z[8 * c8 + 5]);
      h.w = mlpk::silu_bf16x2(z[8 * c8 + 6], z[8 * c8 + 7]);
      *reinterpret_cast<uint4*>(sm.a2 + kmajor_off(t, 16 * q + 8 * c8, 1024)) = h;
    }
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  if (t == 0) {
    fence_after();
    const uint32_t a2 = pbtma::smem_u32(sm.a2), b2 = pbtma::smem_u32(sm.b2);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      mma(sm.tmem, smem_desc(a2 + 256 * kk, 128, 1024), smem_desc(b2 + 256 * kk, 128, 1024), kk > 0);
    commit(&sm.bar);
  }
  pbtma::mbar_wait(&sm.bar, phase, a.err);
  phase ^= 1u;
  fence_after();
  float y = sm.b3;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float z[16];
    tmem_ld16(lane_addr + 16 * q, z);
#pragma unroll
    for (int c = 0; c < 16; c += 2) {
      const int col = 16 * q + c;
      const uint32_t h = mlpk::silu_bf16x2(z[c] + sm.b2f[col], z[c + 1] + sm.b2f[col + 1]);
      const __nv_bfloat162 hb = *reinterpret_cast<const __nv_bfloat162*>(&h);
      y = fmaf(__low2float(hb), sm.w3f[col], y);
      y = fmaf(__high2float(hb), sm.w3f[col + 1], y);
    }
  }
  if (cell >= 0) a.y[cell] = y;
  fence_before();
  __syncthreads();  // TMEM and the A tiles are free for the next tile
}

__global__ void __launch_bounds__(kThreads, 6) mlp_seed_refresh_tc(RefreshTcArgs a) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  SmemTc& sm = *reinterpret_cast<SmemTc*>(smraw);
  const int t = threadIdx.x;
  if (t < 32) {  // warp 0 owns the tensor-memory allocation
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     pbtma::smem_u32(&sm.tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    pbtma::mbar_init(&sm.bar, 1);
    pbtma::mbar_fence_init();
    sm.count = 0;
  }
  stage_weights_tc(sm, a);
  fence_before();
  __syncthreads();
  fence_after();
  uint32_t phase = 0;
  const long long scan = (long long)kThreads * kScanBatch;
  for (long long base = (long long)blockIdx.x * scan; base < a.npg; base += (long long)gridDim.x * scan) {
#pragma unroll
    for (int b = 0; b < kScanBatch; ++b) {
      const long long idx = base + b * kThreads + t;
      if (idx < a.npg) {
        if (__ldg(a.ql + idx) > 0.0) {
          const int pos = atomicAdd(&sm.count, 1);
          sm.queue[pos] = (int)idx;
        } else {
          a.y[idx] = __int_as_float(0x7fc00000);  // not evaluated: NaN, the secant takes its own start
        }
      }
    }
    __syncthreads();
    const int n = sm.count;
    int done = 0;
    while (n - done >= kM) {
      tile_tc(sm, a, sm.queue + done, kM, phase);
      done += kM;
    }
    const int rest = n - done;
    const int moved = t < rest ? sm.queue[done + t] : 0;
    __syncthreads();
    if (t < rest) sm.queue[t] = moved;
    if (t == 0) sm.count = rest;
    __syncthreads();
  }
  const int n = sm.count;
  if (n > 0) tile_tc(sm, a, sm.queue, n, phase);
  fence_before();
  __syncthreads();
  if (t < 32) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace mlptc
