// Learned saturation-adjustment seed: a 3 -> 64 -> 64 -> 1 SiLU MLP.
//
// Warp-level tiles for point lists (pb_mlp_forward) and training
// (pb_mlp_grad); the refresh of a whole field's seeds runs on the tcgen05
// tensor cores with the same arithmetic (mlp_tc.cuh).
//
// One warp evaluates a tile of 16 samples.  The three layers run on the
// tensor cores with mma.sync m16n8k16 (BF16 operands, FP32 accumulation;
// layer 1's inputs split into BF16 high and low parts, layer 3 as an N = 8
// product whose column 0 is the output).  A layer's accumulator fragments
// are, after the activation, exactly the next layer's A fragments, so no
// shuffles or shared memory are needed between layers:
//   A fragment (16x16, row-major), lane = 4*g + t (g = lane/4, t = lane%4):
//     regs 0/1/2/3 = rows {g, g+8, g, g+8} x cols {2t, 2t, 2t+8, 2t+8} (+0,+1)
//   B fragment (16x8, column-major): regs 0/1 = k {2t, 2t+8} (+0,+1), n = g
//   C fragment (16x8): c0,c1 = row g, cols 2t,2t+1; c2,c3 = row g+8
// so the C fragments of n-tiles 2kt and 2kt+1 are, reinterpreted, the A
// fragment of k-tile kt (used between the layers, and by the backward
// pass).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace mlpk {

constexpr int H = 64;
// packed parameter layout (FP32 masters and gradients)
constexpr int OFF_W1 = 0;                // [64][3]
constexpr int OFF_B1 = OFF_W1 + H * 3;   // [64]
constexpr int OFF_W2 = OFF_B1 + H;       // [64][64] (row = output unit)
constexpr int OFF_B2 = OFF_W2 + H * H;   // [64]
constexpr int OFF_W3 = OFF_B2 + H;       // [64]
constexpr int OFF_B3 = OFF_W3 + H;       // [1]
constexpr int NPARAM = OFF_B3 + 1;

// SiLU(z) = z sigmoid(z), sigmoid(z) = (1 + tanh(z/2)) / 2, with the
// hardware tanh approximation (tanh.approx.f32, one special-function
// instruction; relative error ~2^-11, below the BF16 rounding of the
// activations).  Training and inference use the same function.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoid(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ __forceinline__ float silu(float z) {  // z/2 + (z/2) tanh(z/2)
  const float hz = 0.5f * z;
  return fmaf(hz, tanh_approx(hz), hz);
}
__device__ __forceinline__ float silu_grad(float z) {
  const float s = sigmoid(z);
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// Two SiLU activations computed and returned as a BF16 pair (layer 1's
// activations are BF16 operands of layer 2 anyway): z/2 rounded to BF16,
// then z/2 + (z/2) tanh(z/2) with the packed BF16 tanh and FMA.
__device__ __forceinline__ uint32_t silu_bf16x2(float z0, float z1) {
  const uint32_t hz = pack_bf16(0.5f * z0, 0.5f * z1);
  uint32_t t, h;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(hz));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(h) : "r"(hz), "r"(t));
  return h;
}

__device__ __forceinline__ void mma_bf16_16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Weights staged in shared memory by the block.  All three layers run on
// the tensor cores.  Layer 1's A operand holds the three inputs split into
// BF16 high and low parts (columns 0-2 and 3-5, ~16 significant bits per
// input) and two constant-one columns (6, 7), so w1f -- the B fragment
// [ntile][lane] of the 16x64 matrix [W1^T; W1^T; b1_hi; b1_lo; 0] (b1 split
// into BF16 high and low parts, ~16 significant bits) -- adds the bias in
// the product.  w2f holds layer 2 in B fragment order, [ntile][ktile][lane]
// -> {b0, b1}, one conflict-free 8-byte load per lane; its FP32 bias
// initialises the accumulator.  w3f is layer 3 as the B fragment of a 64x8
// matrix whose column 0 is w3 ([ktile][lane]; lanes of groups g > 0 hold
// zeros); w3 (FP32 copy of the BF16 weights) serves the backward pass.
struct Smem {
  uint32_t w1f[8 * 32];
  __nv_bfloat16 w2[H * H];  // [n][k]
  uint2 w2f[8 * 4 * 32];
  uint2 w3f[4 * 32];
  float b2[H];
  float w3[H];
  float b3;
};

// Loads BF16 weights + FP32 biases into shared memory (whole block; tid and
// nthreads are the thread's linear index and the block size).
__device__ __forceinline__ void stage_weights(Smem& sm, const __nv_bfloat16* w1, const float* b1,
                                              const __nv_bfloat16* w2, const float* b2, const __nv_bfloat16* w3,
                                              const float* b3, int tid, int nthreads) {
  for (int i = tid; i < H * H; i += nthreads) sm.w2[i] = w2[i];
  for (int i = tid; i < H; i += nthreads) {
    sm.b2[i] = b2[i];
    sm.w3[i] = __bfloat162float(w3[i]);
  }
  for (int i = tid; i < 8 * 32; i += nthreads) {
    const int lane = i & 31, nt = i >> 5;
    const int n = nt * 8 + (lane >> 2), t = lane & 3;
    // k rows 2t, 2t+1 of [W1^T; W1^T; b1_hi; b1_lo]
    const __nv_bfloat16 bhi = __float2bfloat16_rn(b1[n]);
    const __nv_bfloat16 blo = __float2bfloat16_rn(b1[n] - __bfloat162float(bhi));
    uint16_t e[2];
    for (int u = 0; u < 2; ++u) {
      const int k = 2 * t + u;
      const __nv_bfloat16 v = (k < 6) ? w1[n * 3 + k % 3] : (k == 6 ? bhi : blo);
      e[u] = *reinterpret_cast<const uint16_t*>(&v);
    }
    sm.w1f[i] = (uint32_t)e[0] | ((uint32_t)e[1] << 16);
  }
  for (int i = tid; i < 8 * 4 * 32; i += nthreads) {
    const int lane = i & 31, kt = (i >> 5) & 3, nt = i >> 7;
    const int n = nt * 8 + (lane >> 2), k = kt * 16 + 2 * (lane & 3);
    uint2 b;
    b.x = *reinterpret_cast<const uint32_t*>(w2 + n * H + k);
    b.y = *reinterpret_cast<const uint32_t*>(w2 + n * H + k + 8);
    sm.w2f[i] = b;
  }
  for (int i = tid; i < 4 * 32; i += nthreads) {
    const int lane = i & 31, kt = i >> 5;
    const int k = kt * 16 + 2 * (lane & 3);
    uint2 b = make_uint2(0u, 0u);
    if ((lane >> 2) == 0) {  // column 0
      b.x = *reinterpret_cast<const uint32_t*>(w3 + k);
      b.y = *reinterpret_cast<const uint32_t*>(w3 + k + 8);
    }
    sm.w3f[i] = b;
  }
  if (tid == 0) sm.b3 = b3[0];
}

// Forward pass of one 16-row tile.  xr0/xr1: the 3 normalised inputs of the
// lane's rows g and g+8.  Returns y for rows g (y0) and g+8 (y1) on all four
// lanes of group g.  Optionally keeps the z1 / h1 fragments and z2 / h2 for
// the backward pass (h2 as the BF16 values layer 3 multiplies).
struct Tile {
  float z1[4][4][2];   // [ktile][reg][pair]  (rows/cols as the A fragment)
  uint32_t a1[4][4];   // BF16 h1 A fragments
  float z2[8][4];      // [ntile][c-reg]
  float h2[8][4];
};

// COMPACT keeps the layer-2/3 loop over k-tiles rolled (a quarter of the
// code), for callers that share the instruction cache with much other code
// (the fused thermodynamics kernel); the training and stand-alone forward
// kernels unroll it.  keep must be nullptr when COMPACT.
template <bool COMPACT = false>
__device__ __forceinline__ void forward_tile(const Smem& sm, const float xr0[3], const float xr1[3], float& y0,
                                             float& y1, Tile* keep) {
  const int lane = threadIdx.x & 31;
  const int t = lane & 3;
  // layer 1: A = [x_hi, x_lo, 1, 1, 0...] (16 x 16), lane t holds columns 2t, 2t+1
  uint32_t ax[4] = {0u, 0u, 0u, 0u};
  {
    float v0[6], v1[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      v0[i] = __bfloat162float(__float2bfloat16_rn(xr0[i]));
      v0[3 + i] = xr0[i] - v0[i];
      v1[i] = __bfloat162float(__float2bfloat16_rn(xr1[i]));
      v1[3 + i] = xr1[i] - v1[i];
    }
    if (t < 3) {
      ax[0] = pack_bf16(v0[2 * t], v0[2 * t + 1]);  // row g
      ax[1] = pack_bf16(v1[2 * t], v1[2 * t + 1]);  // row g + 8
    } else {
      ax[0] = ax[1] = pack_bf16(1.0f, 1.0f);        // the bias columns
    }
  }
  uint32_t a1[4][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const uint32_t b[2] = {sm.w1f[nt * 32 + lane], 0u};
    mma_bf16_16816(c, ax, b);
    // C fragments of n-tiles 2kt, 2kt+1 are the A fragment of layer 2's k-tile kt
    const int kt = nt >> 1, half = nt & 1;
    if (keep) {
      keep->z1[kt][half * 2 + 0][0] = c[0];
      keep->z1[kt][half * 2 + 0][1] = c[1];
      keep->z1[kt][half * 2 + 1][0] = c[2];
      keep->z1[kt][half * 2 + 1][1] = c[3];
    }
    a1[kt][half * 2 + 0] = silu_bf16x2(c[0], c[1]);
    a1[kt][half * 2 + 1] = silu_bf16x2(c[2], c[3]);
  }
  if (keep) {
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
      for (int r = 0; r < 4; ++r) keep->a1[kt][r] = a1[kt][r];
  }
  // layer 2 (bias in the accumulator); each pair of n-tiles, once activated,
  // is a complete A fragment of layer 3 and goes straight into it (fewer
  // live registers than holding all of h2)
  float c3[4] = {sm.b3, 0.0f, sm.b3, 0.0f};
#pragma unroll(COMPACT ? 1 : 4)
  for (int kt = 0; kt < 4; ++kt) {
    uint32_t a2[4];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int nt = 2 * kt + half;
      const int c0 = nt * 8 + 2 * t;
      float c[4] = {sm.b2[c0], sm.b2[c0 + 1], sm.b2[c0], sm.b2[c0 + 1]};
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) {
        const uint2 bf = sm.w2f[(nt * 4 + k2) * 32 + lane];
        const uint32_t b[2] = {bf.x, bf.y};
        mma_bf16_16816(c, a1[k2], b);
      }
      a2[half * 2 + 0] = silu_bf16x2(c[0], c[1]);
      a2[half * 2 + 1] = silu_bf16x2(c[2], c[3]);
      if (!COMPACT && keep) {
#pragma unroll
        for (int q = 0; q < 4; ++q) keep->z2[nt][q] = c[q];
        const __nv_bfloat162 h01 = *reinterpret_cast<const __nv_bfloat162*>(&a2[half * 2 + 0]);
        const __nv_bfloat162 h23 = *reinterpret_cast<const __nv_bfloat162*>(&a2[half * 2 + 1]);
        keep->h2[nt][0] = __low2float(h01);
        keep->h2[nt][1] = __high2float(h01);
        keep->h2[nt][2] = __low2float(h23);
        keep->h2[nt][3] = __high2float(h23);
      }
    }
    // layer 3: column 0 of h2 . [w3, 0 ...]
    const uint2 bf = sm.w3f[kt * 32 + lane];
    const uint32_t b[2] = {bf.x, bf.y};
    mma_bf16_16816(c3, a2, b);
  }
  // column 0 sits on the group's lane t == 0: every lane of the group gets it
  y0 = __shfl_sync(0xffffffffu, c3[0], lane & ~3);  // row g
  y1 = __shfl_sync(0xffffffffu, c3[2], lane & ~3);  // row g + 8
}

// 2 (v - lo) / (hi - lo) - 1: the offset in FP64, the scaling in FP32 with
// a fast reciprocal (no FP64 division, whose slow path adds code to every
// kernel that inlines this)
__device__ __forceinline__ float norm_in(double v, float lo, float hi) {
  return fmaf((float)(v - (double)lo), __fdividef(2.0f, hi - lo), -1.0f);
}

}  // namespace mlpk
