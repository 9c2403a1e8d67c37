// Learned saturation-adjustment seed: inference and training kernels.
// (No counterpart in the reference; see mlp.cuh for the network and the
// fragment layouts.)
#include "pb_common.cuh"
#include "mlp.cuh"
#include "mlp_tc.cuh"
#include "thermo_funcs.cuh"

static_assert(mlpk::NPARAM == PB_MLP_NPARAM, "packed parameter count must match the public header");

namespace mlpk {

struct FwdArgs {
  const __nv_bfloat16* w1;
  const float* b1;
  const __nv_bfloat16* w2;
  const float* b2;
  const __nv_bfloat16* w3;
  const float* b3;
  float lo[3], hi[3];
  float out_mean, out_scale;
  const double* p0;
  const double* s;
  const double* qt;
  double* T;
  long long n;
};

__global__ void __launch_bounds__(128) mlp_forward_kernel(FwdArgs a) {
  __shared__ Smem sm;
  stage_weights(sm, a.w1, a.b1, a.w2, a.b2, a.w3, a.b3, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long ntiles = (a.n + 15) / 16;
  for (long long tile = warp; tile < ntiles; tile += nwarps) {
    const long long r0 = tile * 16 + g, r1 = r0 + 8;
    float x0[3] = {0.f, 0.f, 0.f}, x1[3] = {0.f, 0.f, 0.f};
    if (r0 < a.n) {
      x0[0] = norm_in(a.p0[r0], a.lo[0], a.hi[0]);
      x0[1] = norm_in(a.s[r0], a.lo[1], a.hi[1]);
      x0[2] = norm_in(a.qt[r0], a.lo[2], a.hi[2]);
    }
    if (r1 < a.n) {
      x1[0] = norm_in(a.p0[r1], a.lo[0], a.hi[0]);
      x1[1] = norm_in(a.s[r1], a.lo[1], a.hi[1]);
      x1[2] = norm_in(a.qt[r1], a.lo[2], a.hi[2]);
    }
    float y0, y1;
    forward_tile(sm, x0, x1, y0, y1, nullptr);
    if (t == 0) {
      using thermo_f::FastMath;
      if (r0 < a.n)
        a.T[r0] = thermo_f::first_point<FastMath>(a.p0[r0], a.s[r0], a.qt[r0]) + (double)a.out_mean +
                  (double)a.out_scale * (double)y0;
      if (r1 < a.n)
        a.T[r1] = thermo_f::first_point<FastMath>(a.p0[r1], a.s[r1], a.qt[r1]) + (double)a.out_mean +
                  (double)a.out_scale * (double)y1;
    }
  }
}

// The refresh of the learned seed's per-cell network output y for the cells
// that were saturated at the previous thermodynamics update (ql > 0 there)
// runs on the tcgen05 tensor cores (mlp_tc.cuh), as its own kernel ahead of
// the thermodynamics kernel, which then reads y: the network's code and
// shared memory stay out of the FP64 secant kernel (whose instruction cache
// it overflowed).  Cells not flagged get NaN: a cell that saturates between
// refreshes starts its secant from the reference's second point, not from a
// stale output.

// Gradient of sum_r 0.5 (y_r - target_r)^2 over n normalised samples,
// accumulated into grad[NPARAM] (packed, FP32), loss sum into *loss.
//
// Deterministic: no floating-point atomics.  Each warp accumulates its
// tiles (a fixed set: tile = warp + round * warps) into its own
// shared-memory copy of the gradient, in program order; each block writes
// the sum of its warps' copies (warp 0 + warp 1) as one row of a partials
// array, and grad_reduce_kernel adds the rows in block order.  The block
// count depends only on n (kGradMaxBlocks caps it), so the same inputs give
// the same gradient bit for bit on every run and every device.
struct GradArgs {
  const __nv_bfloat16* w1;
  const float* b1;
  const __nv_bfloat16* w2;
  const float* b2;
  const __nv_bfloat16* w3;
  const float* b3;
  const float* x;       // n x 3
  const float* target;  // n
  float* part;  // [gridDim.x][kPartStride]: a block's gradient, then its loss
  long long n;
};

constexpr int kGradWarps = 2;
constexpr int kGradMaxBlocks = 1184;
constexpr int kPartStride = NPARAM + 1;
// dynamic shared memory of mlp_grad_kernel: one FP32 gradient accumulator
// per warp
constexpr size_t kGradSmem = (size_t)kGradWarps * NPARAM * sizeof(float);

inline int grad_blocks(long long n) {
  const long long tiles = (n + 15) / 16;
  long long b = (tiles + kGradWarps - 1) / kGradWarps;
  if (b > kGradMaxBlocks) b = kGradMaxBlocks;
  return (int)(b < 1 ? 1 : b);
}

__global__ void __launch_bounds__(64) mlp_grad_kernel(GradArgs a) {
  __shared__ Smem sm;
  extern __shared__ float acc_all[];  // [kGradWarps][NPARAM]
  __shared__ float dz2_s[kGradWarps][16][H];
  __shared__ float h1_s[kGradWarps][16][H];
  __shared__ float loss_s[kGradWarps];
  stage_weights(sm, a.w1, a.b1, a.w2, a.b2, a.w3, a.b3, threadIdx.x, blockDim.x);
  for (int i = threadIdx.x; i < kGradWarps * NPARAM; i += blockDim.x) acc_all[i] = 0.0f;
  __syncthreads();
  const int wid = threadIdx.x >> 5;
  // this warp's accumulator: every entry is written by one lane at a time
  float* acc = acc_all + wid * NPARAM;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long ntiles = (a.n + 15) / 16;
  // uniform trip count across the block's warps (shared-memory accumulators)
  const long long per_block_tiles = (ntiles + gridDim.x - 1) / gridDim.x;
  const long long rounds = (per_block_tiles + kGradWarps - 1) / kGradWarps;
  float lsum = 0.0f;
  for (long long rnd = 0; rnd < rounds; ++rnd) {
    const long long tile = warp + rnd * nwarps;
    const bool have = tile < ntiles;
    const long long r0 = tile * 16 + g, r1 = r0 + 8;
    const bool v0 = have && r0 < a.n, v1 = have && r1 < a.n;
    float x0[3] = {0.f, 0.f, 0.f}, x1[3] = {0.f, 0.f, 0.f};
    if (v0) for (int i = 0; i < 3; ++i) x0[i] = a.x[r0 * 3 + i];
    if (v1) for (int i = 0; i < 3; ++i) x1[i] = a.x[r1 * 3 + i];
    Tile T;
    float y0, y1;
    forward_tile(sm, x0, x1, y0, y1, &T);
    const float dy0 = v0 ? (y0 - a.target[r0]) : 0.0f;
    const float dy1 = v1 ? (y1 - a.target[r1]) : 0.0f;
    if (t == 0) lsum += 0.5f * (dy0 * dy0 + dy1 * dy1);
    // layer 3 and dz2 (C-fragment layout)
    float dz2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int col = nt * 8 + 2 * t + (q & 1);
        const float dy = (q < 2) ? dy0 : dy1;
        dz2[nt][q] = dy * sm.w3[col] * silu_grad(T.z2[nt][q]);
      }
      // w3, b2 partials: sum the lane's two rows, then over the 8 groups
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        float gw3 = dy0 * T.h2[nt][p] + dy1 * T.h2[nt][p + 2];
        float gb2 = dz2[nt][p] + dz2[nt][p + 2];
        for (int off = 4; off < 32; off <<= 1) {
          gw3 += __shfl_xor_sync(0xffffffffu, gw3, off);
          gb2 += __shfl_xor_sync(0xffffffffu, gb2, off);
        }
        if (g == 0) {
          const int col = nt * 8 + 2 * t + p;
          acc[OFF_W3 + col] += gw3;
          acc[OFF_B2 + col] += gb2;
        }
      }
    }
    float gb3 = dy0 + dy1;
    gb3 += __shfl_xor_sync(0xffffffffu, gb3, 4);
    gb3 += __shfl_xor_sync(0xffffffffu, gb3, 8);
    gb3 += __shfl_xor_sync(0xffffffffu, gb3, 16);
    if (lane == 0) acc[OFF_B3] += gb3;
    // stage dz2 and the BF16 h1 of this tile for the layer-2 weight gradient
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) dz2_s[wid][g + ((q & 2) ? 8 : 0)][nt * 8 + 2 * t + (q & 1)] = dz2[nt][q];
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&T.a1[kt][r]);
        const int row = g + ((r & 1) ? 8 : 0);
        const int col = kt * 16 + 2 * t + ((r & 2) ? 8 : 0);
        h1_s[wid][row][col] = __low2float(h);
        h1_s[wid][row][col + 1] = __high2float(h);
      }
    // dh1 = dz2 . W2 on the tensor cores: dz2's C fragments are the A fragments
    float dh1[8][4];
#pragma unroll
    for (int nt2 = 0; nt2 < 8; ++nt2) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        uint32_t af[4];
        af[0] = pack_bf16(dz2[2 * kt][0], dz2[2 * kt][1]);
        af[1] = pack_bf16(dz2[2 * kt][2], dz2[2 * kt][3]);
        af[2] = pack_bf16(dz2[2 * kt + 1][0], dz2[2 * kt + 1][1]);
        af[3] = pack_bf16(dz2[2 * kt + 1][2], dz2[2 * kt + 1][3]);
        const int n0 = kt * 16 + 2 * t;
        const int kc = nt2 * 8 + g;
        uint32_t b[2];
        __nv_bfloat162 bb;
        bb.x = sm.w2[n0 * H + kc];
        bb.y = sm.w2[(n0 + 1) * H + kc];
        b[0] = *reinterpret_cast<const uint32_t*>(&bb);
        bb.x = sm.w2[(n0 + 8) * H + kc];
        bb.y = sm.w2[(n0 + 9) * H + kc];
        b[1] = *reinterpret_cast<const uint32_t*>(&bb);
        mma_bf16_16816(c, af, b);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) dh1[nt2][q] = c[q];
    }
    // dz1 = dh1 * silu'(z1); W1 and b1 partials
#pragma unroll
    for (int nt2 = 0; nt2 < 8; ++nt2) {
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        const int kt = nt2 >> 1;
        const int rb = (nt2 & 1) * 2;
        const float dz_r0 = dh1[nt2][p] * silu_grad(T.z1[kt][rb + 0][p]);
        const float dz_r1 = dh1[nt2][p + 2] * silu_grad(T.z1[kt][rb + 1][p]);
        float gb1 = dz_r0 + dz_r1;
        float gw[3];
        for (int i = 0; i < 3; ++i) gw[i] = dz_r0 * x0[i] + dz_r1 * x1[i];
        for (int off = 4; off < 32; off <<= 1) {
          gb1 += __shfl_xor_sync(0xffffffffu, gb1, off);
          for (int i = 0; i < 3; ++i) gw[i] += __shfl_xor_sync(0xffffffffu, gw[i], off);
        }
        if (g == 0) {
          const int k = nt2 * 8 + 2 * t + p;
          acc[OFF_B1 + k] += gb1;
          for (int i = 0; i < 3; ++i) acc[OFF_W1 + k * 3 + i] += gw[i];
        }
      }
    }
    __syncwarp();
    // W2 gradient: dW2[n][k] = sum_r dz2[r][n] h1[r][k], 128 entries per lane
    for (int e = lane; e < H * H; e += 32) {
      const int n = e >> 6, k = e & 63;
      float sacc = 0.0f;
#pragma unroll
      for (int r = 0; r < 16; ++r) sacc += dz2_s[wid][r][n] * h1_s[wid][r][k];
      acc[OFF_W2 + e] += sacc;
    }
    __syncwarp();
  }
  for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
  if (lane == 0) loss_s[wid] = lsum;
  __syncthreads();
  static_assert(kGradWarps == 2, "the block's sum below adds two warps' copies");
  float* row = a.part + (long long)blockIdx.x * kPartStride;
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) row[i] = acc_all[i] + acc_all[NPARAM + i];
  if (threadIdx.x == 0) row[NPARAM] = loss_s[0] + loss_s[1];
}

// grad[i] += sum over blocks b (in order) of part[b][i]; *loss likewise from
// the rows' last entry.  One thread per entry; a row is read coalesced.
__global__ void __launch_bounds__(256) grad_reduce_kernel(const float* __restrict__ part, int blocks,
                                                          float* __restrict__ grad, float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kPartStride) return;
  float s = 0.0f;
  for (int b = 0; b < blocks; ++b) s += part[(long long)b * kPartStride + i];
  if (i < NPARAM)
    grad[i] += s;
  else
    *loss += s;
}

// Adam on the FP32 master parameters, then BF16 / FP32 copies for the kernels.
struct AdamArgs {
  float* params;
  float* m;
  float* v;
  const float* grad;
  float lr, beta1, beta2, eps, grad_scale, bc1, bc2;
  __nv_bfloat16* w1;
  float* b1;
  __nv_bfloat16* w2;
  float* b2;
  __nv_bfloat16* w3;
  float* b3;
};

__global__ void mlp_adam_kernel(AdamArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    const float gr = a.grad[i] * a.grad_scale;
    const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * gr;
    const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * gr * gr;
    a.m[i] = m;
    a.v[i] = v;
    const float p = a.params[i] - a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
    a.params[i] = p;
    if (i < OFF_B1) a.w1[i - OFF_W1] = __float2bfloat16_rn(p);
    else if (i < OFF_W2) a.b1[i - OFF_B1] = p;
    else if (i < OFF_B2) a.w2[i - OFF_W2] = __float2bfloat16_rn(p);
    else if (i < OFF_W3) a.b2[i - OFF_B2] = p;
    else if (i < OFF_B3) a.w3[i - OFF_W3] = __float2bfloat16_rn(p);
    else a.b3[0] = p;
  }
}

}  // namespace mlpk

static int mlp_blocks(long long work_tiles, int warps_per_block);

// The refresh on the tcgen05 tensor cores (mlp_tc.cuh): one persistent
// block of 128 threads per resident slot, 6 per SM.
static cudaError_t refresh_tc(const pb_mlp* mlp, const Geo& g, const double* p0, const double* s,
                              const double* qt, const double* ql, cudaStream_t st) {
  mlptc::RefreshTcArgs a;
  a.w1 = static_cast<const __nv_bfloat16*>(mlp->w1);
  a.b1 = mlp->b1;
  a.w2 = static_cast<const __nv_bfloat16*>(mlp->w2);
  a.b2 = mlp->b2;
  a.w3 = static_cast<const __nv_bfloat16*>(mlp->w3);
  a.b3 = mlp->b3;
  for (int i = 0; i < 3; ++i) {
    a.lo[i] = mlp->in_lo[i];
    a.hi[i] = mlp->in_hi[i];
  }
  a.p0 = p0;
  a.s = s;
  a.qt = qt;
  a.ql = ql;
  a.y = mlp->seed_y;
  a.npg = g.npg;
  a.n2 = (int)g.n2;
  a.err = pb_error_word_ptr();
  cudaError_t e = cudaFuncSetAttribute(mlptc::mlp_seed_refresh_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)mlptc::kSmemRequest);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long tiles = (g.npg + mlptc::kThreads * mlptc::kScanBatch - 1) / (mlptc::kThreads * mlptc::kScanBatch);
  const int blocks = (int)(tiles < 6LL * sms ? tiles : 6LL * sms);
  mlptc::mlp_seed_refresh_tc<<<blocks < 1 ? 1 : blocks, mlptc::kThreads, mlptc::kSmemRequest, st>>>(a);
  pb_note_launch();
  return cudaGetLastError();
}

// y[cell] = MLP(p0, s, qt) for every cell with ql > 0 (called by
// pb_thermo_sa before its kernel; mlp validated there).
cudaError_t pb_mlp_seed_refresh(const pb_mlp* mlp, const Geo& g, const double* p0, const double* s,
                                const double* qt, const double* ql, cudaStream_t st) {
  if (g.npg >= (1LL << 31)) return cudaErrorInvalidValue;  // the queues hold 32-bit cell indices
  return refresh_tc(mlp, g, p0, s, qt, ql, st);
}

static int mlp_blocks(long long work_tiles, int warps_per_block) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long b = (work_tiles + warps_per_block - 1) / warps_per_block;
  if (b > (long long)sms * 8) b = (long long)sms * 8;
  return (int)(b < 1 ? 1 : b);
}

extern "C" int pb_mlp_refresh_seed(const pb_mlp* mlp, const pb_dims* dims, const double* p0_half, const double* s,
                                   const double* qt, const double* ql, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!mlp || !mlp->w1 || !mlp->b1 || !mlp->w2 || !mlp->b2 || !mlp->w3 || !mlp->b3 || !mlp->seed_y || !p0_half ||
      !s || !qt || !ql)
    return PB_ERR_ARG;
  const Geo g = make_geo(dims);
  return pb_mlp_seed_refresh(mlp, g, p0_half, s, qt, ql, as_stream(stream)) == cudaSuccess ? PB_OK : PB_ERR_CUDA;
}

extern "C" int pb_mlp_forward(const pb_mlp* mlp, const double* p0, const double* s, const double* qt,
                              double* T_seed, long long n, void* stream) {
  if (!mlp || !mlp->w1 || !mlp->b1 || !mlp->w2 || !mlp->b2 || !mlp->w3 || !mlp->b3) return PB_ERR_ARG;
  if (!p0 || !s || !qt || !T_seed || n < 0) return PB_ERR_ARG;
  if (n == 0) return PB_OK;
  mlpk::FwdArgs a;
  a.w1 = static_cast<const __nv_bfloat16*>(mlp->w1);
  a.b1 = mlp->b1;
  a.w2 = static_cast<const __nv_bfloat16*>(mlp->w2);
  a.b2 = mlp->b2;
  a.w3 = static_cast<const __nv_bfloat16*>(mlp->w3);
  a.b3 = mlp->b3;
  for (int i = 0; i < 3; ++i) {
    a.lo[i] = mlp->in_lo[i];
    a.hi[i] = mlp->in_hi[i];
  }
  a.out_mean = mlp->out_mean;
  a.out_scale = mlp->out_scale;
  a.p0 = p0;
  a.s = s;
  a.qt = qt;
  a.T = T_seed;
  a.n = n;
  mlpk::mlp_forward_kernel<<<mlp_blocks((n + 15) / 16, 4), 128, 0, as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" long long pb_mlp_grad_workspace_bytes(long long n) {
  if (n < 0) return -1;
  return (long long)mlpk::grad_blocks(n) * mlpk::kPartStride * (long long)sizeof(float);
}

extern "C" int pb_mlp_grad(const pb_mlp* mlp, const float* x, const float* target, long long n, float* grad,
                           float* loss, void* workspace, long long workspace_bytes, void* stream) {
  if (!mlp || !mlp->w1 || !mlp->b1 || !mlp->w2 || !mlp->b2 || !mlp->w3 || !mlp->b3) return PB_ERR_ARG;
  if (!x || !target || !grad || !loss || n < 0) return PB_ERR_ARG;
  if (n == 0) return PB_OK;
  if (!workspace || workspace_bytes < pb_mlp_grad_workspace_bytes(n) ||
      (reinterpret_cast<uintptr_t>(workspace) & 15))
    return PB_ERR_WORKSPACE;
  mlpk::GradArgs a;
  a.w1 = static_cast<const __nv_bfloat16*>(mlp->w1);
  a.b1 = mlp->b1;
  a.w2 = static_cast<const __nv_bfloat16*>(mlp->w2);
  a.b2 = mlp->b2;
  a.w3 = static_cast<const __nv_bfloat16*>(mlp->w3);
  a.b3 = mlp->b3;
  a.x = x;
  a.target = target;
  a.part = static_cast<float*>(workspace);
  a.n = n;
  // the shared-memory opt-in is set on each device's copy of the kernel
  static bool attr_set[64] = {};
  int dev = 0;
  PB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !attr_set[dev]) {
    PB_CUDA_TRY(cudaFuncSetAttribute(mlpk::mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)mlpk::kGradSmem));
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  const int blocks = mlpk::grad_blocks(n);
  cudaStream_t st = as_stream(stream);
  mlpk::mlp_grad_kernel<<<blocks, 32 * mlpk::kGradWarps, mlpk::kGradSmem, st>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  mlpk::grad_reduce_kernel<<<ceil_div(mlpk::kPartStride, 256), 256, 0, st>>>(a.part, blocks, grad, loss);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_mlp_adam(float* params, float* m, float* v, const float* grad, int step, float lr, float beta1,
                           float beta2, float eps, float grad_scale, void* w1, float* b1, void* w2, float* b2,
                           void* w3, float* b3, void* stream) {
  if (!params || !m || !v || !grad || !w1 || !b1 || !w2 || !b2 || !w3 || !b3 || step < 1) return PB_ERR_ARG;
  mlpk::AdamArgs a;
  a.params = params;
  a.m = m;
  a.v = v;
  a.grad = grad;
  a.lr = lr;
  a.beta1 = beta1;
  a.beta2 = beta2;
  a.eps = eps;
  a.grad_scale = grad_scale;
  a.bc1 = 1.0f - powf(beta1, (float)step);
  a.bc2 = 1.0f - powf(beta2, (float)step);
  a.w1 = static_cast<__nv_bfloat16*>(w1);
  a.b1 = b1;
  a.w2 = static_cast<__nv_bfloat16*>(w2);
  a.b2 = b2;
  a.w3 = static_cast<__nv_bfloat16*>(w3);
  a.b3 = b3;
  mlpk::mlp_adam_kernel<<<(mlpk::NPARAM + 255) / 256, 256, 0, as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
