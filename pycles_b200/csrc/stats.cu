// Horizontal statistics on the device: the reductions of ParallelMPI.pyx
// (HorizontalMean :196-241, HorizontalMeanofSquares :243-289,
// HorizontalMeanofCubes :291-325, HorizontalMaximum :327-357,
// HorizontalMinimum :359-389, HorizontalMeanSurface :391-428,
// HorizontalMeanConditional :430-483, HorizontalMeanofSquaresConditional
// :485-540) on one rank, so statistics need no host copy of a field.
//
// Two launches, both with a fixed partition and a fixed order of the sums
// (the result does not depend on scheduling): stat_partial -- block b takes
// a contiguous chunk of the interior columns, one thread per level k, and
// writes its per-level partial (and the mask's partial for the conditional
// means); stat_final -- one block per level sums the partials in a fixed
// tree and applies the reference's normalisation.  Each field is read once
// (k contiguous: coalesced).  Compiled with -fmad=false: the products are
// rounded before they are added, as in the reference's loops.
#include <string.h>

#include "pb_common.cuh"

namespace {
namespace stk {

constexpr int kParts = 296;   // 2 x 148 SMs
constexpr int kThreads = 128;
constexpr int kFinal = 256;

struct A {
  long long n0, n1, n2, is, js, gw;
  const double* v[3];
  const double* mask;
  double* partial;  // [2][kParts][n2]
  double* out;
  double n_horizontal_i;
};

template <int KIND>
__device__ __forceinline__ double term(const A& a, long long o) {
  if (KIND == PB_STAT_MEAN || KIND == PB_STAT_MAX || KIND == PB_STAT_MIN) return a.v[0][o];
  if (KIND == PB_STAT_MEAN_SQUARES) return a.v[0][o] * a.v[1][o];
  if (KIND == PB_STAT_MEAN_CUBES) return a.v[0][o] * a.v[1][o] * a.v[2][o];
  if (KIND == PB_STAT_MEAN_CONDITIONAL) return a.v[0][o] * a.mask[o];
  return a.v[0][o] * a.v[1][o] * a.mask[o];  // PB_STAT_MEAN_SQUARES_CONDITIONAL
}

template <int KIND>
__device__ __forceinline__ double combine(double s, double t) {
  if (KIND == PB_STAT_MAX) return fmax(s, t);
  if (KIND == PB_STAT_MIN) return fmin(s, t);
  return s + t;
}

template <int KIND>
__device__ __forceinline__ double identity() {
  // HorizontalMaximum / HorizontalMinimum start from -9e12 / 9e12
  return KIND == PB_STAT_MAX ? -9e12 : (KIND == PB_STAT_MIN ? 9e12 : 0.0);
}

template <int KIND>
__global__ void __launch_bounds__(kThreads) stat_partial(A a) {
  constexpr bool COND = KIND == PB_STAT_MEAN_CONDITIONAL || KIND == PB_STAT_MEAN_SQUARES_CONDITIONAL;
  const long long nl0 = a.n0 - 2 * a.gw, nl1 = a.n1 - 2 * a.gw;
  const long long ncol = nl0 * nl1;
  const long long per = (ncol + kParts - 1) / kParts;
  const long long c0 = (long long)blockIdx.x * per;
  const long long c1 = min(ncol, c0 + per);
  const long long k = (long long)blockIdx.y * kThreads + threadIdx.x;
  if (k >= a.n2) return;
  double s = identity<KIND>(), m = 0.0;
  if (c0 < c1) {
    long long i = a.gw + c0 / nl1, j = a.gw + c0 % nl1;
    long long off = i * a.is + j * a.js + k;
    for (long long c = c0; c < c1; ++c) {
      s = combine<KIND>(s, term<KIND>(a, off));
      if (COND) m += a.mask[off];
      off += a.js;
      if (++j == a.gw + nl1) {
        j = a.gw;
        off += a.is - nl1 * a.js;
      }
    }
  }
  a.partial[(long long)blockIdx.x * a.n2 + k] = s;
  if (COND) a.partial[(long long)(kParts + blockIdx.x) * a.n2 + k] = m;
}

template <int KIND>
__global__ void __launch_bounds__(kFinal) stat_final(A a) {
  constexpr bool COND = KIND == PB_STAT_MEAN_CONDITIONAL || KIND == PB_STAT_MEAN_SQUARES_CONDITIONAL;
  __shared__ double red[kFinal], redm[kFinal];
  const long long k = blockIdx.x;
  double s = identity<KIND>(), m = 0.0;
  for (int b = threadIdx.x; b < kParts; b += kFinal) {
    s = combine<KIND>(s, a.partial[(long long)b * a.n2 + k]);
    if (COND) m += a.partial[(long long)(kParts + b) * a.n2 + k];
  }
  red[threadIdx.x] = s;
  redm[threadIdx.x] = m;
  __syncthreads();
  for (int h = kFinal / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      red[threadIdx.x] = combine<KIND>(red[threadIdx.x], red[threadIdx.x + h]);
      if (COND) redm[threadIdx.x] += redm[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (KIND == PB_STAT_MAX || KIND == PB_STAT_MIN) a.out[k] = red[0];
  else if (COND) a.out[k] = red[0] / fmax(redm[0], 1.0);  // mean / np.maximum(sum, 1.0)
  else a.out[k] = red[0] * a.n_horizontal_i;
}

// HorizontalMeanSurface: one plane of nlg0*nlg1 values, interior columns.
__global__ void __launch_bounds__(kFinal) stat_surface(A a) {
  __shared__ double red[kFinal];
  const long long nl0 = a.n0 - 2 * a.gw, nl1 = a.n1 - 2 * a.gw;
  const long long ncol = nl0 * nl1;
  double s = 0.0;
  for (long long c = threadIdx.x; c < ncol; c += kFinal) {
    const long long i = a.gw + c / nl1, j = a.gw + c % nl1;
    s += a.v[0][i * a.n1 + j];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = kFinal / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.out[0] = red[0] * a.n_horizontal_i;
}

template <int KIND>
void launch(const A& a, cudaStream_t st) {
  const dim3 g1(kParts, (unsigned)((a.n2 + kThreads - 1) / kThreads));
  stat_partial<KIND><<<g1, kThreads, 0, st>>>(a);
  pb_note_launch();
  stat_final<KIND><<<(unsigned)a.n2, kFinal, 0, st>>>(a);
  pb_note_launch();
}

}  // namespace stk
}  // namespace

extern "C" long long pb_stat_workspace_bytes(const pb_dims* dims) {
  if (pb_check_dims(dims)) return -1;
  return 2LL * stk::kParts * dims->nlg[2] * (long long)sizeof(double);
}

extern "C" int pb_horizontal_stat(const pb_dims* dims, int kind, const double* v1, const double* v2,
                                  const double* v3, const double* mask, double* out, void* workspace,
                                  long long workspace_bytes, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!v1 || !out) return PB_ERR_ARG;
  stk::A a;
  memset(&a, 0, sizeof(a));
  a.n0 = dims->nlg[0];
  a.n1 = dims->nlg[1];
  a.n2 = dims->nlg[2];
  a.js = dims->nlg[2];
  a.is = (long long)dims->nlg[1] * dims->nlg[2];
  a.gw = dims->gw;
  a.v[0] = v1;
  a.v[1] = v2;
  a.v[2] = v3;
  a.mask = mask;
  a.out = out;
  a.n_horizontal_i = 1.0 / (double)(dims->n[1] * dims->n[0]);
  cudaStream_t st = as_stream(stream);
  if (kind == PB_STAT_MEAN_SURFACE) {
    stk::stat_surface<<<1, stk::kFinal, 0, st>>>(a);
    pb_note_launch();
    PB_LAUNCH_CHECK();
    return PB_OK;
  }
  const bool two = kind == PB_STAT_MEAN_SQUARES || kind == PB_STAT_MEAN_CUBES ||
                   kind == PB_STAT_MEAN_SQUARES_CONDITIONAL;
  const bool cond = kind == PB_STAT_MEAN_CONDITIONAL || kind == PB_STAT_MEAN_SQUARES_CONDITIONAL;
  if ((two && !v2) || (kind == PB_STAT_MEAN_CUBES && !v3) || (cond && !mask)) return PB_ERR_ARG;
  if (!workspace || workspace_bytes < pb_stat_workspace_bytes(dims)) return PB_ERR_WORKSPACE;
  if ((reinterpret_cast<uintptr_t>(workspace) & 7) != 0) return PB_ERR_ARG;
  a.partial = static_cast<double*>(workspace);
  switch (kind) {
    case PB_STAT_MEAN: stk::launch<PB_STAT_MEAN>(a, st); break;
    case PB_STAT_MEAN_SQUARES: stk::launch<PB_STAT_MEAN_SQUARES>(a, st); break;
    case PB_STAT_MEAN_CUBES: stk::launch<PB_STAT_MEAN_CUBES>(a, st); break;
    case PB_STAT_MAX: stk::launch<PB_STAT_MAX>(a, st); break;
    case PB_STAT_MIN: stk::launch<PB_STAT_MIN>(a, st); break;
    case PB_STAT_MEAN_CONDITIONAL: stk::launch<PB_STAT_MEAN_CONDITIONAL>(a, st); break;
    case PB_STAT_MEAN_SQUARES_CONDITIONAL: stk::launch<PB_STAT_MEAN_SQUARES_CONDITIONAL>(a, st); break;
    default: return PB_ERR_ARG;
  }
  PB_LAUNCH_CHECK();
  return PB_OK;
}
