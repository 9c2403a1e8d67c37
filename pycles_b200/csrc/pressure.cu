// Anelastic pressure solve on one GPU.
//
// The reference's pencil transposes (ParallelMPI.Pencil) become a choice of
// layout: the spectral work array is W[k][j][m] (complex, m fastest), so
// the x-FFT reads physical rows and writes contiguous m, the y-FFT works on
// j-lines batched over contiguous m, and the Thomas solver gives one thread
// to each (kx,ky) column with consecutive threads on consecutive m.
//
// The reference transforms the real right-hand side with a complex FFT and
// solves every (kx,ky) column.  The field is real, so the x-spectrum of each
// row is Hermitian, X[n0 - m] = conj(X[m]); the tridiagonal matrix is real
// and depends on kx only through kx^2, which is even in m; so the columns
// m > n0/2 hold the conjugates of the columns n0 - m (with ky reflected) and
// carry no information.  W keeps the n0/2 + 1 columns m = 0..n0/2.  Two real
// rows (levels 2p, 2p+1) share one complex FFT, z = a + i b, and are
// separated by A[m] = (Z[m] + conj Z[n0-m]) / 2, B[m] = (Z[m] - conj Z[n0-m]) / 2i;
// the inverse rebuilds Z = A + i B over all m from the stored half and
// returns a = Re z, b = Im z.  This halves the x-FFT work, and the y-FFT,
// Thomas and spectral-array traffic, with the same mathematics as the
// reference's full-spectrum solve.
//
//   hmean_partial/hmean_final  HorizontalMean(w), deterministic two-pass sum
//   (remove_mean_u3)           w -= mean[k] on every cell, applied where w is
//                              read: in the divergence and in the correction
//   zero_ghosts                divergence ghosts = 0 (the reference zeroes the
//                              whole array before adding the interior terms)
//   fft_x_fwd                  second_order_divergence (d = 0,1,2 in order)
//                              + x-FFT of each (j, k) row
//   fft_y                      y-FFT (forward, or inverse with 1/n1)
//   tdma                       per-column Thomas (SparseSolvers.pyx:24-44) on
//                              the complex coefficients, mode (0,0) := 0
//   fft_x_inv                  inverse x-FFT, 1/n0, real part -> pressure
//   (ghost fill, sym)          DiagnosticVariables.communicate_variable
//   correction                 second_order_pressure_correction
#include <math.h>
#include <string.h>

#include <vector>

#include "pb_common.cuh"

namespace {

constexpr int kPartials = 1184;  // 8 x 148 SMs
constexpr int kFftThreads = 256;  // stockham_pass: nlines * N <= 16 * kFftThreads

struct PLayout {
  long long partial, mean, twx, twy, twxf, twyf, kx2, ky2, spec, scr, total;
};

long long align256(long long x) { return (x + 255) / 256 * 256; }

PLayout playout(const pb_dims* d) {
  PLayout L;
  const long long n0 = d->n[0], n1 = d->n[1], n2 = d->n[2];
  const long long nlg2 = d->nlg[2];
  long long off = 0;
  L.partial = off; off += align256((long long)kPartials * nlg2 * 8);
  L.mean = off;    off += align256(nlg2 * 8);
  L.twx = off;     off += align256(n0 * 16);
  L.twy = off;     off += align256(n1 * 16);
  L.twxf = off;    off += align256(n0 * 8);
  L.twyf = off;    off += align256(n1 * 8);
  L.kx2 = off;     off += align256(n0 * 8);
  L.ky2 = off;     off += align256(n1 * 8);
  // spectral array W[k][j][m], m < n0/2 + 1 (Hermitian half in x)
  L.spec = off;    off += align256((n0 / 2 + 1) * n1 * n2 * 16);
  L.scr = off;     off += align256((n0 / 2 + 1) * n1 * n2 * 8);
  L.total = off;
  return L;
}

__device__ __forceinline__ bool is_pow2(int n) { return (n & (n - 1)) == 0; }

// Lines per FFT block for a power-of-two length 2^lg (16 lines, or fewer so
// that a block's passes hold nlines * N <= 16 * kFftThreads elements); the
// host's lines_for gives the same count for every power of two.
__host__ __device__ constexpr int ct_lines(int lg) { return (16 * 256 >> lg) < 16 ? (16 * 256 >> lg) : 16; }

// Complex arithmetic on double2 (plain form) or float2 (precision form).
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
template <class C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.0f, 0.0f); }
template <class C> __device__ __forceinline__ C creal(double x);
template <> __device__ __forceinline__ double2 creal<double2>(double x) { return make_double2(x, 0.0); }
template <> __device__ __forceinline__ float2 creal<float2>(double x) { return make_float2((float)x, 0.0f); }

// ---- line FFTs in shared memory --------------------------------------------
// A block transforms `nlines` lines of length N held in shared memory.  Line l
// element x lives at l*line_ld(N) + swz(x): the swizzle (one pad element per
// 8) and the odd line stride keep the strided accesses of the passes and of
// the global loads/stores (consecutive threads on consecutive lines) free of
// bank conflicts.
// The stride is chosen for the transposing loads and stores: a half-warp
// touches IC lines at 16/IC consecutive positions (IC = 4096/N lines for
// powers of two >= 256, 16 below), so with ld = 16/IC (mod 16) its 16
// accesses fall on distinct bank pairs; other lengths take an odd stride.
__host__ __device__ __forceinline__ int line_ld(int N) {
  const int base = N + N / 8;
  if ((N & (N - 1)) != 0 || N < 256) return base + 1;
  const int want = (N / 256) & 15;  // 16 / IC mod 16
  return base + ((want - base % 16) + 16) % 16;
}
__device__ __forceinline__ int swz(int x) { return x + (x >> 3); }

template <class C>
__device__ __forceinline__ C mul_mi(C a, bool inverse) {  // a * (-i), or a * (+i) for the inverse
  C r;
  if (!inverse) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
  return r;
}

// 2-, 4- and 8-point DFTs in registers, y_k = sum_n x_n exp(-+2 pi i n k / R).
template <class C>
__device__ __forceinline__ void dft2(C* v) {
  const C t = v[0];
  v[0] = cadd(t, v[1]);
  v[1] = csub(t, v[1]);
}
template <class C>
__device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3, bool inverse) {
  const C a0 = cadd(x0, x2), a1 = csub(x0, x2);
  const C b0 = cadd(x1, x3), b1 = mul_mi(csub(x1, x3), inverse);
  x0 = cadd(a0, b0);
  x2 = csub(a0, b0);
  x1 = cadd(a1, b1);
  x3 = csub(a1, b1);
}
template <class C>
__device__ __forceinline__ void dft8(C* v, bool inverse) {
  // radix-2 decimation in time over two 4-point DFTs
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4(e0, e1, e2, e3, inverse);
  dft4(o0, o1, o2, o3, inverse);
  using R = decltype(o1.x);
  const R h = (R)0.70710678118654752440;  // 1/sqrt(2)
  C t1, t3;
  if (!inverse) {  // W8 = (1-i)/sqrt2, W8^3 = (-1-i)/sqrt2
    t1.x = (o1.x + o1.y) * h; t1.y = (o1.y - o1.x) * h;
    t3.x = (o3.y - o3.x) * h; t3.y = -(o3.x + o3.y) * h;
  } else {         // conjugates
    t1.x = (o1.x - o1.y) * h; t1.y = (o1.x + o1.y) * h;
    t3.x = -(o3.x + o3.y) * h; t3.y = (o3.x - o3.y) * h;
  }
  const C t2 = mul_mi(o2, inverse);
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1); v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2); v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3); v[7] = csub(e3, t3);
}

// One radix-R pass of the Stockham autosort FFT over all lines, in place:
// every thread reads its items (R values each, stride N/R), twiddles them by
// exp(-+2 pi i (j mod Ns) r / (Ns R)), transforms, and after a barrier
// writes them to (j div Ns) Ns R + (j mod Ns) + r Ns.  Input and output are
// in natural order.  Needs nlines * N <= 16 * kFftThreads (the FFT kernels'
// block size).  When lgN, lgNs and nlines are compile-time constants (the
// kernels instantiated for one length) all index arithmetic folds away.
template <class C, int R>
__device__ __forceinline__ void stockham_pass(C* buf, int nlines, int lgN, int lgNs, const C* __restrict__ tw,
                                              bool inverse) {
  constexpr int MAXI = 16 / R;
  constexpr int lgR = R == 8 ? 3 : (R == 4 ? 2 : 1);
  const int N = 1 << lgN;
  const int lg_per = lgN - lgR;              // per_line = N / R
  const int per_line = 1 << lg_per;
  const int total = nlines << lg_per;
  const int ld = line_ld(N);
  const int lg_tw = lgN - lgNs - lgR;        // twiddle step N / (Ns R)
  const int ns_mask = (1 << lgNs) - 1;
  C v[MAXI][R];
#pragma unroll
  for (int it = 0; it < MAXI; ++it) {
    const int b = threadIdx.x + it * kFftThreads;
    if (b < total) {
      const int l = b >> lg_per;
      const int j = b & (per_line - 1);
      const C* line = buf + l * ld;
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = line[swz(j + r * per_line)];
      if (lgNs > 0) {
        const int k = j & ns_mask;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = tw[(k * r) << lg_tw];
          if (inverse) w.y = -w.y;
          v[it][r] = cmul(v[it][r], w);
        }
      }
      if constexpr (R == 8) dft8(v[it], inverse);
      else if constexpr (R == 4) dft4(v[it][0], v[it][1], v[it][2], v[it][3], inverse);
      else dft2(v[it]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < MAXI; ++it) {
    const int b = threadIdx.x + it * kFftThreads;
    if (b < total) {
      const int l = b >> lg_per;
      const int j = b & (per_line - 1);
      const int k = j & ns_mask;
      const int base = ((j - k) << lgR) + k;
      C* line = buf + l * ld;
#pragma unroll
      for (int r = 0; r < R; ++r) line[swz(base + (r << lgNs))] = v[it][r];
    }
  }
  __syncthreads();
}

// Power-of-two N: radix-8 passes, then one radix-4 or radix-2 pass.
template <class C>
__device__ __forceinline__ void fft_lines_pow2(C* buf, int nlines, int N, const C* __restrict__ tw, bool inverse) {
  const int lgN = __ffs(N) - 1;
  int lgNs = 0;
#pragma unroll
  for (; lgNs + 3 <= lgN; lgNs += 3) stockham_pass<C, 8>(buf, nlines, lgN, lgNs, tw, inverse);
  if (lgNs + 2 == lgN) stockham_pass<C, 4>(buf, nlines, lgN, lgNs, tw, inverse);
  else if (lgNs + 1 == lgN) stockham_pass<C, 2>(buf, nlines, lgN, lgNs, tw, inverse);
}

// e -> (e / d, e % d) with a shift and a mask when d is a power of two
// (the usual case: line counts are powers of two, and so are most N).
__device__ __forceinline__ void split_idx(int e, int d, int& q, int& r) {
  if ((d & (d - 1)) == 0) {
    const int lg = __ffs(d) - 1;
    q = e >> lg;
    r = e & (d - 1);
  } else {
    q = e / d;
    r = e - q * d;
  }
}

// Direct DFT for lengths that are not powers of two: out = DFT(in), both in
// the swizzled line layout.
template <class C>
__device__ void dft_lines(const C* in, C* out, int nlines, int N, const C* __restrict__ tw, bool inverse) {
  const int ld = line_ld(N);
  for (int e = threadIdx.x; e < nlines * N; e += kFftThreads) {
    const int line = e / N;
    const int m = e - line * N;
    C acc = czero<C>();
    const C* x = in + line * ld;
    int idx = 0;
    for (int n = 0; n < N; ++n) {
      C w = tw[idx];
      if (inverse) w.y = -w.y;
      acc = cadd(acc, cmul(w, x[swz(n)]));
      idx += m;
      if (idx >= N) idx -= N;
    }
    out[line * ld + swz(m)] = acc;
  }
  __syncthreads();
}

// Transform the lines in `in`; returns where the result is.
template <class C>
__device__ __forceinline__ C* fft_lines(C* in, int nlines, int maxlines, int N, const C* __restrict__ tw,
                                        bool inverse) {
  if (is_pow2(N)) {
    fft_lines_pow2<C>(in, nlines, N, tw, inverse);
    return in;
  }
  C* out = in + (size_t)maxlines * line_ld(N);
  dft_lines<C>(in, out, nlines, N, tw, inverse);
  return out;
}

struct PArgs {
  const double* rho0;
  const double* rho0_half;
  const double* alpha0;
  const double* alpha0_half;
  double* u;
  double* v;
  double* w;
  double* div;
  double* p;
  double* partial;
  double* mean;
  const double2* twx;
  const double2* twy;
  const float2* twxf;
  const float2* twyf;
  const double* kx2;
  const double* ky2;
  void* spec;     // double2 (plain form) or float2 (precision form) W[k][j][i]
  double* scr;
  // sharded solves (pressure_shard): the x-FFT reads the right-hand side from
  // a dense [i][j][k] interior array, the inverse x-FFT writes the result to
  // one, and the Thomas solve of a slab of j rows starts at global row j0
  const double* src_dense;
  double* dst_dense;
  int j0;
};

template <class C> __device__ __forceinline__ const C* twx_of(const PArgs& a);
template <> __device__ __forceinline__ const double2* twx_of<double2>(const PArgs& a) { return a.twx; }
template <> __device__ __forceinline__ const float2* twx_of<float2>(const PArgs& a) { return a.twxf; }
template <class C> __device__ __forceinline__ const C* twy_of(const PArgs& a);
template <> __device__ __forceinline__ const double2* twy_of<double2>(const PArgs& a) { return a.twy; }
template <> __device__ __forceinline__ const float2* twy_of<float2>(const PArgs& a) { return a.twyf; }

// ---- HorizontalMean (ParallelMPI.pyx:196-241) ------------------------------
// Block b sums a contiguous chunk of interior columns for every level (one
// thread per level, four interleaved accumulators for memory-level
// parallelism); the partition and the order of the sums are fixed, so the
// mean is deterministic.
__global__ void hmean_partial(Geo g, const double* __restrict__ w, double* __restrict__ partial) {
  const long long nl0 = g.n0 - 2 * g.gw, nl1 = g.n1 - 2 * g.gw;
  const long long ncol = nl0 * nl1;
  const long long per = (ncol + gridDim.x - 1) / gridDim.x;
  const long long c0 = (long long)blockIdx.x * per;
  const long long c1 = min(ncol, c0 + per);
  // the chunk's first column, then a walk along j wrapping to the next i
  // (no index division per element)
  const long long i0 = g.gw + c0 / nl1, j0 = g.gw + c0 % nl1;
  for (long long k = threadIdx.x; k < g.n2; k += blockDim.x) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    long long off = i0 * g.is + j0 * g.js + k;
    long long j = j0;
    long long c = c0;
    for (; c + 3 < c1; c += 4) {
      double v[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        v[m] = w[off];
        off += g.js;
        if (++j == g.gw + nl1) {
          j = g.gw;
          off += g.is - nl1 * g.js;
        }
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) s[m] += v[m];
    }
    for (; c < c1; ++c) {
      s[0] += w[off];
      off += g.js;
      if (++j == g.gw + nl1) {
        j = g.gw;
        off += g.is - nl1 * g.js;
      }
    }
    partial[(long long)blockIdx.x * g.n2 + k] = (s[0] + s[1]) + (s[2] + s[3]);
  }
}

// One block per level: each thread sums a fixed strided subset of the
// partials, then a fixed-order tree in shared memory (deterministic).
__global__ void hmean_final(Geo g, const double* __restrict__ partial, double* __restrict__ mean, int np,
                            double n_horizontal_i) {
  __shared__ double red[256];
  const long long k = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < np; b += blockDim.x) s += partial[(long long)b * g.n2 + k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) mean[k] = red[0] * n_horizontal_i;
}

// Plain form: HorizontalMean in the reference's order (ParallelMPI.pyx:219-
// 226).  Each level's sum is one chain of rounded additions over the
// interior columns, i outer and j inner, which no reordering may change:
// w's horizontal mean cancels, and the solve subtracts it from every cell.
// A block owns 32 levels, one lane each.  Warp 0 only adds: it walks a tile
// of kSerialTile columns in shared memory, one dependent addition per column,
// while the other 31 warps load the next tile (kSerialPer columns each, all
// loads in flight at once) into the other half of a double buffer.
constexpr int kSerialWarps = 32;
constexpr int kSerialPer = 12;
constexpr int kSerialTile = (kSerialWarps - 1) * kSerialPer;  // columns per tile
constexpr int kSerialLd = 33;  // doubles per column in the tile (odd: no bank conflicts)
__global__ void __launch_bounds__(kSerialWarps * 32, 1) hmean_serial(Geo g, const double* __restrict__ w,
                                                                     double* __restrict__ mean,
                                                                     double n_horizontal_i) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* tile = reinterpret_cast<double*>(smraw);  // [2][kSerialTile][kSerialLd]
  const int nl1 = (int)(g.n1 - 2 * g.gw);
  const int ncol = (int)(g.n0 - 2 * g.gw) * nl1;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long k = (long long)blockIdx.x * 32 + lane;
  const bool kok = k < g.n2;
  const int ntiles = (ncol + kSerialTile - 1) / kSerialTile;
  auto produce = [&](int t) {
    double v[kSerialPer];
#pragma unroll
    for (int q = 0; q < kSerialPer; ++q) {
      const int col = t * kSerialTile + (wid - 1) * kSerialPer + q;
      v[q] = 0.0;
      if (col < ncol && kok) {
        const int i = col / nl1, j = col - (col / nl1) * nl1;
        v[q] = w[(g.gw + i) * g.is + (g.gw + j) * g.js + k];
      }
    }
    double* dst = tile + (t & 1) * kSerialTile * kSerialLd + (wid - 1) * kSerialPer * kSerialLd + lane;
#pragma unroll
    for (int q = 0; q < kSerialPer; ++q) dst[q * kSerialLd] = v[q];
  };
  double s = 0.0;
  if (wid > 0) produce(0);
  __syncthreads();
  for (int t = 0; t < ntiles; ++t) {
    if (wid > 0) {
      if (t + 1 < ntiles) produce(t + 1);
    } else {
      const double* cur = tile + (t & 1) * kSerialTile * kSerialLd + lane;
      const int nc = min(kSerialTile, ncol - t * kSerialTile);
      if (nc == kSerialTile) {
#pragma unroll 12
        for (int c = 0; c < kSerialTile; ++c) s = add_rn(s, cur[c * kSerialLd]);
      } else {
        for (int c = 0; c < nc; ++c) s = add_rn(s, cur[c * kSerialLd]);
      }
    }
    __syncthreads();
  }
  if (wid == 0 && kok) mean[k] = mul_rn(s, n_horizontal_i);
}

__global__ void zero_ghosts(Geo g, double* __restrict__ f, long long nghost) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nghost; t += stride) {
    long long i, j, k;
    ghost_decode(g, t, i, j, k);
    f[i * g.is + j * g.js + k] = 0.0;
  }
}

// Right-hand side of the forward x-FFT (fft_x_fwd's SRC) and destination of
// the inverse (fft_x_inv's DST).
constexpr int kSrcDivergence = 0, kSrcResidual = 1, kSrcDense = 2;
constexpr int kDstWrite = 0, kDstAccumulate = 1, kDstDense = 2;

// second_order_divergence (PressureSolver.pyx:138-175, d = 0, 1, 2 in order)
// of the cell ijk at level k, w taken after remove_mean_u3 (w - mean[k]).
// Plain form: the reference's divisions by alpha0 in its order, separately
// rounded; precision form: multiplications by rho0 = 1/alpha0.
template <bool PLAIN>
__device__ __forceinline__ double divergence_at(const Geo& g, const PArgs& a, long long ijk, long long k) {
  const double* __restrict__ U = a.u;
  const double* __restrict__ V = a.v;
  const double* __restrict__ Wv = a.w;
  const double wc = sub_rn(Wv[ijk], a.mean[k]);
  const double wm = sub_rn(Wv[ijk - 1], a.mean[k - 1]);
  if constexpr (PLAIN) {
    const double ah = a.alpha0_half[k];
    double d = 0.0;
    d = add_rn(d, mul_rn(sub_rn(U[ijk] / ah, U[ijk - g.is] / ah), g.dxi0));
    d = add_rn(d, mul_rn(sub_rn(V[ijk] / ah, V[ijk - g.js] / ah), g.dxi1));
    d = add_rn(d, mul_rn(sub_rn(wc / a.alpha0[k], wm / a.alpha0[k - 1]), g.dxi2));
    return d;
  } else {
    const double rh = a.rho0_half[k];
    return (U[ijk] - U[ijk - g.is]) * rh * g.dxi0 + (V[ijk] - V[ijk - g.js]) * rh * g.dxi1 +
           (wc * a.rho0[k] - wm * a.rho0[k - 1]) * g.dxi2;
  }
}

// The refinement residual div - A p of the cell ijk (level k, kk = k - gw),
// A the operator the spectral solve inverts: second differences in x and y,
// the rows of compute_off_diagonals / compute_diagonal in z.
__device__ __forceinline__ double residual_at(const Geo& g, const PArgs& a, long long ijk, long long k, long long kk,
                                              long long nz) {
  const double* __restrict__ p = a.p;
  const double pc = p[ijk];
  const double lap_h = a.rho0_half[k] * ((p[ijk + g.is] - 2.0 * pc + p[ijk - g.is]) * (g.dxi0 * g.dxi0) +
                                         (p[ijk + g.js] - 2.0 * pc + p[ijk - g.js]) * (g.dxi1 * g.dxi1));
  double vert = 0.0;
  if (kk < nz - 1) vert += a.rho0[k] * (p[ijk + 1] - pc);
  if (kk > 0) vert -= a.rho0[k - 1] * (pc - p[ijk - 1]);
  return a.div[ijk] - (lap_h + vert * (g.dxi2 * g.dxi2));
}

// ---- divergence (or refinement residual) + forward x-FFT --------------------
// block = (interior j, chunk of KC = 2 LC interior levels); smem LC complex
// lines of n0, line p holding levels 2p (real part) and 2p + 1 (imaginary).
// SRC = kSrcDivergence: the right-hand side is second_order_divergence
//   (divergence_at), written to `div`.
// SRC = kSrcResidual: the right-hand side is the residual div - A p of the
//   current pressure (residual_at); used by the iterative refinement of the
//   precision form.
// SRC = kSrcDense: the right-hand side is read from a dense interior array
//   (a slab of levels of a sharded solve).
//
// LGN > 0 instantiates the kernel for N = 2^LGN (KC = 2 ct_lines(LGN)), so
// that the index arithmetic and the FFT passes are compile-time; LGN = 0
// takes N and KC at run time.
template <class C, int SRC, int LGN>
__global__ void __launch_bounds__(kFftThreads) fft_x_fwd(Geo g, PArgs a, int KCrt) {
  using R = decltype(C().x);
  constexpr bool CT = LGN > 0;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* in = reinterpret_cast<C*>(smraw);
  R* inr = reinterpret_cast<R*>(smraw);
  const int N = CT ? (1 << LGN) : (int)(g.n0 - 2 * g.gw);
  const int KC = CT ? 2 * ct_lines(LGN) : KCrt;
  const int Nh = N / 2 + 1;
  const int nz = (int)(g.n2 - 2 * g.gw);
  const int jl = blockIdx.x;
  const int k0 = blockIdx.y * KC;
  const int kc = min(KC, nz - k0);
  const int lc = (kc + 1) >> 1;
  const long long j = g.gw + jl;
  const int ld = line_ld(N);
  const long long ny = g.n1 - 2 * g.gw;
  double* __restrict__ div = a.div;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * KC; e += kFftThreads) {
    int kl, il;
    split_idx(e, KC, il, kl);
    const int slot = 2 * ((kl >> 1) * ld + swz(il)) + (kl & 1);
    if (kl >= kc) {  // the imaginary half of an odd chunk's last line
      inr[slot] = (R)0;
      continue;
    }
    const long long k = g.gw + k0 + kl;
    const long long ijk = (g.gw + il) * g.is + j * g.js + k;
    double d;
    if constexpr (SRC == kSrcDivergence) {
      d = divergence_at<sizeof(C) == sizeof(double2)>(g, a, ijk, k);
      div[ijk] = d;
    } else if constexpr (SRC == kSrcResidual) {
      d = residual_at(g, a, ijk, k, k - g.gw, nz);
    } else {  // a dense interior array (il, jl, k0 + kl)
      d = a.src_dense[((long long)il * ny + jl) * nz + k0 + kl];
    }
    inr[slot] = (R)d;
  }
  __syncthreads();
  const C* res = fft_lines<C>(in, CT ? (KC >> 1) : lc, KC >> 1, N, twx_of<C>(a), false);
  // separate the two rows of each line; write the columns m = 0..N/2
  C* spec = reinterpret_cast<C*>(a.spec);
  const long long nxy = (long long)Nh * (g.n1 - 2 * g.gw);
  const R half = (R)0.5;
#pragma unroll 4
  for (int e = threadIdx.x; e < Nh * kc; e += kFftThreads) {
    const int kl = e / Nh;
    const int m = e - kl * Nh;
    const C* line = res + (kl >> 1) * ld;
    const C z = line[swz(m)];
    const C zr = line[swz(m == 0 ? 0 : N - m)];  // Z[N - m]
    C o;
    if ((kl & 1) == 0) {  // A = (Z[m] + conj Z[N-m]) / 2
      o.x = (z.x + zr.x) * half;
      o.y = (z.y - zr.y) * half;
    } else {              // B = (Z[m] - conj Z[N-m]) / 2i
      o.x = (z.y + zr.y) * half;
      o.y = (zr.x - z.x) * half;
    }
    spec[(long long)(k0 + kl) * nxy + (long long)jl * Nh + m] = o;
  }
}

// ---- y-FFT over W[k][j][m] lines along j, IC columns m per block ----------
// (LGN as for fft_x_fwd: N = 2^LGN and IC = ct_lines(LGN) at compile time.)
template <class C, bool INV, int LGN>
__global__ void __launch_bounds__(kFftThreads) fft_y(Geo g, PArgs a, int ICrt) {
  constexpr bool CT = LGN > 0;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* in = reinterpret_cast<C*>(smraw);
  const int Nx = (int)(g.n0 - 2 * g.gw) / 2 + 1;  // stored x-modes
  const int N = CT ? (1 << LGN) : (int)(g.n1 - 2 * g.gw);
  const int IC = CT ? ct_lines(LGN) : ICrt;
  const int kk = blockIdx.y;
  const int i0 = blockIdx.x * IC;
  const int ic = min(IC, Nx - i0);
  const int ld = line_ld(N);
  C* plane = reinterpret_cast<C*>(a.spec) + (long long)kk * N * Nx;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * IC; e += kFftThreads) {
    int il, jl;
    split_idx(e, IC, jl, il);
    if (il >= ic) continue;
    in[il * ld + swz(jl)] = plane[(long long)jl * Nx + i0 + il];
  }
  __syncthreads();
  const C* res = fft_lines<C>(in, CT ? IC : ic, IC, N, twy_of<C>(a), INV);
  const double sc = INV ? 1.0 / (double)N : 1.0;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * IC; e += kFftThreads) {
    int il, jl;
    split_idx(e, IC, jl, il);
    if (il >= ic) continue;
    C r = res[il * ld + swz(jl)];
    if (INV) {
      r.x *= sc;
      r.y *= sc;
    }
    plane[(long long)jl * Nx + i0 + il] = r;
  }
}

__device__ __forceinline__ void to_d(double2 c, double& x, double& y) { x = c.x; y = c.y; }
__device__ __forceinline__ void to_d(float2 c, double& x, double& y) { x = c.x; y = c.y; }
template <class C> __device__ __forceinline__ C from_d(double x, double y);
template <> __device__ __forceinline__ double2 from_d<double2>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 from_d<float2>(double x, double y) {
  return make_float2((float)x, (float)y);
}

// ---- per-column tridiagonal solve (always FP64 arithmetic) -----------------
// Matrix of PressureFFTParallel.compute_off_diagonals (:100-127) and
// compute_diagonal (:129-148); Thomas algorithm of TDMA.solve applied to the
// real and imaginary parts (the matrix is real, so both share m and scratch).
template <class C>
__global__ void __launch_bounds__(256, sizeof(C) == 8 ? 4 : 2) tdma_kernel(Geo g, PArgs a) {
  const int Nx = (int)(g.n0 - 2 * g.gw) / 2 + 1;  // stored x-modes
  const int Ny = (int)(g.n1 - 2 * g.gw);
  const int nz = (int)(g.n2 - 2 * g.gw);
  const long long ncol = (long long)Nx * Ny;
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int i = (int)(col % Nx);
  const int j = (int)(col / Nx) + a.j0;  // global row (a slab of rows in a sharded solve)
  C* x = reinterpret_cast<C*>(a.spec) + col;
  double* scr = a.scr + col;
  if (i == 0 && j == 0) {  // mode (0,0) is set to zero (:197-200)
    for (int k = 0; k < nz; ++k) x[(long long)k * ncol] = from_d<C>(0.0, 0.0);
    return;
  }
  const long long gw = g.gw;
  const double dzi = g.dxi2;
  const double kk = a.kx2[i] + a.ky2[j];
  const double* rho0 = a.rho0;
  const double* rho0h = a.rho0_half;
  // row 0 (for a single level the last-row formulas overwrite it, :119-127, :145-146)
  double b, c;
  if (nz > 1) {
    b = sub_rn(mul_rn(rho0h[gw], kk), mul_rn(mul_rn(rho0[gw], dzi), dzi));
    c = mul_rn(mul_rn(dzi, dzi), rho0[gw]);
  } else {
    b = sub_rn(mul_rn(rho0h[gw], kk), mul_rn(mul_rn(rho0[gw - 1], dzi), dzi));
    c = 0.0;
  }
  double s_prev = c / b;
  double xpx, xpy;
  to_d(x[0], xpx, xpy);
  xpx = xpx / b;
  xpy = xpy / b;
  x[0] = from_d<C>(xpx, xpy);
  scr[0] = s_prev;
  // The sweeps walk the levels in batches of kB; the loads of the next batch
  // are issued before the current one is processed, so every thread keeps
  // kB independent loads in flight behind its serial recurrence.
  constexpr int kB = sizeof(C) == 8 ? 4 : 8;  // FP32 spectra: 4 blocks per SM at 64 registers
  C cur[kB], nxt[kB];
#pragma unroll
  for (int m = 0; m < kB; ++m) cur[m] = (1 + m < nz) ? x[(long long)(1 + m) * ncol] : from_d<C>(0.0, 0.0);
  for (int kb = 1; kb < nz; kb += kB) {
#pragma unroll
    for (int m = 0; m < kB; ++m) {
      const int kn = kb + kB + m;
      nxt[m] = (kn < nz) ? x[(long long)kn * ncol] : from_d<C>(0.0, 0.0);
    }
#pragma unroll
    for (int m = 0; m < kB; ++m) {
      const int k = kb + m;
      if (k < nz) {
        const double ak = mul_rn(mul_rn(dzi, dzi), rho0[k + gw - 1]);
        double ck, bk;
        if (k < nz - 1) {
          ck = mul_rn(mul_rn(dzi, dzi), rho0[k + gw]);
          bk = sub_rn(mul_rn(rho0h[k + gw], kk), mul_rn(mul_rn(add_rn(rho0[k + gw], rho0[k + gw - 1]), dzi), dzi));
        } else {
          ck = 0.0;
          bk = sub_rn(mul_rn(rho0h[k + gw], kk), mul_rn(mul_rn(rho0[k + gw - 1], dzi), dzi));
        }
        const double m_ = 1.0 / sub_rn(bk, mul_rn(ak, s_prev));
        s_prev = mul_rn(ck, m_);
        scr[(long long)k * ncol] = s_prev;
        double xkx, xky;
        to_d(cur[m], xkx, xky);
        xkx = mul_rn(sub_rn(xkx, mul_rn(ak, xpx)), m_);
        xky = mul_rn(sub_rn(xky, mul_rn(ak, xpy)), m_);
        x[(long long)k * ncol] = from_d<C>(xkx, xky);
        xpx = xkx;
        xpy = xky;
      }
    }
#pragma unroll
    for (int m = 0; m < kB; ++m) cur[m] = nxt[m];
  }
  // back substitution from the last value, reading the stored sweep values,
  // in batches of kB levels going down
  double scur[kB], snxt[kB];
#pragma unroll
  for (int m = 0; m < kB; ++m) {
    const int k = nz - 2 - m;
    cur[m] = (k >= 0) ? x[(long long)k * ncol] : from_d<C>(0.0, 0.0);
    scur[m] = (k >= 0) ? scr[(long long)k * ncol] : 0.0;
  }
  for (int kb = nz - 2; kb >= 0; kb -= kB) {
#pragma unroll
    for (int m = 0; m < kB; ++m) {
      const int kn = kb - kB - m;
      nxt[m] = (kn >= 0) ? x[(long long)kn * ncol] : from_d<C>(0.0, 0.0);
      snxt[m] = (kn >= 0) ? scr[(long long)kn * ncol] : 0.0;
    }
#pragma unroll
    for (int m = 0; m < kB; ++m) {
      const int k = kb - m;
      if (k >= 0) {
        double xkx, xky;
        to_d(cur[m], xkx, xky);
        xkx = sub_rn(xkx, mul_rn(scur[m], xpx));
        xky = sub_rn(xky, mul_rn(scur[m], xpy));
        x[(long long)k * ncol] = from_d<C>(xkx, xky);
        xpx = xkx;
        xpy = xky;
      }
    }
#pragma unroll
    for (int m = 0; m < kB; ++m) {
      cur[m] = nxt[m];
      scur[m] = snxt[m];
    }
  }
}

// ---- inverse x-FFT -> pressure ----------------------------------------------
// DST = kDstWrite: write the pressure; kDstAccumulate: add to the current
// pressure (refinement); kDstDense: write a dense interior array (a slab of
// levels of a sharded solve).
// block = (interior j, chunk of KC = 2 LC levels).  Line p gets
// Z = A + i B over all m, A and B the stored half-spectra of levels 2p and
// 2p + 1 extended by A[N-m] = conj A[m]; the inverse transform returns the
// two real rows as Re z and Im z.
// (LGN as for fft_x_fwd.)
template <class C, int DST, int LGN>
__global__ void __launch_bounds__(kFftThreads) fft_x_inv(Geo g, PArgs a, int KCrt) {
  constexpr bool ACC = DST == kDstAccumulate;
  constexpr bool CT = LGN > 0;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* in = reinterpret_cast<C*>(smraw);
  const int N = CT ? (1 << LGN) : (int)(g.n0 - 2 * g.gw);
  const int KC = CT ? 2 * ct_lines(LGN) : KCrt;
  const int Nh = N / 2 + 1;
  const int nz = (int)(g.n2 - 2 * g.gw);
  const int jl = blockIdx.x;
  const int k0 = blockIdx.y * KC;
  const int kc = min(KC, nz - k0);
  const int lc = (kc + 1) >> 1;
  const int ld = line_ld(N);
  const C* spec = reinterpret_cast<const C*>(a.spec);
  const long long nxy = (long long)Nh * (g.n1 - 2 * g.gw);
#pragma unroll 4
  for (int e = threadIdx.x; e < Nh * lc; e += kFftThreads) {
    const int p = e / Nh;
    const int m = e - p * Nh;
    const long long src = (long long)(k0 + 2 * p) * nxy + (long long)jl * Nh + m;
    const C A = spec[src];
    const C B = (2 * p + 1 < kc) ? spec[src + nxy] : czero<C>();
    C* line = in + p * ld;
    C z;
    z.x = A.x - B.y;
    z.y = A.y + B.x;
    line[swz(m)] = z;
    if (m >= 1 && m <= N - Nh) {  // Z[N-m] = conj A[m] + i conj B[m]
      C zr;
      zr.x = A.x + B.y;
      zr.y = B.x - A.y;
      line[swz(N - m)] = zr;
    }
  }
  __syncthreads();
  const C* res = fft_lines<C>(in, CT ? (KC >> 1) : lc, KC >> 1, N, twx_of<C>(a), true);
  const double sc = 1.0 / (double)N;
  const long long j = g.gw + jl;
  double* __restrict__ p = a.p;
  if constexpr (DST == kDstDense) {
    const long long ny = g.n1 - 2 * g.gw;
    for (int e = threadIdx.x; e < N * KC; e += kFftThreads) {
      int kl = 0, il = 0;
      split_idx(e, KC, il, kl);
      if (kl >= kc) continue;
      const C z = res[(kl >> 1) * ld + swz(il)];
      a.dst_dense[((long long)il * ny + jl) * nz + k0 + kl] = (double)((kl & 1) ? z.y : z.x) * sc;
    }
    return;
  }
  // batches of kBatch elements: the pressure loads of a batch (ACC) are all
  // issued before its stores
  constexpr int kBatch = 8;
  for (int e0 = threadIdx.x; e0 < N * KC; e0 += kBatch * kFftThreads) {
    long long ijk[kBatch];
    double val[kBatch], old[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int e = e0 + b * kFftThreads;
      int kl = 0, il = 0;
      split_idx(e, KC, il, kl);
      const bool ok = e < N * KC && kl < kc;
      ijk[b] = ok ? (g.gw + il) * g.is + j * g.js + g.gw + k0 + kl : -1;
      if (ok) {
        const C z = res[(kl >> 1) * ld + swz(il)];
        val[b] = (double)((kl & 1) ? z.y : z.x) * sc;
      }
      old[b] = (ACC && ok) ? p[ijk[b]] : 0.0;
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (ijk[b] >= 0) p[ijk[b]] = ACC ? old[b] + val[b] : val[b];
  }
}

// ---- pressure ghost fill (sym), communicate_variable on one rank -----------
__global__ void ghost_sym(Geo g, double* __restrict__ f, long long nghost) {
  const long long gw = g.gw, n0 = g.n0, n1 = g.n1, n2 = g.n2;
  const long long nl0 = n0 - 2 * gw, nl1 = n1 - 2 * gw;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nghost; t += stride) {
    long long i, j, k;
    ghost_decode(g, t, i, j, k);
    const long long is_ = (i < gw) ? i + nl0 : ((i >= n0 - gw) ? i - nl0 : i);
    const long long js_ = (j < gw) ? j + nl1 : ((j >= n1 - gw) ? j - nl1 : j);
    long long ks = k;
    if (k >= n2 - gw) ks = n2 - gw - 1 - (k - (n2 - gw));
    else if (k < gw) ks = gw + (gw - 1 - k);
    f[i * g.is + j * g.js + k] = f[is_ * g.is + js_ * g.js + ks];
  }
}

// ---- second_order_pressure_correction (PressureSolver.pyx:83-110) ---------
// w enters as it was before remove_mean_u3; every cell first gets w - mean[k]
// (the reference's remove_mean_u3 over all cells), then the correction on
// [0, nlg-1) in every dimension.
__global__ void correction(Geo g, const double* __restrict__ p, double* __restrict__ u, double* __restrict__ v,
                           double* __restrict__ w, const double* __restrict__ mean) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < g.npg; t += stride) {
    const long long k = t % g.n2;
    const long long r = t / g.n2;
    const long long j = r % g.n1;
    const long long i = r / g.n1;
    const double wt = sub_rn(w[t], mean[k]);
    if (i >= g.n0 - 1 || j >= g.n1 - 1 || k >= g.n2 - 1) {
      w[t] = wt;
      continue;
    }
    const double pc = p[t];
    u[t] = sub_rn(u[t], mul_rn(sub_rn(p[t + g.is], pc), g.dxi0));
    v[t] = sub_rn(v[t], mul_rn(sub_rn(p[t + g.js], pc), g.dxi1));
    w[t] = sub_rn(wt, mul_rn(sub_rn(p[t + 1], pc), g.dxi2));
  }
}

int stream_blocks(long long work) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long b = (work + 255) / 256;
  if (b > (long long)sms * 8) b = (long long)sms * 8;
  return (int)(b < 1 ? 1 : b);
}

bool pow2(long long n) { return (n & (n - 1)) == 0; }

// Horizontal sizes the line FFTs support: powers of two up to 4096 (a
// block's Stockham passes hold at most 16 * kFftThreads elements, one line of
// 4096) and other lengths up to 1024 (direct DFT).
bool fft_sizes_ok(const pb_dims* d) {
  for (int dim = 0; dim < 2; ++dim) {
    const long long n = d->n[dim];
    if (pow2(n) ? n > 4096 : n > 1024) return false;
  }
  return true;
}

size_t fft_smem(long long N, int lines, size_t elem) {
  return (size_t)(pow2(N) ? 1 : 2) * (size_t)line_ld((int)N) * lines * elem;
}

// Lines per FFT block: a power of two, up to 16, with nlines * N <=
// 16 * kFftThreads for the Stockham passes and the block's shared memory
// within 48 KiB (FP32) / 80 KiB (FP64), so that several blocks share an SM
// and one block's loads overlap another's passes.
int lines_for(long long N, size_t elem) {
  const long long per = (pow2(N) ? 1 : 2) * (long long)line_ld((int)N) * (long long)elem;
  long long L = (elem <= 8 ? 49152 : 81920) / per;
  if (L > 16) L = 16;
  if (pow2(N) && L * N > 16LL * kFftThreads) L = 16LL * kFftThreads / N;
  if (L < 1) L = 1;
  while (L & (L - 1)) L &= L - 1;  // a power of two: shifts in the index arithmetic
  return (int)L;
}

}  // namespace

extern "C" long long pb_pressure_workspace_bytes(const pb_dims* dims) {
  if (pb_check_dims(dims)) return -1;
  return playout(dims).total;
}

// PressureFFTParallel.initialize (:27-62): the modified wave numbers
// (compute_modified_wave_numbers, :64-98) are evaluated on the host with the
// C library cos, as the reference does, so they match it bit for bit; the
// FFT twiddles exp(-2 pi i m/N) are evaluated in long double and rounded.
extern "C" int pb_pressure_init(const pb_dims* dims, void* workspace, long long workspace_bytes) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  const PLayout L = playout(dims);
  if (!workspace || workspace_bytes < L.total) return PB_ERR_WORKSPACE;
  if (reinterpret_cast<uintptr_t>(workspace) & 255) return PB_ERR_WORKSPACE;
  const double pi = 3.141592653589793;
  char* base = static_cast<char*>(workspace);
  for (int dim = 0; dim < 2; ++dim) {
    const long n = dims->n[dim];
    std::vector<double> k2(n);
    std::vector<double2> tw(n);
    for (long ii = 0; ii < n; ++ii) {
      const long i = dims->indx_lo[dim] + ii;
      double xi;
      if ((double)i <= (double)n / 2.0) xi = (double)i;
      else xi = (double)(i - n);
      k2[ii] = (2.0 * cos((2.0 * pi / (double)n) * xi) - 2.0) / dims->dx[dim] / dims->dx[dim];
      const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)ii / (long double)n;
      tw[ii] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    if (dims->indx_lo[dim] == 0) k2[0] = 0.0;
    PB_CUDA_TRY(cudaMemcpy(base + (dim == 0 ? L.kx2 : L.ky2), k2.data(), n * sizeof(double),
                           cudaMemcpyHostToDevice));
    PB_CUDA_TRY(cudaMemcpy(base + (dim == 0 ? L.twx : L.twy), tw.data(), n * sizeof(double2),
                           cudaMemcpyHostToDevice));
    std::vector<float2> twf(n);
    for (long ii = 0; ii < n; ++ii) twf[ii] = make_float2((float)tw[ii].x, (float)tw[ii].y);
    PB_CUDA_TRY(cudaMemcpy(base + (dim == 0 ? L.twxf : L.twyf), twf.data(), n * sizeof(float2),
                           cudaMemcpyHostToDevice));
  }
  return PB_OK;
}

// log2 of a length that has compile-time FFT kernels (128 ... 1024), else 0
int ct_lg(long long n) {
  if (!pow2(n) || n < 128 || n > 1024) return 0;
  int lg = 0;
  while ((1LL << lg) < n) ++lg;
  return lg;
}

template <class C, int SRC, int LG>
static int launch_x_fwd_src(const Geo& g, PArgs& a, dim3 grid, size_t sm, int KC, cudaStream_t st) {
  if (sm > 48 * 1024)
    PB_CUDA_TRY(cudaFuncSetAttribute(fft_x_fwd<C, SRC, LG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  fft_x_fwd<C, SRC, LG><<<grid, kFftThreads, sm, st>>>(g, a, KC);
  return PB_OK;
}

template <class C, int LG>
static int launch_x_fwd(const Geo& g, PArgs& a, int src, dim3 grid, size_t sm, int KC, cudaStream_t st) {
  if (src == kSrcDense) return launch_x_fwd_src<C, kSrcDense, LG>(g, a, grid, sm, KC, st);
  if constexpr (sizeof(C) == 8) {  // the refinement residual exists in the precision form only
    if (src == kSrcResidual) return launch_x_fwd_src<C, kSrcResidual, LG>(g, a, grid, sm, KC, st);
  }
  return launch_x_fwd_src<C, kSrcDivergence, LG>(g, a, grid, sm, KC, st);
}

template <class C, int DST, int LG>
static int launch_x_inv_dst(const Geo& g, PArgs& a, dim3 grid, size_t sm, int KC, cudaStream_t st) {
  if (sm > 48 * 1024)
    PB_CUDA_TRY(cudaFuncSetAttribute(fft_x_inv<C, DST, LG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  fft_x_inv<C, DST, LG><<<grid, kFftThreads, sm, st>>>(g, a, KC);
  return PB_OK;
}

template <class C, int LG>
static int launch_x_inv(const Geo& g, PArgs& a, int dst, dim3 grid, size_t sm, int KC, cudaStream_t st) {
  if (dst == kDstDense) return launch_x_inv_dst<C, kDstDense, LG>(g, a, grid, sm, KC, st);
  if constexpr (sizeof(C) == 8) {
    if (dst == kDstAccumulate) return launch_x_inv_dst<C, kDstAccumulate, LG>(g, a, grid, sm, KC, st);
  }
  return launch_x_inv_dst<C, kDstWrite, LG>(g, a, grid, sm, KC, st);
}

template <class C, int LG>
static int launch_y(const Geo& g, PArgs& a, bool inverse, dim3 grid, size_t sm, int IC, cudaStream_t st) {
  if (sm > 48 * 1024) {
    PB_CUDA_TRY(cudaFuncSetAttribute(fft_y<C, false, LG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    PB_CUDA_TRY(cudaFuncSetAttribute(fft_y<C, true, LG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  }
  if (inverse)
    fft_y<C, true, LG><<<grid, kFftThreads, sm, st>>>(g, a, IC);
  else
    fft_y<C, false, LG><<<grid, kFftThreads, sm, st>>>(g, a, IC);
  return PB_OK;
}

// Dispatch on a length's compile-time instantiation (LG = 0: run-time length).
#define PB_FFT_DISPATCH(lg, call)         \
  switch (lg) {                           \
    case 7: { constexpr int L_ = 7; call; } break;   \
    case 8: { constexpr int L_ = 8; call; } break;   \
    case 9: { constexpr int L_ = 9; call; } break;   \
    case 10: { constexpr int L_ = 10; call; } break; \
    default: { constexpr int L_ = 0; call; } break;  \
  }

// The spectral solve in phases, so that a sharded solve can exchange data
// between them: (1) forward x-FFT (from src) and forward y-FFT of every level
// of the grid; (2) the Thomas solve of every (kx, ky) column; (3) inverse
// y-FFT and inverse x-FFT (to dst).
struct FftShape {
  long long Nx, Ny, nz, Nh;
  int LC, KC, IC, lgx, lgy;
  size_t smx, smy;
  dim3 gx, gy;
};

template <class C>
static int fft_shape(const Geo& g, FftShape& f) {
  f.Nx = g.n0 - 2 * g.gw;
  f.Ny = g.n1 - 2 * g.gw;
  f.nz = g.n2 - 2 * g.gw;
  f.Nh = f.Nx / 2 + 1;  // stored x-modes
  f.LC = lines_for(f.Nx, sizeof(C));  // complex lines per x-FFT block
  f.KC = 2 * f.LC;                    // levels per x-FFT block (two per line)
  f.smx = fft_smem(f.Nx, f.LC, sizeof(C));
  f.IC = lines_for(f.Ny, sizeof(C));
  f.smy = fft_smem(f.Ny, f.IC, sizeof(C));
  f.lgx = ct_lg(f.Nx);
  f.lgy = ct_lg(f.Ny);
  if ((f.lgx && f.LC != ct_lines(f.lgx)) || (f.lgy && f.IC != ct_lines(f.lgy))) return PB_ERR_UNSUPPORTED;
  f.gx = dim3((unsigned)f.Ny, ceil_div(f.nz, f.KC));
  f.gy = dim3(ceil_div(f.Nh, f.IC), (unsigned)f.nz);
  return PB_OK;
}

template <class C>
static int fft_forward(const Geo& g, PArgs& a, int src, cudaStream_t st) {
  FftShape f;
  int rc = fft_shape<C>(g, f);
  if (rc) return rc;
  PB_FFT_DISPATCH(f.lgx, rc = (launch_x_fwd<C, L_>(g, a, src, f.gx, f.smx, f.KC, st)));
  if (rc) return rc;
  pb_note_launch();
  PB_LAUNCH_CHECK();
  PB_FFT_DISPATCH(f.lgy, rc = (launch_y<C, L_>(g, a, false, f.gy, f.smy, f.IC, st)));
  if (rc) return rc;
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

template <class C>
static int fft_columns(const Geo& g, PArgs& a, cudaStream_t st) {
  const long long Nh = (g.n0 - 2 * g.gw) / 2 + 1, Ny = g.n1 - 2 * g.gw;
  // one thread per column; on grids with fewer columns than 256 per SM the
  // blocks shrink (to a multiple of 32 threads) so that every SM gets some
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long per_sm = (Nh * Ny + sms - 1) / sms;
  const int threads = per_sm >= 256 ? 256 : (int)((per_sm + 31) / 32 * 32);
  tdma_kernel<C><<<ceil_div(Nh * Ny, threads), threads, 0, st>>>(g, a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

template <class C>
static int fft_inverse(const Geo& g, PArgs& a, int dst, cudaStream_t st) {
  FftShape f;
  int rc = fft_shape<C>(g, f);
  if (rc) return rc;
  PB_FFT_DISPATCH(f.lgy, rc = (launch_y<C, L_>(g, a, true, f.gy, f.smy, f.IC, st)));
  if (rc) return rc;
  pb_note_launch();
  PB_LAUNCH_CHECK();
  PB_FFT_DISPATCH(f.lgx, rc = (launch_x_inv<C, L_>(g, a, dst, f.gx, f.smx, f.KC, st)));
  if (rc) return rc;
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

template <class C>
static int fft_solve(const Geo& g, PArgs& a, bool resid, bool acc, cudaStream_t st) {
  int rc;
  if ((rc = fft_forward<C>(g, a, resid ? kSrcResidual : kSrcDivergence, st))) return rc;
  if ((rc = fft_columns<C>(g, a, st))) return rc;
  return fft_inverse<C>(g, a, acc ? kDstAccumulate : kDstWrite, st);
}
#undef PB_FFT_DISPATCH

static int pressure_solve_impl(const pb_dims* dims, const double* rho0, const double* rho0_half,
                               const double* alpha0, const double* alpha0_half, double* u, double* v, double* w,
                               double* divergence, double* dynamic_pressure, char* base, int precision,
                               int refine_sweeps, cudaStream_t st) {
  const Geo g = make_geo(dims);
  const PLayout L = playout(dims);
  PArgs a{};
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.alpha0 = alpha0;
  a.alpha0_half = alpha0_half;
  a.u = u;
  a.v = v;
  a.w = w;
  a.div = divergence;
  a.p = dynamic_pressure;
  a.partial = reinterpret_cast<double*>(base + L.partial);
  a.mean = reinterpret_cast<double*>(base + L.mean);
  a.twx = reinterpret_cast<const double2*>(base + L.twx);
  a.twy = reinterpret_cast<const double2*>(base + L.twy);
  a.twxf = reinterpret_cast<const float2*>(base + L.twxf);
  a.twyf = reinterpret_cast<const float2*>(base + L.twyf);
  a.kx2 = reinterpret_cast<const double*>(base + L.kx2);
  a.ky2 = reinterpret_cast<const double*>(base + L.ky2);
  a.spec = base + L.spec;
  a.scr = reinterpret_cast<double*>(base + L.scr);
  const long long Nx = dims->n[0], Ny = dims->n[1], nz = dims->n[2];
  const long long nghost = g.npg - Nx * Ny * nz;

  if (precision == PB_FP64) {  // the reference's summation order
    const size_t sm = 2 * (size_t)kSerialTile * kSerialLd * sizeof(double);
    PB_CUDA_TRY(cudaFuncSetAttribute(hmean_serial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    hmean_serial<<<ceil_div(g.n2, 32), kSerialWarps * 32, sm, st>>>(g, w, a.mean, 1.0 / (double)(Ny * Nx));
    pb_note_launch();
  } else {  // precision form: a deterministic parallel sum
    const int kpad = (int)((g.n2 + 31) / 32 * 32);
    hmean_partial<<<kPartials, kpad < 1024 ? kpad : 1024, 0, st>>>(g, w, a.partial);
    pb_note_launch();
    hmean_final<<<(unsigned)g.n2, 256, 0, st>>>(g, a.partial, a.mean, kPartials, 1.0 / (double)(Ny * Nx));
    pb_note_launch();
  }
  if (nghost > 0) {
    zero_ghosts<<<stream_blocks(nghost), 256, 0, st>>>(g, divergence, nghost);
    pb_note_launch();
  }
  PB_LAUNCH_CHECK();

  int rc;
  if (precision == PB_FP64) {
    if ((rc = fft_solve<double2>(g, a, false, false, st))) return rc;
  } else {
    // precision form: FP32 FFTs, FP64 tridiagonal solve, then refinement
    // sweeps p += solve(div - A p) on the FP64 residual
    if ((rc = fft_solve<float2>(g, a, false, false, st))) return rc;
    for (int s = 0; s < refine_sweeps; ++s) {
      if (nghost > 0) {
        ghost_sym<<<stream_blocks(nghost), 256, 0, st>>>(g, dynamic_pressure, nghost);
        pb_note_launch();
      }
      if ((rc = fft_solve<float2>(g, a, true, true, st))) return rc;
    }
  }
  if (nghost > 0) {
    ghost_sym<<<stream_blocks(nghost), 256, 0, st>>>(g, dynamic_pressure, nghost);
    pb_note_launch();
  }
  correction<<<stream_blocks(g.npg), 256, 0, st>>>(g, dynamic_pressure, u, v, w, a.mean);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_pressure_solve(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                 const double* alpha0, const double* alpha0_half, double* u, double* v, double* w,
                                 double* divergence, double* dynamic_pressure, void* workspace,
                                 long long workspace_bytes, int precision, int refine_sweeps, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w || !divergence || !dynamic_pressure)
    return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  if (refine_sweeps < 0 || refine_sweeps > 8) return PB_ERR_ARG;
  const PLayout L = playout(dims);
  if (!workspace || workspace_bytes < L.total) return PB_ERR_WORKSPACE;
  if (reinterpret_cast<uintptr_t>(workspace) & 255) return PB_ERR_WORKSPACE;
  if (!fft_sizes_ok(dims)) return PB_ERR_UNSUPPORTED;
  return pressure_solve_impl(dims, rho0, rho0_half, alpha0, alpha0_half, u, v, w, divergence, dynamic_pressure,
                             static_cast<char*>(workspace), precision, refine_sweeps, as_stream(stream));
}
