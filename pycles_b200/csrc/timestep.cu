// SSP-RK3 stage update and ghost-cell fills.
#include <string.h>

#include <mutex>

#include "pb_common.cuh"

__device__ unsigned int pb_device_error = 0u;

unsigned int* pb_error_word_ptr() {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, pb_device_error) != cudaSuccess) return nullptr;
    addr[dev] = p;
  }
  return static_cast<unsigned int*>(addr[dev]);
}

namespace {

// TimeStepping.update_third (TimeStepping.pyx:131-151), streaming over
// nv*npg values (ghosts included), two values per thread iteration.
// The result goes to vout (the values array itself, or a second buffer).
template <int STAGE>
__global__ void __launch_bounds__(256) rk3_kernel(const double* v, double* vout, double* __restrict__ t,
                                                   double* __restrict__ c, long long n, double dt) {
  const long long n2 = n >> 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const double2* v2 = reinterpret_cast<const double2*>(v);
  double2* o2 = reinterpret_cast<double2*>(vout);
  double2* t2 = reinterpret_cast<double2*>(t);
  double2* c2 = reinterpret_cast<double2*>(c);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
    double2 vv = v2[i];
    const double2 tt = t2[i];
    // separately rounded, as the reference's C loop (the kernel is
    // bandwidth bound, so this costs nothing)
    if (STAGE == 0) {
      c2[i] = vv;
      vv.x = add_rn(vv.x, mul_rn(tt.x, dt));
      vv.y = add_rn(vv.y, mul_rn(tt.y, dt));
    } else {
      const double2 cc = c2[i];
      const double a = (STAGE == 1) ? 0.75 : (1.0 / 3.0);
      const double b = (STAGE == 1) ? 0.25 : (2.0 / 3.0);
      vv.x = add_rn(mul_rn(a, cc.x), mul_rn(b, add_rn(vv.x, mul_rn(tt.x, dt))));
      vv.y = add_rn(mul_rn(a, cc.y), mul_rn(b, add_rn(vv.y, mul_rn(tt.y, dt))));
    }
    o2[i] = vv;
    t2[i] = make_double2(0.0, 0.0);
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const long long i = n - 1;
    const double vi = v[i];
    if (STAGE == 0) {
      c[i] = vi;
      vout[i] = add_rn(vi, mul_rn(t[i], dt));
    } else if (STAGE == 1) {
      vout[i] = add_rn(mul_rn(0.75, c[i]), mul_rn(0.25, add_rn(vi, mul_rn(t[i], dt))));
    } else {
      vout[i] = add_rn(mul_rn(1.0 / 3.0, c[i]), mul_rn(2.0 / 3.0, add_rn(vi, mul_rn(t[i], dt))));
    }
    t[i] = 0.0;
  }
}

constexpr int kMaxBcVars = 16;
struct BcArgs {
  double factor[kMaxBcVars];
  int nv;
};

// Ghost fill of nv fields.  On one rank the reference's sequence (x
// exchange over all j,k; y exchange over all i,k; z set_bcs over all i,j;
// PrognosticVariables.pyx:199-233) gives every ghost cell a value derived
// from exactly one interior cell:  periodic images i', j' and, for z
// ghosts, the mirror level k' of set_bcs (Csrc/prognostic_variables.h:
// 205-270) with its factor.  Reads touch only interior cells and writes
// only ghost cells, so one pass over the ghost cells reproduces it.
__global__ void __launch_bounds__(256) ghost_fill_kernel(Geo g, double* __restrict__ vals, BcArgs bc,
                                                         long long nghost) {
  const long long gw = g.gw;
  const long long n0 = g.n0, n1 = g.n1, n2 = g.n2;
  const long long nl0 = n0 - 2 * gw, nl1 = n1 - 2 * gw, nl2 = n2 - 2 * gw;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nghost; t += stride) {
    long long i, j, k;
    ghost_decode(g, t, i, j, k);
    const long long is_ = (i < gw) ? i + nl0 : ((i >= n0 - gw) ? i - nl0 : i);
    const long long js_ = (j < gw) ? j + nl1 : ((j >= n1 - gw) ? j - nl1 : j);
    const long long dst = i * g.is + j * g.js + k;
    const long long colsrc = is_ * g.is + js_ * g.js;
    // reads touch interior cells only and writes ghost cells only, so the
    // variables' loads of a batch are all issued before its stores; each
    // variable's value is mult * f[src], or exactly 0 on the first
    // antisymmetric level (set_bcs with factor != 1, 2)
    constexpr int kB = 4;
    for (int v0 = 0; v0 < bc.nv; v0 += kB) {
      double out[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const int v = v0 + b;
        out[b] = 0.0;
        if (v >= bc.nv) continue;
        const double fac = bc.factor[v];
        long long src = colsrc + k;
        double mult = 1.0;
        bool zero = false;
        if (k >= n2 - gw) {  // top, set_bcs s = -1
          const long long tt = k - (n2 - gw);
          if (fac == 1.0) src = colsrc + (n2 - gw - 1 - tt);
          else if (fac == 2.0) src = colsrc + (n2 - gw - 1);
          else { src = colsrc + (n2 - gw - tt); mult = fac; zero = tt == 0; }
        } else if (k < gw) {  // bottom, set_bcs s = +1
          const long long tt = gw - 1 - k;
          if (fac == 1.0) src = colsrc + (gw + tt);
          else if (fac == 2.0) src = colsrc + gw;
          else { src = colsrc + (gw - 1 + tt); mult = fac; zero = tt == 0; }
        }
        if (!zero) out[b] = mult * vals[(long long)v * g.npg + src];
      }
#pragma unroll
      for (int b = 0; b < kB; ++b)
        if (v0 + b < bc.nv) vals[(long long)(v0 + b) * g.npg + dst] = out[b];
    }
    (void)nl2;
  }
}

}  // namespace

int pb_check_dims(const pb_dims* d) {
  if (!d) return PB_ERR_ARG;
  if (d->gw < 1) return PB_ERR_ARG;
  for (int i = 0; i < 3; ++i) {
    if (d->n[i] < 1 || d->nlg[i] != d->n[i] + 2 * d->gw || d->nl[i] != d->n[i]) return PB_ERR_ARG;
    if (!(d->dx[i] > 0.0)) return PB_ERR_ARG;
  }
  if (d->npg != d->nlg[0] * d->nlg[1] * d->nlg[2]) return PB_ERR_ARG;
  if (d->npl != d->n[0] * d->n[1] * d->n[2]) return PB_ERR_ARG;
  // ghost regions must fit inside the domain for the periodic images
  for (int i = 0; i < 3; ++i)
    if (d->n[i] < d->gw) return PB_ERR_UNSUPPORTED;
  return PB_OK;
}

static int grid_blocks(long long work, int threads) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long b = (work + threads - 1) / threads;
  const long long cap = (long long)sms * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

static int rk3_launch(const double* values, double* out, double* tendencies, double* value_copy, long long n,
                      double dt, int rk_step, void* stream) {
  if (!values || !out || !tendencies || !value_copy || n < 0) return PB_ERR_ARG;
  if (rk_step < 0 || rk_step > 2) return PB_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(values) | reinterpret_cast<uintptr_t>(out) |
       reinterpret_cast<uintptr_t>(tendencies) | reinterpret_cast<uintptr_t>(value_copy)) & 15)
    return PB_ERR_ARG;
  if (n == 0) return PB_OK;
  cudaStream_t st = as_stream(stream);
  const int blocks = grid_blocks((n + 1) / 2, 256);
  if (rk_step == 0)
    rk3_kernel<0><<<blocks, 256, 0, st>>>(values, out, tendencies, value_copy, n, dt);
  else if (rk_step == 1)
    rk3_kernel<1><<<blocks, 256, 0, st>>>(values, out, tendencies, value_copy, n, dt);
  else
    rk3_kernel<2><<<blocks, 256, 0, st>>>(values, out, tendencies, value_copy, n, dt);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_rk3_update(double* values, double* tendencies, double* value_copy, long long n, double dt,
                             int rk_step, void* stream) {
  return rk3_launch(values, values, tendencies, value_copy, n, dt, rk_step, stream);
}

extern "C" int pb_rk3_update_to(const double* values, double* values_out, double* tendencies,
                                double* value_copy, long long n, double dt, int rk_step, void* stream) {
  return rk3_launch(values, values_out, tendencies, value_copy, n, dt, rk_step, stream);
}

extern "C" int pb_update_all_bcs(const pb_dims* dims, double* values, const double* bc_factor, int nv,
                                 void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!values || !bc_factor || nv < 1) return PB_ERR_ARG;
  const Geo g = make_geo(dims);
  const long long npl = (long long)dims->n[0] * dims->n[1] * dims->n[2];
  const long long nghost = g.npg - npl;
  if (nghost == 0) return PB_OK;
  cudaStream_t st = as_stream(stream);
  for (int v0 = 0; v0 < nv; v0 += kMaxBcVars) {
    BcArgs a;
    memset(&a, 0, sizeof(a));
    a.nv = (nv - v0 < kMaxBcVars) ? nv - v0 : kMaxBcVars;
    for (int v = 0; v < a.nv; ++v) a.factor[v] = bc_factor[v0 + v];
    ghost_fill_kernel<<<grid_blocks(nghost, 256), 256, 0, st>>>(g, values + (long long)v0 * g.npg, a, nghost);
    pb_note_launch();
    PB_LAUNCH_CHECK();
  }
  return PB_OK;
}

extern "C" int pb_get_error(unsigned int* word) {
  if (!word) return PB_ERR_ARG;
  PB_CUDA_TRY(cudaMemcpyFromSymbol(word, pb_device_error, sizeof(unsigned int)));
  return PB_OK;
}

extern "C" int pb_clear_error(void* stream) {
  void* p = nullptr;
  PB_CUDA_TRY(cudaGetSymbolAddress(&p, pb_device_error));
  PB_CUDA_TRY(cudaMemsetAsync(p, 0, sizeof(unsigned int), as_stream(stream)));
  return PB_OK;
}

extern "C" const char* pb_status_string(int status) {
  switch (status) {
    case PB_OK: return "ok";
    case PB_ERR_ARG: return "invalid argument";
    case PB_ERR_CUDA: return "CUDA runtime error";
    case PB_ERR_UNSUPPORTED: return "unsupported configuration";
    case PB_ERR_WORKSPACE: return "workspace missing or too small";
    default: return "unknown status";
  }
}

extern "C" long long pb_launch_count(void) { return pb_launch_counter().load(std::memory_order_relaxed); }
