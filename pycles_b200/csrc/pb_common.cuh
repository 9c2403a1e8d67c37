// Shared definitions for the B200 hot-path kernels.
//
// Layout contract (identical to the reference, Csrc/grid.h and
// PrognosticVariables.pyx:78-79): every field is a flat ghosted array
// [i][j][k] with k contiguous, istride = nlg1*nlg2, jstride = nlg2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/pycles_b200.h"

// Physical constants as generate_parameters.py:19-41 writes them
// (eps_v = Rd/Rv, eps_vi = 1/eps_v, kappa = Rd/cpd, shortest round-trip
// decimal of the Python double).
namespace pbc {
constexpr double g = 9.80665;
constexpr double Rd = 287.1;
constexpr double Rv = 461.5;
constexpr double eps_v = 0.6221018418201517;
constexpr double eps_vi = 1.6074538488331591;
constexpr double cpd = 1004.0;
constexpr double cpv = 1859.0;
constexpr double kappa = 0.2859561752988048;
constexpr double T_tilde = 298.15;
constexpr double p_tilde = 100000.0;
constexpr double sd_tilde = 6864.8;
constexpr double sv_tilde = 10513.6;
}  // namespace pbc

// Error word bits (pb_get_error); kernels OR them in, the host reads once
// per step.
#define PB_ERR_TABLE_RANGE 0x1u   // lookup argument outside the pv* table
#define PB_ERR_SECANT_CAP 0x2u    // saturation-adjustment secant hit its cap
#define PB_ERR_NONFINITE 0x4u     // non-finite temperature produced

// Device address of this device's error word (defined in timestep.cu); the
// library has two translation units, so kernels receive it as an argument.
unsigned int* pb_error_word_ptr();

__device__ __forceinline__ void pb_flag_at(unsigned int* word, unsigned int bit) { atomicOr(word, bit); }

// Separately rounded IEEE operations.  The compiler contracts a*b+c into an
// FMA; where a result is formed by cancellation (the divergence of a nearly
// solenoidal field, alpha - alpha0, near-singular tridiagonal rows) that one
// rounding difference shows up at 1e-12 relative, so these spots use the
// reference's separately rounded sequence.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

struct Geo {
  long long n0, n1, n2;     // nlg
  long long is, js;         // strides in elements
  long long gw;
  long long npg;
  double dxi0, dxi1, dxi2;
  double dx2;
};

// Ghost cell number t -> (i, j, k).  The ghost set is ordered as: the x
// slabs (i < gw or i >= n0-gw, all j, k), then the y slabs of the interior
// x range, then the z slabs of the interior columns.  Unsigned 32-bit
// division when the field has fewer than 2^31 cells (a few instructions
// instead of a 64-bit division sequence), 64-bit otherwise.
template <class I>
__device__ __forceinline__ void ghost_decode_t(I t, I gw, I n0, I n1, I n2, I& i, I& j, I& k) {
  const I nl0 = n0 - 2 * gw, nl1 = n1 - 2 * gw;
  const I A = 2 * gw * n1 * n2;
  const I B = nl0 * 2 * gw * n2;
  if (t < A) {
    const I gi = t / (n1 * n2);
    const I r = t - gi * (n1 * n2);
    i = gi < gw ? gi : n0 - 2 * gw + gi;
    j = r / n2;
    k = r - j * n2;
  } else if (t < A + B) {
    const I u = t - A;
    const I q = u / (2 * gw * n2);
    const I r = u - q * (2 * gw * n2);
    i = gw + q;
    const I gj = r / n2;
    j = gj < gw ? gj : n1 - 2 * gw + gj;
    k = r - gj * n2;
  } else {
    const I u = t - A - B;
    const I q = u / (nl1 * 2 * gw);
    const I r = u - q * (nl1 * 2 * gw);
    i = gw + q;
    const I rj = r / (2 * gw);
    j = gw + rj;
    const I gk = r - rj * (2 * gw);
    k = gk < gw ? gk : n2 - 2 * gw + gk;
  }
}

__device__ __forceinline__ void ghost_decode(const Geo& g, long long t, long long& i, long long& j, long long& k) {
  if (g.npg < (1LL << 31)) {
    unsigned int i32, j32, k32;
    ghost_decode_t<unsigned int>((unsigned int)t, (unsigned int)g.gw, (unsigned int)g.n0, (unsigned int)g.n1,
                                 (unsigned int)g.n2, i32, j32, k32);
    i = i32;
    j = j32;
    k = k32;
  } else {
    ghost_decode_t<long long>(t, g.gw, g.n0, g.n1, g.n2, i, j, k);
  }
}

static inline Geo make_geo(const pb_dims* d) {
  Geo g;
  g.n0 = d->nlg[0];
  g.n1 = d->nlg[1];
  g.n2 = d->nlg[2];
  g.js = g.n2;
  g.is = g.n1 * g.n2;
  g.gw = d->gw;
  g.npg = g.n0 * g.n1 * g.n2;
  g.dxi0 = d->dxi[0];
  g.dxi1 = d->dxi[1];
  g.dxi2 = d->dxi[2];
  g.dx2 = d->dx[2];
  return g;
}

// Validates the geometry fields every entry point relies on.
int pb_check_dims(const pb_dims* d);

#define PB_CUDA_TRY(expr)                          \
  do {                                             \
    cudaError_t _e = (expr);                       \
    if (_e != cudaSuccess) return PB_ERR_CUDA;     \
  } while (0)

#define PB_LAUNCH_CHECK()                          \
  do {                                             \
    cudaError_t _e = cudaGetLastError();           \
    if (_e != cudaSuccess) return PB_ERR_CUDA;     \
  } while (0)

// Host-side count of kernels this library has launched (pb_launch_count).
inline std::atomic<long long>& pb_launch_counter() {
  static std::atomic<long long> c{0};
  return c;
}
static inline void pb_note_launch() { pb_launch_counter().fetch_add(1, std::memory_order_relaxed); }

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

static inline unsigned int ceil_div(long long a, long long b) { return (unsigned int)((a + b - 1) / b); }
