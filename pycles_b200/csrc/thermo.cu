// Saturation-adjustment and dry thermodynamics: the FP64 plain form and the
// C entry points (translation unit compiled with -fmad=false).
//
// With -fmad=false and correctly rounded exp/log (crmath.cuh) the
// temperature follows the reference's separately rounded C arithmetic bit
// for bit (see crmath.cuh for why that matters here).  The precision form's
// instantiations live in thermo_fast.cu.
#include "pb_common.cuh"
#include "crmath.cuh"
#include "thermo_kernels.cuh"

namespace {
struct ExactMath {
  static constexpr bool exact = true;  // keep the reference's operations and order
  static __device__ __forceinline__ double exp(double x) { return crm::exp(x); }
  static __device__ __forceinline__ double log(double x) { return crm::log(x); }
};
}  // namespace

namespace thermo_k {

void column_launch_shape(long long n2, int per_col_arrays, dim3* blk, size_t* smem) {
  const int kpad = (int)((n2 + 31) / 32 * 32);
  int cols = 256 / kpad;
  if (cols < 1) cols = 1;
  *blk = dim3(kpad, cols);
  *smem = (size_t)per_col_arrays * kpad * cols * sizeof(double);
}

cudaError_t launch_sa_exact(const Geo& geo, const SaArgs& a, cudaStream_t st) {
  return thermo_kk::launch_sa<ExactMath, false>(geo, a, st);
}

cudaError_t launch_dry_exact(const Geo& geo, const DryArgs& a, cudaStream_t st) {
  return thermo_kk::launch_dry<ExactMath>(geo, a, st);
}

}  // namespace thermo_k

using namespace thermo_k;

// mlp.cu: refresh of the seed's per-cell network output (cells with ql > 0)
cudaError_t pb_mlp_seed_refresh(const pb_mlp* mlp, const Geo& g, const double* p0, const double* s,
                                const double* qt, const double* ql, cudaStream_t st);

extern "C" int pb_thermo_sa(const pb_dims* dims, const double* p0_half, const double* alpha0_half,
                            const pb_table* table, const double* s, double* qt, double* T, double* qv,
                            double* ql, double* qi, double* alpha, double* buoyancy, double* theta_rho,
                            double* bvf, double* thetali, double* w_tend, int clip_qt, const pb_mlp* mlp,
                            long long* secant_iters, int max_iter, int precision, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!p0_half || !alpha0_half || !table || !table->y || table->n < 2 || !(table->dx > 0.0)) return PB_ERR_ARG;
  if (!s || !qt || !T || !qv || !ql || !qi || !alpha || !buoyancy || !theta_rho || !bvf || !thetali || !w_tend)
    return PB_ERR_ARG;
  if (max_iter < 1) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  if (mlp && (precision != PB_FP32 || !mlp->w1 || !mlp->b1 || !mlp->w2 || !mlp->b2 || !mlp->w3 || !mlp->b3 ||
              !mlp->seed_y))
    return PB_ERR_ARG;
  if (dims->nlg[2] > 1024) return PB_ERR_UNSUPPORTED;
  const Geo geo = make_geo(dims);
  SaArgs a{};
  a.p0 = p0_half;
  a.alpha0 = alpha0_half;
  a.LT = *table;
  a.s = s;
  a.qt = qt;
  a.T = T;
  a.qv = qv;
  a.ql = ql;
  a.qi = qi;
  a.alpha = alpha;
  a.buoy = buoyancy;
  a.theta_rho = theta_rho;
  a.bvf = bvf;
  a.thetali = thetali;
  a.wt = w_tend;
  a.stats = reinterpret_cast<unsigned long long*>(secant_iters);
  a.err = pb_error_word_ptr();
  if (!a.err) return PB_ERR_CUDA;
  a.clip = clip_qt;
  a.max_iter = max_iter;
  const cudaStream_t st = as_stream(stream);
  if (mlp) {
    // the network's output for the cells saturated at the previous call,
    // at the current (p0, s, qt); the kernel below starts their secant there
    a.net.y = mlp->seed_y;
    a.net.out_mean = mlp->out_mean;
    a.net.out_scale = mlp->out_scale;
    if (mlp->seed_refresh && pb_mlp_seed_refresh(mlp, geo, p0_half, s, qt, ql, st) != cudaSuccess)
      return PB_ERR_CUDA;
  }
  const cudaError_t e = precision == PB_FP64 ? launch_sa_exact(geo, a, st) : launch_sa_fast(geo, a, mlp != nullptr, st);
  return e == cudaSuccess ? PB_OK : PB_ERR_CUDA;
}

extern "C" int pb_thermo_dry(const pb_dims* dims, const double* p0_half, const double* alpha0_half,
                             const double* s, double* T, double* alpha, double* buoyancy, double* theta,
                             double* bvf, double* w_tend, int precision, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!p0_half || !alpha0_half || !s || !T || !alpha || !buoyancy || !theta || !bvf || !w_tend) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  if (dims->nlg[2] > 1024) return PB_ERR_UNSUPPORTED;
  const Geo geo = make_geo(dims);
  DryArgs a{p0_half, alpha0_half, s, T, alpha, buoyancy, theta, bvf, w_tend};
  const cudaStream_t st = as_stream(stream);
  const cudaError_t e = precision == PB_FP64 ? launch_dry_exact(geo, a, st) : launch_dry_fast(geo, a, st);
  return e == cudaSuccess ? PB_OK : PB_ERR_CUDA;
}

// ---- pointwise saturation adjustment ----------------------------------------
// ThermodynamicsSA.eos (ThermodynamicsSA.pyx:169-174): eos_c for a list of
// (p0, s, qt) points with the FP64 plain-form arithmetic.  Used to generate
// the learned seed's training pairs (T and the secant's first point T_1) and
// to count secant iterations with and without a seed.
namespace {

struct EosPointArgs {
  pb_table LT;
  const double* p0;
  const double* s;
  const double* qt;
  const double* seed;  // nullable: second secant point per point
  double* T;
  double* ql;
  double* qi;
  double* T_first;     // nullable: the secant's first point T_1
  int* iters;          // nullable: secant iterations per point (0 = unsaturated)
  unsigned int* err;
  long long n;
  int max_iter;
};

__global__ void eos_points_kernel(EosPointArgs a) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const double p0 = a.p0[i], s = a.s[i], qt = a.qt[i];
    const thermo_f::EosStart st = thermo_f::eos_start<ExactMath>(a.LT, p0, s, qt, a.err);
    const thermo_f::EosOut e = thermo_f::eos_finish<ExactMath>(a.LT, st, p0, s, qt, a.max_iter, a.seed != nullptr,
                                                               a.seed ? a.seed[i] : 0.0, a.err);
    a.T[i] = e.T;
    if (a.ql) a.ql[i] = e.ql;
    if (a.qi) a.qi[i] = e.qi;
    if (a.T_first) a.T_first[i] = st.T_1;
    if (a.iters) a.iters[i] = e.iters;
  }
}

}  // namespace

extern "C" int pb_eos_sa(const pb_table* table, const double* p0, const double* s, const double* qt,
                         const double* seed, double* T, double* ql, double* qi, double* T_first, int* iters,
                         long long n, int max_iter, void* stream) {
  if (!table || !table->y || table->n < 2 || !(table->dx > 0.0)) return PB_ERR_ARG;
  if (!p0 || !s || !qt || !T || n < 0 || max_iter < 1) return PB_ERR_ARG;
  if (n == 0) return PB_OK;
  EosPointArgs a;
  a.LT = *table;
  a.p0 = p0;
  a.s = s;
  a.qt = qt;
  a.seed = seed;
  a.T = T;
  a.ql = ql;
  a.qi = qi;
  a.T_first = T_first;
  a.iters = iters;
  a.err = pb_error_word_ptr();
  if (!a.err) return PB_ERR_CUDA;
  a.n = n;
  a.max_iter = max_iter;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sms * 16) blocks = (long long)sms * 16;
  eos_points_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
