// Saturation-adjustment and dry thermodynamics (translation unit 2).
//
// One thread block owns whole (i,j) columns, one thread per level k, so the
// vertical neighbours that buoyancy_update_sa / bvf_sa need come from shared
// memory and every cell's state is computed exactly once.
//
// Compiled with -fmad=false and with correctly rounded exp/log (crmath.cuh):
// the temperature then follows the reference's separately rounded C
// arithmetic bit for bit (see crmath.cuh for why that matters here).
#include "pb_common.cuh"
#include "crmath.cuh"
#include "mlp.cuh"

namespace thermo_k {

using namespace pbc;

// ---- thermodynamic functions (Csrc/thermodynamic_functions.h, entropies.h)
__device__ __forceinline__ double pd_c(double p0, double qt, double qv) {
  return p0 * (1.0 - qt) / (1.0 - qt + eps_vi * qv);
}
__device__ __forceinline__ double pv_c(double p0, double qt, double qv) {
  return p0 * eps_vi * qv / (1.0 - qt + eps_vi * qv);
}
__device__ __forceinline__ double qv_star_c(double p0, double qt, double pv) {
  return eps_v * (1.0 - qt) * pv / (p0 - pv);
}
// alpha and buoyancy: buoyancy cancels ~3 digits of alpha, so both keep the
// reference's separately rounded operations.
__device__ __forceinline__ double alpha_c(double p0, double T, double qt, double qv) {
  return mul_rn((Rd * T) / p0, add_rn(sub_rn(1.0, qt), mul_rn(eps_vi, qv)));
}
__device__ __forceinline__ double buoyancy_c(double alpha0, double alpha) {
  return mul_rn(g, sub_rn(alpha, alpha0)) / alpha0;
}
__device__ __forceinline__ double cpm_c(double qt) { return (1.0 - qt) * cpd + qt * cpv; }
__device__ __forceinline__ double sd_c(double pd, double T) {
  return sd_tilde + cpd * crm::log(T / T_tilde) - Rd * crm::log(pd / p_tilde);
}
__device__ __forceinline__ double sv_c(double pv, double T) {
  return sv_tilde + cpv * crm::log(T / T_tilde) - Rv * crm::log(pv / p_tilde);
}
__device__ __forceinline__ double sc_c(double L, double T) { return -L / T; }
__device__ __forceinline__ double interp_2(double a, double b) { return 0.5 * (a + b); }

// latent_heat_variable with lambda_constant (Microphysics.pxd:65-75)
__device__ __forceinline__ double latent_heat(double T) {
  const double TC = T - 273.15;
  return (2500.8 - 2.36 * TC + 0.0016 * TC * TC - 0.00006 * TC * TC * TC) * 1000.0;
}

// lookup (Csrc/lookup.h:48-54) with a range check the reference lacks:
// out-of-table arguments flag PB_ERR_TABLE_RANGE and are clamped.
__device__ __forceinline__ double table_lookup(const pb_table& t, double x, unsigned int* err) {
  const double fi = floor((x - t.x_min) * t.dxi);
  long long indx;
  if (!(fi >= 0.0 && fi <= (double)(t.n - 2))) {
    pb_flag_at(err, PB_ERR_TABLE_RANGE);
    indx = (fi >= 0.0) ? t.n - 2 : 0;
  } else {
    indx = (long long)fi;
  }
  const double y1 = __ldg(t.y + indx);
  const double y2 = __ldg(t.y + indx + 1);
  const double x1 = t.x_min + t.dx * indx;
  return y1 + (x - x1) * (y2 - y1) * t.dxi;
}

// temperature_no_ql (Csrc/thermodynamics_sa.h:10-15)
__device__ __forceinline__ double temperature_no_ql(double pd, double pv, double s, double qt) {
  return T_tilde * crm::exp((s - (1.0 - qt) * (sd_tilde - Rd * crm::log(pd / p_tilde)) -
                             qt * (sv_tilde - Rv * crm::log(pv / p_tilde))) /
                            ((1.0 - qt) * cpd + qt * cpv));
}

struct EosOut {
  double T, qv, ql, qi;
  int iters;
  bool sat;
};

// eos_c (Csrc/thermodynamics_sa.h:17-66).  The secant loop is the
// reference's; it is capped at max_iter (the reference loops without a cap),
// reaching the cap sets PB_ERR_SECANT_CAP.  use_seed replaces the second
// secant point T_2 (:39) by a learned guess; the loop and its stopping test
// stay the reference's.
__device__ __forceinline__ EosOut eos_sa(const pb_table& LT, double p0, double s, double qt, int max_iter,
                                         bool use_seed, double seed, unsigned int* err) {
  EosOut o;
  o.qv = qt;
  o.ql = 0.0;
  o.qi = 0.0;
  o.iters = 0;
  const double pv_1 = pv_c(p0, qt, qt);
  const double pd_1 = p0 - pv_1;
  double T_1 = temperature_no_ql(pd_1, pv_1, s, qt);
  const double pv_star_1 = table_lookup(LT, T_1, err);
  const double qv_star_1 = qv_star_c(p0, qt, pv_star_1);
  if (qt <= qv_star_1) {
    o.T = T_1;
    o.sat = false;
    return o;
  }
  o.sat = true;
  const double sigma_1 = qt - qv_star_1;
  const double L_1 = latent_heat(T_1);
  const double s_1 = sd_c(pd_1, T_1) * (1.0 - qt) + sv_c(pv_1, T_1) * qt + sc_c(L_1, T_1) * sigma_1;
  double f_1 = s - s_1;
  double T_2 = T_1 + sigma_1 * L_1 / ((1.0 - qt) * cpd + qv_star_1 * cpv);
  if (use_seed) T_2 = seed;
  double delta_T;
  double qv_star_2, sigma_2;
  int it = 0;
  do {
    const double pv_star_2 = table_lookup(LT, T_2, err);
    qv_star_2 = qv_star_c(p0, qt, pv_star_2);
    const double pv_2 = pv_c(p0, qt, qv_star_2);
    const double pd_2 = p0 - pv_2;
    sigma_2 = qt - qv_star_2;
    const double L_2 = latent_heat(T_2);
    const double s_2 = sd_c(pd_2, T_2) * (1.0 - qt) + sv_c(pv_2, T_2) * qt + sc_c(L_2, T_2) * sigma_2;
    const double f_2 = s - s_2;
    const double T_n = T_2 - f_2 * (T_2 - T_1) / (f_2 - f_1);
    T_1 = T_2;
    T_2 = T_n;
    f_1 = f_2;
    delta_T = fabs(T_2 - T_1);
    ++it;
    if (it >= max_iter) {
      if (delta_T >= 1.0e-3 || sigma_2 < 0.0) pb_flag_at(err, PB_ERR_SECANT_CAP);
      break;
    }
  } while (delta_T >= 1.0e-3 || sigma_2 < 0.0);
  o.T = T_2;
  o.qv = qv_star_2;
  o.ql = 1.0 * sigma_2;           // lambda = 1
  o.qi = (1.0 - 1.0) * sigma_2;
  o.iters = it;
  return o;
}

struct SaArgs {
  const double* p0;          // RS.p0_half
  const double* alpha0;      // RS.alpha0_half
  pb_table LT;
  const double* s;
  double* qt;
  double* T;
  double* qv;
  double* ql;
  double* qi;
  double* alpha;
  double* buoy;
  double* theta_rho;
  double* bvf;
  double* thetali;
  double* wt;
  const double* seed;        // learned T_2 per cell (nullable)
  unsigned long long* stats; // {iterations, saturated cells} (nullable)
  unsigned int* err;         // device error word
  int clip;
  int max_iter;
};

// Shared-memory layout per column: T, qt, theta_rho, buoyancy.  Each block
// walks a uniform number of column groups (grid-stride), so the per-level
// constants (p0, alpha0, the Exner function) are evaluated once per thread.
__global__ void thermo_sa_kernel(Geo geo, SaArgs a, long long ncols) {
  extern __shared__ double sm[];
  const int kpad = blockDim.x;
  const int k = threadIdx.x;
  const long long n2 = geo.n2;
  double* sT = sm + (size_t)threadIdx.y * 4 * kpad;
  double* sQ = sT + kpad;
  double* sR = sQ + kpad;
  double* sB = sR + kpad;
  const bool kin = k < n2;
  const double p0 = kin ? a.p0[k] : 1.0;
  const double a0 = kin ? a.alpha0[k] : 1.0;
  const double exner = pow(p0 / p_tilde, kappa);
  const double dzi = 1.0 / geo.dx2;
  unsigned long long my_it = 0, my_sat = 0;
  for (long long cbase = (long long)blockIdx.x * blockDim.y; cbase < ncols; cbase += (long long)gridDim.x * blockDim.y) {
    const long long col = cbase + threadIdx.y;
    const bool active = (col < ncols) && kin;
    const long long idx = col * n2 + k;  // columns are contiguous: (i*n1 + j)*n2
    double qt = 0.0, qv = 0.0, T = 0.0;
    if (active) {
      qt = a.qt[idx];
      if (a.clip) {  // clip_qt (Csrc/thermodynamics_sa.h:213-219)
        qt = fmax(qt, 1e-11);
        a.qt[idx] = qt;
      }
      const double s = a.s[idx];
      const EosOut e = eos_sa(a.LT, p0, s, qt, a.max_iter, a.seed != nullptr, a.seed ? a.seed[idx] : 0.0, a.err);
      T = e.T;
      qv = e.qv;
      if (!isfinite(T)) pb_flag_at(a.err, PB_ERR_NONFINITE);
      my_it += (unsigned long long)e.iters;
      my_sat += e.sat ? 1ull : 0ull;
      a.T[idx] = T;
      a.qv[idx] = qv;
      a.ql[idx] = e.ql;
      a.qi[idx] = e.qi;
      const double al = alpha_c(p0, T, qt, qv);
      a.alpha[idx] = al;
      // thetali_update (:185-211) with thetali_c (thermodynamic_functions.h:15-18);
      // without condensate the exponential is exp(-0) = 1 exactly
      const double theta = T / exner;
      if (e.ql == 0.0 && e.qi == 0.0) {
        a.thetali[idx] = theta * 1.0;
      } else {
        const double Lv = latent_heat(T);
        a.thetali[idx] = theta * crm::exp(-Lv * (e.ql / (1.0 - qt) + e.qi / (1.0 - qt)) / (T * cpd));
      }
      // bvf_sa first loop (:147-157): theta_rho on k in [1, n2-1)
      double thr = 0.0;
      if (k >= 1 && k < n2 - 1) {
        thr = T * (1.0 - qt + eps_vi * qv) / exner;
        a.theta_rho[idx] = thr;
      }
      // buoyancy_update_sa first loop (:110-119): k in [0, n2-1)
      double b = 0.0;
      if (k < n2 - 1) {
        b = buoyancy_c(a0, al);
        a.buoy[idx] = b;
      }
      sT[k] = T;
      sQ[k] = qt;
      sR[k] = thr;
      sB[k] = b;
    }
    __syncthreads();
    if (active) {
      // buoyancy_update_sa second loop (:121-130): k in [1, n2-3)
      if (k >= 1 && k < n2 - 3) a.wt[idx] = a.wt[idx] + interp_2(sB[k], sB[k + 1]);
      // bvf_sa second loop (:159-180): k in [2, n2-2)
      if (k >= 2 && k < n2 - 2) {
        double bv;
        if (qv < qt) {
          const double Lv = latent_heat(T);
          const double pv_star = table_lookup(a.LT, T, a.err);
          const double rsl = eps_v * pv_star / (p0 - pv_star);
          const double gamma_w = g / cpd * (1.0 / (1.0 - qt)) * (1.0 + Lv * rsl / (Rd * T)) /
                                 (cpm_c(qt) / cpd + Lv * Lv * (eps_v + rsl) * rsl / (cpd * Rd * T * T));
          const double dTdz = (interp_2(sT[k], sT[k + 1]) - interp_2(sT[k - 1], sT[k])) * dzi;
          const double dqtdz = (interp_2(sQ[k], sQ[k + 1]) - interp_2(sQ[k - 1], sQ[k])) * dzi;
          bv = g / T * (dTdz + gamma_w) * (1.0 + Lv * rsl / (Rd * T)) - dqtdz / (1.0 - qt);
        } else {
          bv = g / sR[k] * (interp_2(sR[k], sR[k + 1]) - interp_2(sR[k - 1], sR[k])) * dzi;
        }
        a.bvf[idx] = bv;
      }
    }
    __syncthreads();  // shared memory is reused by the next column group
  }
  if (a.stats) {
    // warp-aggregated secant statistics
    for (int off = 16; off > 0; off >>= 1) {
      my_it += __shfl_down_sync(0xffffffffu, my_it, off);
      my_sat += __shfl_down_sync(0xffffffffu, my_sat, off);
    }
    if ((threadIdx.x & 31) == 0 && (my_it | my_sat)) {
      atomicAdd(a.stats, my_it);
      atomicAdd(a.stats + 1, my_sat);
    }
  }
}

struct DryArgs {
  const double* pd;       // RS.p0_half
  const double* alpha0;   // RS.alpha0_half
  const double* s;
  double* T;
  double* alpha;
  double* buoy;
  double* theta;
  double* bvf;
  double* wt;
};

// ThermodynamicsDry.update (ThermodynamicsDry.pyx:105-120).
__global__ void thermo_dry_kernel(Geo geo, DryArgs a, long long ncols) {
  extern __shared__ double sm[];
  const int kpad = blockDim.x;
  const long long col = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  const int k = threadIdx.x;
  const long long n2 = geo.n2;
  double* sTh = sm + (size_t)threadIdx.y * 2 * kpad;
  double* sB = sTh + kpad;
  const bool active = (col < ncols) && (k < n2);
  const long long i = col / geo.n1;
  const long long j = col - i * geo.n1;
  long long idx = 0;
  double T = 0.0;
  if (active) {
    idx = col * n2 + k;
    const double pd = a.pd[k];
    // eos_c (Csrc/thermodynamics_dry.h:8-10), eos_update (:12-37)
    T = T_tilde * (crm::exp((a.s[idx] - sd_tilde + Rd * crm::log(pd / p_tilde)) / cpd));
    a.T[idx] = T;
    const double al = mul_rn((Rd * T) / pd, 1.0);
    a.alpha[idx] = al;
    // buoyancy_update (:39-73): i < n0-1, j < n1-1, k < n2-1
    const bool bij = (i < geo.n0 - 1) && (j < geo.n1 - 1);
    double b = 0.0;
    if (bij && k < n2 - 1) {
      b = buoyancy_c(a.alpha0[k], al);
      a.buoy[idx] = b;
    } else if (bij) {
      b = a.buoy[idx];  // level n2-1 keeps the field's current value
    }
    sB[k] = b;
    // bvf_dry (:75-110): theta on k in [1, n2)
    double th = 0.0;
    if (k >= 1) {
      th = T / pow(pd / p_tilde, kappa);
      a.theta[idx] = th;
    }
    sTh[k] = th;
  }
  __syncthreads();
  if (active) {
    if ((i < geo.n0 - 1) && (j < geo.n1 - 1) && k < n2 - 1) a.wt[idx] += interp_2(sB[k], sB[k + 1]);
    if (k >= 2 && k < n2 - 1) {
      const double dzi = 1.0 / geo.dx2;
      a.bvf[idx] = g / sTh[k] * (interp_2(sTh[k], sTh[k + 1]) - interp_2(sTh[k - 1], sTh[k])) * dzi;
    }
  }
}

// Learned seeds for the saturated cells (the learned path of pb_thermo_sa):
// each warp takes 32 consecutive cells, finds the saturated ones with the
// same first temperature estimate eos_c starts from (:22-32), compacts them
// into warp-private shared slots and evaluates the MLP on them in tiles of
// 16 on the tensor cores; seed[ijk] then replaces the secant's second point.
struct SeedArgs {
  const double* p0;
  const double* s;
  const double* qt;
  pb_table LT;
  unsigned int* err;
  double* seed;
  const __nv_bfloat16* w1;
  const float* b1;
  const __nv_bfloat16* w2;
  const float* b2;
  const __nv_bfloat16* w3;
  const float* b3;
  float lo[3], hi[3];
  float out_mean, out_scale;
  long long npg;
  long long n2;
  int clip;
};

constexpr int kSeedWarps = 4;

__global__ void __launch_bounds__(128) thermo_seed_kernel(SeedArgs a) {
  __shared__ mlpk::Smem sm;
  __shared__ float slot_x[kSeedWarps][32][3];
  __shared__ long long slot_i[kSeedWarps][32];
  mlpk::stage_weights(sm, a.w1, a.b1, a.w2, a.b2, a.w3, a.b3);
  __syncthreads();
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long base = gwarp * 32; base < a.npg; base += nwarps * 32) {
    const long long idx = base + lane;
    bool sat = false;
    double p0 = 0.0, s = 0.0, qt = 0.0;
    if (idx < a.npg) {
      p0 = a.p0[idx % a.n2];
      qt = a.qt[idx];
      if (a.clip) qt = fmax(qt, 1e-11);
      s = a.s[idx];
      const double pv_1 = pv_c(p0, qt, qt);
      const double pd_1 = p0 - pv_1;
      const double T_1 = temperature_no_ql(pd_1, pv_1, s, qt);
      const double qv_star_1 = qv_star_c(p0, qt, table_lookup(a.LT, T_1, a.err));
      sat = !(qt <= qv_star_1);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, sat);
    const int count = __popc(mask);
    if (sat) {
      const int pos = __popc(mask & ((1u << lane) - 1u));
      slot_x[wid][pos][0] = mlpk::norm_in(p0, a.lo[0], a.hi[0]);
      slot_x[wid][pos][1] = mlpk::norm_in(s, a.lo[1], a.hi[1]);
      slot_x[wid][pos][2] = mlpk::norm_in(qt, a.lo[2], a.hi[2]);
      slot_i[wid][pos] = idx;
    }
    __syncwarp();
    for (int t0 = 0; t0 < count; t0 += 16) {
      const int r0 = t0 + g, r1 = t0 + g + 8;
      float x0[3] = {0.f, 0.f, 0.f}, x1[3] = {0.f, 0.f, 0.f};
      if (r0 < count) for (int i = 0; i < 3; ++i) x0[i] = slot_x[wid][r0][i];
      if (r1 < count) for (int i = 0; i < 3; ++i) x1[i] = slot_x[wid][r1][i];
      float y0, y1;
      mlpk::forward_tile(sm, x0, x1, y0, y1, nullptr);
      if (t == 0) {
        if (r0 < count) a.seed[slot_i[wid][r0]] = (double)a.out_mean + (double)a.out_scale * (double)y0;
        if (r1 < count) a.seed[slot_i[wid][r1]] = (double)a.out_mean + (double)a.out_scale * (double)y1;
      }
    }
    __syncwarp();
  }
}

// Column-group grid: enough blocks to fill the GPU several times over, each
// looping over its share of columns.
unsigned int column_grid(long long ncols, dim3 blk) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long groups = (ncols + blk.y - 1) / blk.y;
  const long long cap = (long long)sms * 16;
  return (unsigned int)(groups < cap ? groups : cap);
}

void column_launch_shape(long long n2, int per_col_arrays, dim3* blk, size_t* smem) {
  const int kpad = (int)((n2 + 31) / 32 * 32);
  int cols = 256 / kpad;
  if (cols < 1) cols = 1;
  *blk = dim3(kpad, cols);
  *smem = (size_t)per_col_arrays * kpad * cols * sizeof(double);
}

}  // namespace thermo_k

using namespace thermo_k;

extern "C" int pb_thermo_sa(const pb_dims* dims, const double* p0_half, const double* alpha0_half,
                            const pb_table* table, const double* s, double* qt, double* T, double* qv,
                            double* ql, double* qi, double* alpha, double* buoyancy, double* theta_rho,
                            double* bvf, double* thetali, double* w_tend, int clip_qt, const pb_mlp* mlp,
                            double* seed_scratch, long long* secant_iters, int max_iter, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!p0_half || !alpha0_half || !table || !table->y || table->n < 2 || !(table->dx > 0.0)) return PB_ERR_ARG;
  if (!s || !qt || !T || !qv || !ql || !qi || !alpha || !buoyancy || !theta_rho || !bvf || !thetali || !w_tend)
    return PB_ERR_ARG;
  if (max_iter < 1) return PB_ERR_ARG;
  if (dims->nlg[2] > 1024) return PB_ERR_UNSUPPORTED;
  if (mlp && (!seed_scratch || !mlp->w1 || !mlp->b1 || !mlp->w2 || !mlp->b2 || !mlp->w3 || !mlp->b3))
    return PB_ERR_ARG;
  const Geo geo = make_geo(dims);
  SaArgs a;
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
  a.seed = nullptr;
  a.stats = reinterpret_cast<unsigned long long*>(secant_iters);
  a.err = pb_error_word_ptr();
  if (!a.err) return PB_ERR_CUDA;
  if (mlp) {
    SeedArgs sa;
    sa.p0 = p0_half;
    sa.s = s;
    sa.qt = qt;
    sa.LT = *table;
    sa.err = a.err;
    sa.seed = seed_scratch;
    sa.w1 = static_cast<const __nv_bfloat16*>(mlp->w1);
    sa.b1 = mlp->b1;
    sa.w2 = static_cast<const __nv_bfloat16*>(mlp->w2);
    sa.b2 = mlp->b2;
    sa.w3 = static_cast<const __nv_bfloat16*>(mlp->w3);
    sa.b3 = mlp->b3;
    for (int i = 0; i < 3; ++i) {
      sa.lo[i] = mlp->in_lo[i];
      sa.hi[i] = mlp->in_hi[i];
    }
    sa.out_mean = mlp->out_mean;
    sa.out_scale = mlp->out_scale;
    sa.npg = geo.npg;
    sa.n2 = geo.n2;
    sa.clip = clip_qt;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long blocks = (geo.npg + 32 * kSeedWarps - 1) / (32 * kSeedWarps);
    if (blocks > (long long)sms * 16) blocks = (long long)sms * 16;
    thermo_seed_kernel<<<(unsigned)blocks, 32 * kSeedWarps, 0, as_stream(stream)>>>(sa);
    pb_note_launch();
    PB_LAUNCH_CHECK();
    a.seed = seed_scratch;
  }
  a.clip = clip_qt;
  a.max_iter = max_iter;
  dim3 blk;
  size_t smem;
  column_launch_shape(geo.n2, 4, &blk, &smem);
  const long long ncols = geo.n0 * geo.n1;
  thermo_sa_kernel<<<column_grid(ncols, blk), blk, smem, as_stream(stream)>>>(geo, a, ncols);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_thermo_dry(const pb_dims* dims, const double* p0_half, const double* alpha0_half,
                             const double* s, double* T, double* alpha, double* buoyancy, double* theta,
                             double* bvf, double* w_tend, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!p0_half || !alpha0_half || !s || !T || !alpha || !buoyancy || !theta || !bvf || !w_tend) return PB_ERR_ARG;
  if (dims->nlg[2] > 1024) return PB_ERR_UNSUPPORTED;
  const Geo geo = make_geo(dims);
  DryArgs a{p0_half, alpha0_half, s, T, alpha, buoyancy, theta, bvf, w_tend};
  dim3 blk;
  size_t smem;
  column_launch_shape(geo.n2, 2, &blk, &smem);
  const long long ncols = geo.n0 * geo.n1;
  thermo_dry_kernel<<<ceil_div(ncols, blk.y), blk, smem, as_stream(stream)>>>(geo, a, ncols);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

// ---- pointwise saturation adjustment ----------------------------------------
// ThermodynamicsSA.eos (ThermodynamicsSA.pyx:169-174): eos_c for a list of
// (p0, s, qt) points.  Used to generate the learned seed's training pairs and
// to count secant iterations with and without a seed.
namespace thermo_k {

struct EosPointArgs {
  pb_table LT;
  const double* p0;
  const double* s;
  const double* qt;
  const double* seed;  // nullable: second secant point per point
  double* T;
  double* ql;
  double* qi;
  int* iters;          // nullable: secant iterations per point (0 = unsaturated)
  unsigned int* err;
  long long n;
  int max_iter;
};

__global__ void eos_points_kernel(EosPointArgs a) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const EosOut e = eos_sa(a.LT, a.p0[i], a.s[i], a.qt[i], a.max_iter, a.seed != nullptr,
                            a.seed ? a.seed[i] : 0.0, a.err);
    a.T[i] = e.T;
    if (a.ql) a.ql[i] = e.ql;
    if (a.qi) a.qi[i] = e.qi;
    if (a.iters) a.iters[i] = e.iters;
  }
}

}  // namespace thermo_k

extern "C" int pb_eos_sa(const pb_table* table, const double* p0, const double* s, const double* qt,
                         const double* seed, double* T, double* ql, double* qi, int* iters, long long n,
                         int max_iter, void* stream) {
  if (!table || !table->y || table->n < 2 || !(table->dx > 0.0)) return PB_ERR_ARG;
  if (!p0 || !s || !qt || !T || n < 0 || max_iter < 1) return PB_ERR_ARG;
  if (n == 0) return PB_OK;
  thermo_k::EosPointArgs a;
  a.LT = *table;
  a.p0 = p0;
  a.s = s;
  a.qt = qt;
  a.seed = seed;
  a.T = T;
  a.ql = ql;
  a.qi = qi;
  a.iters = iters;
  a.err = pb_error_word_ptr();
  if (!a.err) return PB_ERR_CUDA;
  a.n = n;
  a.max_iter = max_iter;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sms * 16) blocks = (long long)sms * 16;
  thermo_k::eos_points_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
