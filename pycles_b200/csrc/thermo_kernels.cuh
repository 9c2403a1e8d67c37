// Saturation-adjustment and dry thermodynamics kernels, templated on the
// exp/log implementation (thermo_funcs.cuh) and instantiated by
// thermo.cu (FP64 plain form, correctly rounded exp/log, no FMA) and
// thermo_fast.cu (precision form: CUDA exp/log, FMA, optional learned seed).
//
// Saturation adjustment: warps own vertical segments of columns (see
// thermo_sa_kernel).  Dry thermodynamics: one thread block owns whole (i,j)
// columns, one thread per level, neighbours through shared memory.
#pragma once

#include "pb_common.cuh"
#include "thermo_funcs.cuh"

namespace thermo_k {

struct SeedNet {             // learned seed (precision form), see pb_mlp
  const float* y;            // network output per cell, refreshed before the kernel
  float out_mean, out_scale;
};

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
  unsigned long long* stats; // {iterations, saturated cells} (nullable)
  unsigned int* err;         // device error word
  SeedNet net;
  int clip;
  int max_iter;
};

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

// Launch shape of the dry kernel: blocks of (kpad, cols) threads, kpad = n2
// rounded up to a warp, cols columns per block; dynamic shared memory for the
// per-column arrays.
void column_launch_shape(long long n2, int per_col_arrays, dim3* blk, size_t* smem);

// Per-translation-unit launchers.
cudaError_t launch_sa_exact(const Geo& geo, const SaArgs& a, cudaStream_t st);
cudaError_t launch_dry_exact(const Geo& geo, const DryArgs& a, cudaStream_t st);
cudaError_t launch_sa_fast(const Geo& geo, const SaArgs& a, bool seeded, cudaStream_t st);
cudaError_t launch_dry_fast(const Geo& geo, const DryArgs& a, cudaStream_t st);

}  // namespace thermo_k

namespace {
namespace thermo_kk {

using namespace pbc;
using namespace thermo_f;
using thermo_k::DryArgs;
using thermo_k::SaArgs;

// ThermodynamicsSA.update (ThermodynamicsSA.pyx:176-213): clip_qt, eos_update,
// buoyancy_update_sa, bvf_sa, thetali_update.
//
// Work is split into tasks of one segment of kSeg levels of one column:
// lane L of the warp holds level k = kSeg*seg - 1 + L, lanes 1..kSeg are the
// segment's cells and lanes 0 and kSeg+1 recompute the neighbouring levels
// (same code, same inputs, same result as the warp that owns them), so the
// vertical neighbours that buoyancy_update_sa / bvf_sa need come by shuffle
// and no block barrier is needed.  Warps take the tasks in column-major
// order, grid-stride, so every warp sees every segment and the cloud-layer
// segments, whose secant iterates, are spread over all warps.  The Exner
// function of every level is tabulated in shared memory once per block.
//
// SEED: each saturated cell starts the secant from
//   T_2 = T_1 + out_mean + out_scale * y[cell]
// (clamped in eos_finish), y refreshed by the network kernel beforehand;
// a cell whose y is NaN (not saturated at the last refresh) takes the
// reference's second point.
constexpr int kSeg = 30;
constexpr int kSaThreads = 256;

template <class M, bool SEED>
__global__ void __launch_bounds__(kSaThreads, 4) thermo_sa_kernel(Geo geo, SaArgs a, long long ncols, int nseg) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31;
  const long long n2 = geo.n2;
  // per level: the Exner function, and for the precision form the
  // reciprocals of p0, alpha0 and the Exner function (FP64 divisions by
  // them become multiplications)
  double* exner_tab = reinterpret_cast<double*>(smraw);  // [n2] (x4 in the precision form)
  for (int k = threadIdx.x; k < n2; k += blockDim.x) {
    const double ex = pow(a.p0[k] / p_tilde, kappa);
    exner_tab[k] = ex;
    if constexpr (!M::exact) {
      exner_tab[n2 + k] = 1.0 / ex;
      exner_tab[2 * n2 + k] = 1.0 / a.p0[k];
      exner_tab[3 * n2 + k] = 1.0 / a.alpha0[k];
    }
  }
  __syncthreads();
  const long long ntask = ncols * nseg;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const double dzi = 1.0 / geo.dx2;
  unsigned long long my_it = 0, my_sat = 0;
  for (long long task = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; task < ntask; task += nwarps) {
    const long long col = task / nseg;
    const int seg = (int)(task - col * nseg);
    const long long k = (long long)seg * kSeg - 1 + lane;
    const bool kin = k >= 0 && k < n2;
    const bool own = kin && lane >= 1 && lane <= kSeg;
    const double p0 = kin ? __ldg(a.p0 + k) : 1.0;
    const double a0 = kin ? __ldg(a.alpha0 + k) : 1.0;
    const double exner = kin ? exner_tab[k] : 1.0;
    const long long idx = col * n2 + k;  // columns are contiguous: (i*n1 + j)*n2
    double qt = 0.0, s = 0.0;
    EosStart st{};
    if (kin) {
      qt = a.qt[idx];
      if (a.clip) {  // clip_qt (Csrc/thermodynamics_sa.h:213-219)
        qt = fmax(qt, 1e-11);
        if (own) a.qt[idx] = qt;
      }
      s = a.s[idx];
      st = eos_start<M>(a.LT, p0, s, qt, a.err);
    }
    double seed = 0.0;
    bool seeded = false;
    if constexpr (SEED) {
      if (kin && st.sat) {
        const float y = a.net.y[idx];  // NaN: not evaluated at the last refresh
        seeded = isfinite(y);
        seed = st.T_1 + (double)a.net.out_mean + (double)a.net.out_scale * (double)y;
      }
    }
    double T = 0.0, qv = 0.0, thr = 0.0, b = 0.0;
    if (kin) {
      const EosOut e = eos_finish<M>(a.LT, st, p0, s, qt, a.max_iter, SEED && st.sat && seeded, seed, a.err);
      T = e.T;
      qv = e.qv;
      double al;
      if constexpr (M::exact) {
        al = alpha_c(p0, T, qt, qv);
        // bvf_sa first loop (:147-157): theta_rho on k in [1, n2-1)
        if (k >= 1 && k < n2 - 1) thr = T * (1.0 - qt + eps_vi * qv) / exner;
        // buoyancy_update_sa first loop (:110-119): k in [0, n2-1)
        if (k < n2 - 1) b = buoyancy_c(a0, al);
      } else {
        al = (Rd * T) * exner_tab[2 * n2 + k] * (1.0 - qt + eps_vi * qv);
        if (k >= 1 && k < n2 - 1) thr = T * (1.0 - qt + eps_vi * qv) * exner_tab[n2 + k];
        if (k < n2 - 1) b = g * (al - a0) * exner_tab[3 * n2 + k];
      }
      if (own) {
        if (!isfinite(T)) pb_flag_at(a.err, PB_ERR_NONFINITE);
        my_it += (unsigned long long)e.iters;
        my_sat += e.sat ? 1ull : 0ull;
        a.T[idx] = T;
        a.qv[idx] = qv;
        a.ql[idx] = e.ql;
        a.qi[idx] = e.qi;
        a.alpha[idx] = al;
        // thetali_update (:185-211) with thetali_c (thermodynamic_functions.h:15-18);
        // without condensate the exponential is exp(-0) = 1 exactly
        const double theta = M::exact ? T / exner : T * exner_tab[n2 + k];
        if (e.ql == 0.0 && e.qi == 0.0) {
          a.thetali[idx] = theta * 1.0;
        } else {
          const double Lv = latent_heat(T);
          a.thetali[idx] = theta * M::exp(-Lv * (e.ql / (1.0 - qt) + e.qi / (1.0 - qt)) / (T * cpd));
        }
        if (k >= 1 && k < n2 - 1) a.theta_rho[idx] = thr;
        if (k < n2 - 1) a.buoy[idx] = b;
      }
    }
    // vertical neighbours from the adjacent lanes
    const double T_dn = __shfl_up_sync(0xffffffffu, T, 1), T_up = __shfl_down_sync(0xffffffffu, T, 1);
    const double q_dn = __shfl_up_sync(0xffffffffu, qt, 1), q_up = __shfl_down_sync(0xffffffffu, qt, 1);
    const double r_dn = __shfl_up_sync(0xffffffffu, thr, 1), r_up = __shfl_down_sync(0xffffffffu, thr, 1);
    const double b_up = __shfl_down_sync(0xffffffffu, b, 1);
    if (own) {
      // buoyancy_update_sa second loop (:121-130): k in [1, n2-3)
      if (k >= 1 && k < n2 - 3) a.wt[idx] = a.wt[idx] + interp_2(b, b_up);
      // bvf_sa second loop (:159-180): k in [2, n2-2)
      if (k >= 2 && k < n2 - 2) {
        double bv;
        if (qv < qt) {
          const double Lv = latent_heat(T);
          const double pv_star = table_lookup(a.LT, T, a.err);
          const double rsl = eps_v * pv_star / (p0 - pv_star);
          const double gamma_w = g / cpd * (1.0 / (1.0 - qt)) * (1.0 + Lv * rsl / (Rd * T)) /
                                 (cpm_c(qt) / cpd + Lv * Lv * (eps_v + rsl) * rsl / (cpd * Rd * T * T));
          const double dTdz = (interp_2(T, T_up) - interp_2(T_dn, T)) * dzi;
          const double dqtdz = (interp_2(qt, q_up) - interp_2(q_dn, qt)) * dzi;
          bv = g / T * (dTdz + gamma_w) * (1.0 + Lv * rsl / (Rd * T)) - dqtdz / (1.0 - qt);
        } else {
          bv = g / thr * (interp_2(thr, r_up) - interp_2(r_dn, thr)) * dzi;
        }
        a.bvf[idx] = bv;
      }
    }
  }
  if (a.stats) {
    // warp-aggregated secant statistics
    for (int off = 16; off > 0; off >>= 1) {
      my_it += __shfl_down_sync(0xffffffffu, my_it, off);
      my_sat += __shfl_down_sync(0xffffffffu, my_sat, off);
    }
    if (lane == 0 && (my_it | my_sat)) {
      atomicAdd(a.stats, my_it);
      atomicAdd(a.stats + 1, my_sat);
    }
  }
}

// ThermodynamicsDry.update (ThermodynamicsDry.pyx:105-120).
template <class M>
__global__ void thermo_dry_kernel(Geo geo, DryArgs a, long long ncols) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* sm = reinterpret_cast<double*>(smraw);
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
    T = T_tilde * (M::exp((a.s[idx] - sd_tilde + Rd * M::log(pd / p_tilde)) / cpd));
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

template <class M, bool SEED>
cudaError_t launch_sa(const Geo& geo, const SaArgs& a, cudaStream_t st) {
  const size_t smem = ((M::exact ? 1 : 4) * geo.n2 * sizeof(double) + 15) / 16 * 16;
  if (smem > 48 * 1024) {
    const cudaError_t e =
        cudaFuncSetAttribute(thermo_sa_kernel<M, SEED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const long long ncols = geo.n0 * geo.n1;
  const int nseg = (int)((geo.n2 + kSeg - 1) / kSeg);
  // resident blocks only; their warps stride over the tasks
  int dev = 0, sms = 148, per_sm = 1;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, thermo_sa_kernel<M, SEED>, kSaThreads, smem);
  if (per_sm < 1) per_sm = 1;
  long long blocks = (long long)sms * per_sm;
  const long long need = (ncols * nseg + kSaThreads / 32 - 1) / (kSaThreads / 32);
  if (blocks > need) blocks = need;
  thermo_sa_kernel<M, SEED><<<(unsigned)blocks, kSaThreads, smem, st>>>(geo, a, ncols, nseg);
  pb_note_launch();
  return cudaGetLastError();
}

template <class M>
cudaError_t launch_dry(const Geo& geo, const DryArgs& a, cudaStream_t st) {
  dim3 blk;
  size_t smem;
  thermo_k::column_launch_shape(geo.n2, 2, &blk, &smem);
  const long long ncols = geo.n0 * geo.n1;
  thermo_dry_kernel<M><<<ceil_div(ncols, blk.y), blk, smem, st>>>(geo, a, ncols);
  pb_note_launch();
  return cudaGetLastError();
}

}  // namespace thermo_kk
}  // namespace
