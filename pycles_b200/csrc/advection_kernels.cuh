// WENO scalar and momentum advection kernels with flux divergence, shared by
// the two translation units that instantiate them: advection_f64.cu (the FP64
// plain form, compiled without FMA contraction so that every operation is
// rounded as the reference's C evaluates it) and advection.cu (the FP32
// precision form and the C entry points).
//
// Direction-split, one launch per (direction, group): the x and y kernels
// give each thread one (other-axis, k) column and march along the advection
// axis, keeping the stencil in a register window and the previous face flux
// in a register, so every face flux is computed once and each cell's
// tendency is read-modified-written once per direction.  The z kernel puts
// k on the lanes; lane L computes the flux of face f = k0-1+L and takes the
// flux of face f-1 from lane L-1 by shuffle (31 cells per warp).  The
// precision form's momentum advection runs all three directions in one pass
// instead (momentum_fused).
//
// Order of the tendency updates per variable is the reference's: d = 0, 1, 2
// (ScalarAdvection.pyx:81, MomentumAdvection.pyx:56-60), each
//   tend -= alpha(k) * (F[f] - F[f-1]) * dxi[d]      (Csrc/flux_divergence.h)
#pragma once

#include "pb_common.cuh"
#include "weno.cuh"

namespace pbadv {

constexpr int kMaxScalars = 4;

struct ScalarArgs {
  const double* vel;           // advecting velocity of this direction
  const double* rho0;
  const double* rho0_half;
  const double* alpha0_half;
  const double* s[kMaxScalars];
  double* t[kMaxScalars];
  double* flux[kMaxScalars];   // this direction's flux slab or nullptr
  int ns;
};

struct MomArgs {
  const double* vel[3];        // u, v, w
  double* tend[3];
  const double* rho0;
  const double* rho0_half;
  const double* alpha0;
  const double* alpha0_half;
};

template <int ORDER>
struct St {
  static constexpr int R = (ORDER + 1) / 2;  // half-width: faces read f-R+1 .. f+R
  static constexpr int W = 2 * R;            // register window
};

namespace {
// ---------------------------------------------------------------------------
// scalars, x / y directions
// ---------------------------------------------------------------------------
template <int D, int ORDER, bool F32, int NS>
__global__ void __launch_bounds__(128) scalar_march(Geo g, ScalarArgs a, int chunk) {
  constexpr int R = St<ORDER>::R;
  constexpr int W = St<ORDER>::W;
  const long long k = g.gw + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long o = g.gw + (long long)blockIdx.y * blockDim.y + threadIdx.y;
  const long long nD = (D == 0) ? g.n0 : g.n1;
  const long long nO = (D == 0) ? g.n1 : g.n0;
  if (k >= g.n2 - g.gw || o >= nO - g.gw) return;
  const long long sD = (D == 0) ? g.is : g.js;
  const long long sO = (D == 0) ? g.js : g.is;
  const long long c0 = g.gw + (long long)blockIdx.z * chunk;
  if (c0 >= nD - g.gw) return;
  const long long c1 = min(c0 + (long long)chunk, nD - g.gw);
  const long long base = o * sO + k;
  const double rho = a.rho0_half[k];
  const double alpha = a.alpha0_half[k];
  const double dxi = (D == 0) ? g.dxi0 : g.dxi1;

  double win[NS][W];
  double fprev[NS];
  double nxt[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
#pragma unroll
    for (int m = 0; m < W - 1; ++m) win[q][m] = a.s[q][(c0 - 1 - R + 1 + m) * sD + base];
    nxt[q] = a.s[q][(c0 - 1 + R) * sD + base];
    fprev[q] = 0.0;
  }
  double vnxt = a.vel[(c0 - 1) * sD + base];
  for (long long f = c0 - 1; f < c1; ++f) {
    const long long idx = f * sD + base;
    const double vel = vnxt;
    // software prefetch of the next face's loads, consumed one iteration later
    const bool more = f + 1 < c1;
    if (more) vnxt = a.vel[idx + sD];
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      win[q][W - 1] = nxt[q];
      if (more) nxt[q] = a.s[q][(f + 1 + R) * sD + base];
      const double phi = weno_upwind<ORDER, F32>(vel >= 0.0, win[q]);
      const double F = upwind_flux1(vel, phi, rho);
      if (f >= c0) a.t[q][idx] -= alpha * (F - fprev[q]) * dxi;
      if (a.flux[q] != nullptr) a.flux[q][idx] = F;
      fprev[q] = F;
#pragma unroll
      for (int m = 0; m < W - 1; ++m) win[q][m] = win[q][m + 1];
    }
  }
}

// ---------------------------------------------------------------------------
// scalars, z direction
// ---------------------------------------------------------------------------
template <int ORDER, bool F32, int NS>
__global__ void __launch_bounds__(128) scalar_z(Geo g, ScalarArgs a, long long nwarps) {
  constexpr int R = St<ORDER>::R;
  const int lane = threadIdx.x & 31;
  const long long wid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (wid >= nwarps) return;
  const long long nl1 = g.n1 - 2 * g.gw;
  const long long nl2 = g.n2 - 2 * g.gw;
  const long long nseg = (nl2 + 30) / 31;
  const long long seg = wid % nseg;
  const long long rest = wid / nseg;
  const long long j = g.gw + rest % nl1;
  const long long i = g.gw + rest / nl1;
  const long long f = g.gw + seg * 31 - 1 + lane;   // face of this lane = cell of this lane
  const bool valid = f <= g.n2 - g.gw - 1;
  const long long col = i * g.is + j * g.js;
  const double dzi = g.dxi2;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    double F = 0.0;
    if (valid) {
      const double* s = a.s[q] + col + f - (R - 1);
      double v[2 * R];
#pragma unroll
      for (int m = 0; m < 2 * R; ++m) v[m] = s[m];
      const double vel = a.vel[col + f];
      F = upwind_flux1(vel, weno_upwind<ORDER, F32>(vel >= 0.0, v), a.rho0[f]);
      if (a.flux[q] != nullptr) a.flux[q][col + f] = F;
    }
    const double Fm = __shfl_up_sync(0xffffffffu, F, 1);
    if (valid && lane > 0) a.t[q][col + f] -= a.alpha0_half[f] * (F - Fm) * dzi;
  }
}

// ---------------------------------------------------------------------------
// momentum, x / y directions (advecting velocity = component D)
// ---------------------------------------------------------------------------
template <int D, int ORDER, bool F32>
__global__ void __launch_bounds__(128) momentum_march(Geo g, MomArgs a, int chunk) {
  constexpr int R = St<ORDER>::R;
  constexpr int W = St<ORDER>::W;
  constexpr int O = 1 - D;  // other horizontal axis
  const long long k = g.gw + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long o = g.gw + (long long)blockIdx.y * blockDim.y + threadIdx.y;
  const long long nD = (D == 0) ? g.n0 : g.n1;
  const long long nO = (D == 0) ? g.n1 : g.n0;
  if (k >= g.n2 - g.gw || o >= nO - g.gw) return;
  const long long sD = (D == 0) ? g.is : g.js;
  const long long sO = (D == 0) ? g.js : g.is;
  const long long c0 = g.gw + (long long)blockIdx.z * chunk;
  if (c0 >= nD - g.gw) return;
  const long long c1 = min(c0 + (long long)chunk, nD - g.gw);
  const long long base = o * sO + k;
  const double dxi = (D == 0) ? g.dxi0 : g.dxi1;
  const double* vD = a.vel[D];
  // rho/alpha per advected component (momentum_advection_weno.h:145-236,
  // flux_divergence.h:45-58): horizontal components use the half levels,
  // w uses the full levels.
  const double rho_h = a.rho0_half[k];
  const double rho_f = a.rho0[k];
  const double al_h = a.alpha0_half[k];
  const double al_f = a.alpha0[k];

  double win[3][W];
  double fprev[3];
  double nxt[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int m = 0; m < W - 1; ++m) win[c][m] = a.vel[c][(c0 - 1 - R + 1 + m) * sD + base];
    nxt[c] = a.vel[c][(c0 - 1 + R) * sD + base];
    fprev[c] = 0.0;
  }
  for (long long f = c0 - 1; f < c1; ++f) {
    const long long idx = f * sD + base;
    const bool more = f + 1 < c1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      win[c][W - 1] = nxt[c];
      if (more) nxt[c] = a.vel[c][(f + 1 + R) * sD + base];
    }
    // window position of face f is R-1
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double vel_adv;
      if (c == D) {
        if constexpr (ORDER == 5)
          vel_adv = interp_4<double>(win[D][R - 2], win[D][R - 1], win[D][R], win[D][R + 1]);
        else
          vel_adv = interp_6<double>(win[D][R - 3], win[D][R - 2], win[D][R - 1], win[D][R], win[D][R + 1],
                                     win[D][R + 2]);
      } else {
        const long long st = (c == O) ? sO : 1;
        const double* p = vD + idx;
        if constexpr (ORDER == 5)
          vel_adv = interp_4<double>(p[-st], p[0], p[st], p[2 * st]);
        else
          vel_adv = interp_6<double>(p[-2 * st], p[-st], p[0], p[st], p[2 * st], p[3 * st]);
      }
      const double phi = weno_upwind<ORDER, F32>(vel_adv >= 0.0, win[c]);
      const double F = upwind_flux1(vel_adv, phi, (c == 2) ? rho_f : rho_h);
      if (f >= c0) a.tend[c][idx] -= ((c == 2) ? al_f : al_h) * (F - fprev[c]) * dxi;
      fprev[c] = F;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int m = 0; m < W - 1; ++m) win[c][m] = win[c][m + 1];
    }
  }
}

// ---------------------------------------------------------------------------
// momentum, z direction (advecting velocity = w)
// ---------------------------------------------------------------------------
template <int ORDER, bool F32>
__global__ void __launch_bounds__(128) momentum_z(Geo g, MomArgs a, long long nwarps) {
  const int lane = threadIdx.x & 31;
  const long long wid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (wid >= nwarps) return;
  const long long nl1 = g.n1 - 2 * g.gw;
  const long long nl2 = g.n2 - 2 * g.gw;
  const long long nseg = (nl2 + 30) / 31;
  const long long seg = wid % nseg;
  const long long rest = wid / nseg;
  const long long j = g.gw + rest % nl1;
  const long long i = g.gw + rest / nl1;
  const long long f = g.gw + seg * 31 - 1 + lane;
  const bool valid = f <= g.n2 - g.gw - 1;
  const long long idx = i * g.is + j * g.js + f;
  const double dzi = g.dxi2;
  const double* wv = a.vel[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double F = 0.0;
    if (valid) {
      const long long st = (c == 0) ? g.is : ((c == 1) ? g.js : 1);
      const double* p = wv + idx;
      double vel_adv;
      if constexpr (ORDER == 5)
        vel_adv = interp_4<double>(p[-st], p[0], p[st], p[2 * st]);
      else
        vel_adv = interp_6<double>(p[-2 * st], p[-st], p[0], p[st], p[2 * st], p[3 * st]);
      constexpr int R = St<ORDER>::R;
      const double* s = a.vel[c] + idx - (R - 1);
      double v[2 * R];
#pragma unroll
      for (int m = 0; m < 2 * R; ++m) v[m] = s[m];
      const double rho = (c == 2) ? a.rho0_half[f + 1] : a.rho0[f];
      F = upwind_flux1(vel_adv, weno_upwind<ORDER, F32>(vel_adv >= 0.0, v), rho);
    }
    const double Fm = __shfl_up_sync(0xffffffffu, F, 1);
    if (valid && lane > 0) {
      const double al = (c == 2) ? a.alpha0[f] : a.alpha0_half[f];
      a.tend[c][idx] -= al * (F - Fm) * dzi;
    }
  }
}

// ---------------------------------------------------------------------------
// momentum, all three advecting directions in one pass (precision form)
// ---------------------------------------------------------------------------
// Block (32, 4): lane L holds level k = k0 - 1 + L (lanes 1..31 are cells,
// lane 0 the level below), threadIdx.y the row j; every thread marches along
// x over a chunk of cells.  Per cell and advected component: the x face flux
// from the register window (the previous face kept in a register), the two
// y face fluxes from the row's neighbours (L1-cached loads), the z face flux
// of the lane's upper face with the lower one from lane L-1 by shuffle.  The
// x windows also give the x neighbours that the y and z faces'
// advecting-velocity interpolations need (v and w along x); the rest comes
// from L1-cached loads.  Each tendency gets its x, y and z terms in the
// reference's order and is read and written once, so u, v, w and the three
// tendencies cross DRAM about once per stage instead of three times; the
// y faces are evaluated twice (once by each neighbouring cell), which costs
// less than a shared-memory exchange with its barriers (measured: 4.9 ms
// per stage for the three split launches, 4.6-4.9 fused, 512x512x256).
template <int ORDER, bool F32>
__device__ __forceinline__ double interp_c(const double* p) {  // p[0 .. ORDER-2]: the interpolant's points
  if constexpr (ORDER == 5)
    return interp_4<double>(p[0], p[1], p[2], p[3]);
  else
    return interp_6<double>(p[0], p[1], p[2], p[3], p[4], p[5]);
}

template <int ORDER, bool F32>
__global__ void __launch_bounds__(128) momentum_fused(Geo g, MomArgs a, int chunk) {
  constexpr int R = St<ORDER>::R;
  constexpr int W = St<ORDER>::W;
  constexpr int NI = ORDER - 1;  // points of the advecting-velocity interpolant (4 or 6)
  constexpr int HI = NI / 2 - 1; // it reads offsets -HI .. NI-1-HI around the face's lower cell
  const int lane = threadIdx.x;
  const long long k = g.gw - 1 + (long long)blockIdx.x * 31 + lane;
  const long long j = g.gw + (long long)blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= g.n1 - g.gw) return;  // whole warps
  const long long c0 = g.gw + (long long)blockIdx.z * chunk;
  const long long c1 = min(c0 + (long long)chunk, g.n0 - g.gw);
  const bool face_ok = k <= g.n2 - g.gw - 1;
  const bool cell = face_ok && lane >= 1;
  const long long base = j * g.js + k;
  const double rho_h = face_ok ? a.rho0_half[k] : 0.0;
  const double rho_f = face_ok ? a.rho0[k] : 0.0;
  const double rho_h1 = face_ok ? a.rho0_half[k + 1] : 0.0;
  const double al_h = face_ok ? a.alpha0_half[k] : 0.0;
  const double al_f = face_ok ? a.alpha0[k] : 0.0;
  const double dxi = g.dxi0, dyi = g.dxi1, dzi = g.dxi2;
  const double* __restrict__ U = a.vel[0];
  const double* __restrict__ V = a.vel[1];
  const double* __restrict__ Wv = a.vel[2];

  double win[3][W];
  double fprev[3];
  double nxt[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int m = 0; m < W - 1; ++m) win[c][m] = face_ok ? a.vel[c][(c0 - R + m) * g.is + base] : 0.0;
    nxt[c] = face_ok ? a.vel[c][(c0 - 1 + R) * g.is + base] : 0.0;
    fprev[c] = 0.0;
  }
  for (long long f = c0 - 1; f < c1; ++f) {
    const long long idx = f * g.is + base;
    const bool more = f + 1 < c1;
    const bool upd = f >= c0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      win[c][W - 1] = nxt[c];
      if (more && face_ok) nxt[c] = a.vel[c][(f + 1 + R) * g.is + base];
    }
    // window entry m holds x index f - R + 1 + m: the interpolant points
    // f - HI .. f - HI + NI - 1 start at m = R - 1 - HI
    constexpr int MI = R - 1 - HI;
    double Fx[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double vel_adv = 0.0;
      if (c == 0) {
        vel_adv = interp_c<ORDER, F32>(&win[0][MI]);
      } else if (face_ok) {
        const long long st = (c == 1) ? g.js : 1;
        double p[NI];
#pragma unroll
        for (int m = 0; m < NI; ++m) p[m] = U[idx + (m - HI) * st];
        vel_adv = interp_c<ORDER, F32>(p);
      }
      Fx[c] = upwind_flux1(vel_adv, weno_upwind<ORDER, F32>(vel_adv >= 0.0, win[c]), (c == 2) ? rho_f : rho_h);
    }
    if (upd) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double al = (c == 2) ? al_f : al_h;
        double ty = 0.0, Fz = 0.0;
        if (face_ok) {
          const double* pc = a.vel[c] + idx;
          double ys[2 * R + 1];  // component c along y, rows j-R .. j+R
#pragma unroll
          for (int m = 0; m <= 2 * R; ++m) ys[m] = pc[(m - R) * g.js];
          // advecting v interpolated along c, at the faces j+1/2 (row j) and j-1/2 (row j-1)
          double vap, vam;
          if (c == 0) {
            vap = interp_c<ORDER, F32>(&win[1][MI]);
            double p[NI];
#pragma unroll
            for (int m = 0; m < NI; ++m) p[m] = V[idx - g.js + (m - HI) * g.is];
            vam = interp_c<ORDER, F32>(p);
          } else if (c == 1) {
            vap = interp_c<ORDER, F32>(&ys[R - HI]);
            vam = interp_c<ORDER, F32>(&ys[R - 1 - HI]);
          } else {
            double p[NI], q[NI];
#pragma unroll
            for (int m = 0; m < NI; ++m) {
              p[m] = V[idx + (m - HI)];
              q[m] = V[idx - g.js + (m - HI)];
            }
            vap = interp_c<ORDER, F32>(p);
            vam = interp_c<ORDER, F32>(q);
          }
          const double rho = (c == 2) ? rho_f : rho_h;
          const double Fyp = upwind_flux1(vap, weno_upwind<ORDER, F32>(vap >= 0.0, ys + 1), rho);
          const double Fym = upwind_flux1(vam, weno_upwind<ORDER, F32>(vam >= 0.0, ys), rho);
          ty = al * (Fyp - Fym) * dyi;
          // z face k+1/2: component c along z, advecting w interpolated along c
          double zs[2 * R];
#pragma unroll
          for (int m = 0; m < 2 * R; ++m) zs[m] = pc[m - R + 1];
          double waz;
          if (c == 0) {
            waz = interp_c<ORDER, F32>(&win[2][MI]);
          } else if (c == 1) {
            double p[NI];
#pragma unroll
            for (int m = 0; m < NI; ++m) p[m] = Wv[idx + (m - HI) * g.js];
            waz = interp_c<ORDER, F32>(p);
          } else {
            waz = interp_c<ORDER, F32>(&zs[R - 1 - HI]);
          }
          Fz = upwind_flux1(waz, weno_upwind<ORDER, F32>(waz >= 0.0, zs), (c == 2) ? rho_h1 : rho_f);
        }
        const double Fzm = __shfl_up_sync(0xffffffffu, Fz, 1);
        if (cell) {
          double t = a.tend[c][idx];
          t -= al * (Fx[c] - fprev[c]) * dxi;
          t -= ty;
          t -= al * (Fz - Fzm) * dzi;
          a.tend[c][idx] = t;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      fprev[c] = Fx[c];
#pragma unroll
      for (int m = 0; m < W - 1; ++m) win[c][m] = win[c][m + 1];
    }
  }
}

constexpr int kChunk = 64;  // cells per marching thread along x / y

template <int ORDER, bool F32, int NS>
cudaError_t launch_scalar_group(const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                                const double* const vel[3], cudaStream_t st) {
  const long long nl0 = g.n0 - 2 * g.gw, nl1 = g.n1 - 2 * g.gw, nl2 = g.n2 - 2 * g.gw;
  dim3 blk(32, 4);
  {
    ScalarArgs a = base;
    a.vel = vel[0];
    for (int q = 0; q < NS; ++q) a.flux[q] = flux_dir[0] ? flux_dir[0][q] : nullptr;
    dim3 grd(ceil_div(nl2, 32), ceil_div(nl1, 4), ceil_div(nl0, kChunk));
    scalar_march<0, ORDER, F32, NS><<<grd, blk, 0, st>>>(g, a, kChunk);
    pb_note_launch();
  }
  {
    ScalarArgs a = base;
    a.vel = vel[1];
    for (int q = 0; q < NS; ++q) a.flux[q] = flux_dir[1] ? flux_dir[1][q] : nullptr;
    dim3 grd(ceil_div(nl2, 32), ceil_div(nl0, 4), ceil_div(nl1, kChunk));
    scalar_march<1, ORDER, F32, NS><<<grd, blk, 0, st>>>(g, a, kChunk);
    pb_note_launch();
  }
  {
    ScalarArgs a = base;
    a.vel = vel[2];
    for (int q = 0; q < NS; ++q) a.flux[q] = flux_dir[2] ? flux_dir[2][q] : nullptr;
    const long long nseg = (nl2 + 30) / 31;
    const long long nwarps = nl0 * nl1 * nseg;
    scalar_z<ORDER, F32, NS><<<ceil_div(nwarps, 4), 128, 0, st>>>(g, a, nwarps);
    pb_note_launch();
  }
  return cudaGetLastError();
}

template <int ORDER, bool F32>
cudaError_t launch_scalar_ns(int ns, const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                             const double* const vel[3], cudaStream_t st) {
  if constexpr (F32) {
    // precision form: one scalar per launch keeps the FP32 kernels at ~56
    // registers (twice the resident warps of the two-scalar windows); the
    // velocity is read once more per scalar
    for (int q = 0; q < ns; ++q) {
      ScalarArgs a = base;
      a.s[0] = base.s[q];
      a.t[0] = base.t[q];
      a.ns = 1;
      double* fq[3][1];
      double* const* fd[3];
      for (int d = 0; d < 3; ++d) {
        fq[d][0] = flux_dir[d] ? flux_dir[d][q] : nullptr;
        fd[d] = flux_dir[d] ? fq[d] : nullptr;
      }
      const cudaError_t e = launch_scalar_group<ORDER, F32, 1>(g, a, fd, vel, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  } else {
    switch (ns) {
      case 1: return launch_scalar_group<ORDER, F32, 1>(g, base, flux_dir, vel, st);
      case 2: return launch_scalar_group<ORDER, F32, 2>(g, base, flux_dir, vel, st);
      case 3: return launch_scalar_group<ORDER, F32, 3>(g, base, flux_dir, vel, st);
      default: return launch_scalar_group<ORDER, F32, 4>(g, base, flux_dir, vel, st);
    }
  }
}

template <int ORDER, bool F32>
cudaError_t launch_momentum(const Geo& g, const MomArgs& a, cudaStream_t st) {
  const long long nl0 = g.n0 - 2 * g.gw, nl1 = g.n1 - 2 * g.gw, nl2 = g.n2 - 2 * g.gw;
  dim3 blk(32, 4);
  if constexpr (F32) {  // precision form: one pass for the three advecting directions
    momentum_fused<ORDER, F32><<<dim3(ceil_div(nl2, 31), ceil_div(nl1, 4), ceil_div(nl0, kChunk)), blk, 0, st>>>(
        g, a, kChunk);
    pb_note_launch();
    return cudaGetLastError();
  } else {
  momentum_march<0, ORDER, F32><<<dim3(ceil_div(nl2, 32), ceil_div(nl1, 4), ceil_div(nl0, kChunk)), blk, 0,
                                  st>>>(g, a, kChunk);
  pb_note_launch();
  momentum_march<1, ORDER, F32><<<dim3(ceil_div(nl2, 32), ceil_div(nl0, 4), ceil_div(nl1, kChunk)), blk, 0,
                                  st>>>(g, a, kChunk);
  pb_note_launch();
  const long long nseg = (nl2 + 30) / 31;
  const long long nwarps = nl0 * nl1 * nseg;
  momentum_z<ORDER, F32><<<ceil_div(nwarps, 4), 128, 0, st>>>(g, a, nwarps);
  pb_note_launch();
  return cudaGetLastError();
  }
}

}  // namespace

// FP64 plain form (advection_f64.cu) and FP32 precision form (advection.cu).
cudaError_t scalar_fp64(int order, int ns, const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                        const double* const vel[3], cudaStream_t st);
cudaError_t scalar_fp32(int order, int ns, const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                        const double* const vel[3], cudaStream_t st);
cudaError_t momentum_fp64(int order, const Geo& g, const MomArgs& a, cudaStream_t st);
cudaError_t momentum_fp32(int order, const Geo& g, const MomArgs& a, cudaStream_t st);

}  // namespace pbadv
