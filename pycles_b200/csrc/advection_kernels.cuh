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
// instead (momentum_tile).
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
  // the SSP-RK3 stage fused into the precision form's scalar passes (one
  // scalar per launch): the x pass sets the tendency, the z pass applies
  // the stage and writes the new value and (stage 0) the copy
  int fused;
  double* vnew[kMaxScalars];
  double* copy[kMaxScalars];
  double dt;
  int stage;
};

struct MomArgs {
  const double* vel[3];        // u, v, w
  double* tend[3];
  const double* rho0;
  const double* rho0_half;
  const double* alpha0;
  const double* alpha0_half;
  // the SSP-RK3 stage fused into the precision form's momentum pass
  // (momentum_tile<ORDER, true>): new values, the stage-0 copies, dt, stage
  double* vnew[3];
  double* copy[3];
  double dt;
  int stage;
  unsigned int* err;           // device error word (bounded waits of the TMA plane ring)
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
__global__ void __launch_bounds__(128) scalar_z(Geo g, ScalarArgs a) {
  constexpr int R = St<ORDER>::R;
  const int lane = threadIdx.x & 31;
  // grid (segment, group of 4 rows, x): warp w of the block takes row 4*blockIdx.y + w
  const long long seg = blockIdx.x;
  const long long j = g.gw + (long long)blockIdx.y * 4 + (threadIdx.x >> 5);
  const long long i = g.gw + (long long)blockIdx.z;
  if (j >= g.n1 - g.gw) return;  // whole warps
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
// scalars, precision form: first-difference windows
// ---------------------------------------------------------------------------
// x / y: the marching thread keeps the FP32 first differences of the face's
// stencil (2R-1 of them) and the FP64 values phi[f .. f+R] (the possible
// centres, now and for the next R faces); each new cell costs one FP64
// subtraction and one rounding to FP32.  Face flux vel * phi_face * rho, the
// tendency update t -= (alpha dxi) (F - F_prev).
// SET: the pass is the first to touch the tendency in the stage (fused
// stepping), so it stores the x term instead of adding it to the stored
// value (0 - x, as the reference's accumulation into a zeroed tendency).
template <int D, int ORDER, bool SET>
__global__ void __launch_bounds__(128) scalar_march_f32(Geo g, ScalarArgs a, int chunk) {
  constexpr int R = St<ORDER>::R;
  constexpr int ND = 2 * R - 1;
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
  const double* __restrict__ phi = a.s[0] + o * sO + k;
  const double* __restrict__ vel = a.vel + o * sO + k;
  double* __restrict__ tend = a.t[0] + o * sO + k;
  double* __restrict__ flux = a.flux[0] ? a.flux[0] + o * sO + k : nullptr;
  const double rho = a.rho0_half[k];
  const double ad = a.alpha0_half[k] * ((D == 0) ? g.dxi0 : g.dxi1);

  // first face f = c0 - 1 reads phi[f-R+1 .. f+R]
  float d[ND];
  double ph[R + 1];  // phi[f .. f+R]
  {
    double w[2 * R];
#pragma unroll
    for (int m = 0; m < 2 * R; ++m) w[m] = phi[(c0 - R + m) * sD];
#pragma unroll
    for (int m = 0; m < ND; ++m) d[m] = (float)(w[m + 1] - w[m]);
#pragma unroll
    for (int m = 0; m <= R; ++m) ph[m] = w[R - 1 + m];
  }
  double nxt = phi[(c0 + R) * sD];
  double vnxt = vel[(c0 - 1) * sD];
  double tnxt = SET ? 0.0 : tend[c0 * sD];
  double fprev = 0.0;
  for (long long f = c0 - 1; f < c1; ++f) {
    const double u = vnxt;
    const double lead = nxt;
    const double t = tnxt;
    // prefetch: the next face's velocity and tendency, and the cell the
    // window takes on after the next face (none after the last face: phi
    // stays in bounds)
    if (f + 1 < c1) {
      vnxt = vel[(f + 1) * sD];
      if (!SET) tnxt = tend[(f + 1) * sD];
    }
    if (f + 2 < c1) nxt = phi[(f + 2 + R) * sD];
    const bool pos = u >= 0.0;
    const float r = weno_delta<ORDER>(pos, d);
    const double F = u * ((pos ? ph[0] : ph[1]) + (double)r) * rho;
    if (f >= c0) tend[f * sD] = fma(-ad, F - fprev, t);
    if (flux != nullptr) flux[f * sD] = F;
    fprev = F;
#pragma unroll
    for (int m = 0; m < ND - 1; ++m) d[m] = d[m + 1];
    d[ND - 1] = (float)(lead - ph[R]);
#pragma unroll
    for (int m = 0; m < R; ++m) ph[m] = ph[m + 1];
    ph[R] = lead;
  }
}

// z: lane L takes face f = k0 - 1 + L from the 2R values around it (L1
// hits: the warp's lanes overlap) and the lower face's flux from lane L-1.
// RK: the last pass over the tendency in fused stepping -- the cell's
// SSP-RK3 stage (the separately rounded operations of rk3_kernel) is
// applied here, the new value written to a.vnew (the stencils of other
// warps still read the current values) and, at stage 0, the copy; the
// tendency is not stored.
template <int ORDER, bool RK>
__global__ void __launch_bounds__(128) scalar_z_f32(Geo g, ScalarArgs a) {
  constexpr int R = St<ORDER>::R;
  constexpr int ND = 2 * R - 1;
  const int lane = threadIdx.x & 31;
  // grid (segment, group of 4 rows, x): warp w of the block takes row 4*blockIdx.y + w
  const long long seg = blockIdx.x;
  const long long j = g.gw + (long long)blockIdx.y * 4 + (threadIdx.x >> 5);
  const long long i = g.gw + (long long)blockIdx.z;
  if (j >= g.n1 - g.gw) return;  // whole warps
  const long long f = g.gw + seg * 31 - 1 + lane;
  const bool valid = f <= g.n2 - g.gw - 1;
  const long long col = i * g.is + j * g.js;
  double F = 0.0, val = 0.0;
  if (valid) {
    const double* s = a.s[0] + col + f - (R - 1);
    double w[2 * R];
#pragma unroll
    for (int m = 0; m < 2 * R; ++m) w[m] = s[m];
    float d[ND];
#pragma unroll
    for (int m = 0; m < ND; ++m) d[m] = (float)(w[m + 1] - w[m]);
    const double u = a.vel[col + f];
    const bool pos = u >= 0.0;
    F = u * ((pos ? w[R - 1] : w[R]) + (double)weno_delta<ORDER>(pos, d)) * a.rho0[f];
    if (a.flux[0] != nullptr) a.flux[0][col + f] = F;
    val = w[R - 1];
  }
  const double Fm = __shfl_up_sync(0xffffffffu, F, 1);
  if (valid && lane > 0) {
    const long long at = col + f;
    const double t = fma(-a.alpha0_half[f] * g.dxi2, F - Fm, a.t[0][at]);
    if constexpr (RK) {
      double nv;
      if (a.stage == 0) {
        a.copy[0][at] = val;
        nv = add_rn(val, mul_rn(t, a.dt));
      } else if (a.stage == 1) {
        nv = add_rn(mul_rn(0.75, a.copy[0][at]), mul_rn(0.25, add_rn(val, mul_rn(t, a.dt))));
      } else {
        nv = add_rn(mul_rn(1.0 / 3.0, a.copy[0][at]), mul_rn(2.0 / 3.0, add_rn(val, mul_rn(t, a.dt))));
      }
      a.vnew[0][at] = nv;
    } else {
      a.t[0][at] = t;
    }
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
__global__ void __launch_bounds__(128) momentum_z(Geo g, MomArgs a) {
  const int lane = threadIdx.x & 31;
  // grid (segment, group of 4 rows, x): warp w of the block takes row 4*blockIdx.y + w
  const long long seg = blockIdx.x;
  const long long j = g.gw + (long long)blockIdx.y * 4 + (threadIdx.x >> 5);
  const long long i = g.gw + (long long)blockIdx.z;
  if (j >= g.n1 - g.gw) return;  // whole warps
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
// momentum, precision form: the three advecting directions in one pass
// ---------------------------------------------------------------------------
// A block of TJ + 1 warps marches along x over a chunk of cells.  Warp w
// holds row j = j0 - 1 + w (w = 0 is the row below the block's cells and
// only supplies the y face j0 - 1/2), lane L level k = k0 - 1 + L (lane 0
// only supplies the z face k0 - 1/2): TJ x 31 cells per x step.  Per x
// position f and advected component c:
//   x face  from the thread's register window along x (FP32 first
//           differences + the FP64 values phi[f-HI .. f+R]), the face
//           below kept from the previous step;
//   y face  j+1/2 from the y-z plane of u, v, w at x = f in shared memory
//           (the block's rows and levels with a halo of R); the face j-1/2
//           is the upper face of the warp below, through shared memory;
//   z face  k+1/2 from the plane; the face k-1/2 from lane L-1 by shuffle.
// Every face is evaluated once, every global load is issued one step ahead
// of its use, and each tendency is read and written once per stage with the
// x, y and z terms subtracted in the reference's order.  The advecting
// velocity of each face is the reference's interpolant
// (momentum_advection_weno.h:145-236), in FP64; the WENO runs on FP32 first
// differences (weno_delta) and the flux vel * phi * rho in FP64.
template <int ORDER>
struct MomTile {
  static constexpr int R = St<ORDER>::R;
  static constexpr int NI = ORDER - 1;         // points of the advecting-velocity interpolant
  static constexpr int HI = NI / 2 - 1;        // it reads offsets -HI .. NI-1-HI from the face's lower cell
  static constexpr int TJ = 15;                // cell rows per block (16 warps)
  static constexpr int NW = TJ + 1;            // warps
  static constexpr int NT = NW * 32;           // threads
  static constexpr int NR = TJ + 2 * R;        // plane rows j0-R .. j0+TJ+R-1
  static constexpr int NK = 31 + 2 * R;        // plane levels k0-R .. k0+30+R
  static constexpr int NKP = NK + 1;           // plane row length
  static constexpr int PLANE = NR * NKP;
  static constexpr int NHALO = NR * NK - NT;   // plane entries no thread owns
  static constexpr int HPT = (NHALO + NT - 1) / NT;
  static constexpr int NX = HI + 1 + R;        // FP64 window values phi[f-HI .. f+R]
};

template <int ORDER>
__device__ __forceinline__ double interp_n(const double* p) {  // p[0 .. NI-1]
  if constexpr (ORDER == 5)
    return interp_4<double>(p[0], p[1], p[2], p[3]);
  else
    return interp_6<double>(p[0], p[1], p[2], p[3], p[4], p[5]);
}

// RK: the cell's SSP-RK3 stage (TimeStepping.update_third,
// TimeStepping.pyx:131-151, the same separately rounded operations as
// rk3_kernel) is applied here instead of a separate pass: the u and v
// tendencies are never stored (they start from zero and are complete in
// registers), the w tendency (the thermodynamics' buoyancy) is read, and
// the new values go to a second buffer (neighbouring blocks still read the
// old ones), with the stage-0 copies written here.
// Only interior cells are written; the ghost fill that follows the stage
// overwrites the ghosts.
template <int ORDER, bool RK>
__global__ void __launch_bounds__(MomTile<ORDER>::NT, 1) momentum_tile(Geo g, MomArgs a, int chunk) {
  using T = MomTile<ORDER>;
  constexpr int R = T::R, NI = T::NI, HI = T::HI, NX = T::NX, NKP = T::NKP;
  constexpr int ND = 2 * R - 1;
  __shared__ double plane[3][T::PLANE];
  __shared__ double fy[3][T::NW][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long k0 = g.gw + (long long)blockIdx.x * 31;
  const long long j0 = g.gw + (long long)blockIdx.y * T::TJ;
  const long long k = k0 - 1 + lane, j = j0 - 1 + w;
  const long long c0 = g.gw + (long long)blockIdx.z * chunk;
  const long long c1 = min(c0 + (long long)chunk, g.n0 - g.gw);
  const bool own_ok = j < g.n1 && k < g.n2;  // j, k >= gw - 1 >= 0
  const bool cell = w >= 1 && lane >= 1 && j <= g.n1 - g.gw - 1 && k <= g.n2 - g.gw - 1;
  const int rs = w - 1 + R, ls = lane - 1 + R;  // this thread's plane row and level
  const int me = rs * NKP + ls;
  const int jk = (int)(j * g.js + k);  // offset within an x plane (n1 * n2 < 2^31)

  // halo entries of this thread: plane index and offset within an x plane
  // (-1: none, or outside the arrays; such entries are zero and are read by
  // no cell of the domain)
  int hs[T::HPT], hg[T::HPT];
#pragma unroll
  for (int q = 0; q < T::HPT; ++q) {
    const int h = threadIdx.x + q * T::NT;
    hs[q] = -1;
    hg[q] = -1;
    if (h < T::NHALO) {
      constexpr int A = (R - 1) * T::NK, BW = T::NK - 32, B = T::NW * BW;
      int r, l;
      if (h < A) {
        r = h / T::NK;
        l = h - r * T::NK;
      } else if (h < A + B) {
        const int t = h - A;
        r = R - 1 + t / BW;
        const int m = t - (t / BW) * BW;
        l = (m < R - 1) ? m : m + 32;
      } else {
        const int t = h - A - B;
        r = R - 1 + T::NW + t / T::NK;
        l = t - (t / T::NK) * T::NK;
      }
      hs[q] = r * NKP + l;
      const long long jj = j0 - R + r, kk = k0 - R + l;
      if (jj < g.n1 && kk < g.n2) hg[q] = (int)(jj * g.js + kk);
    }
  }
#pragma unroll
  for (int q = 0; q < T::HPT; ++q)
    if (hs[q] >= 0 && hg[q] < 0)
      for (int c = 0; c < 3; ++c) plane[c][hs[q]] = 0.0;

  const double rho_h = own_ok ? a.rho0_half[k] : 0.0;  // the halo row and level supply faces too
  const double rho_f = own_ok ? a.rho0[k] : 0.0;
  const double rho_h1 = (own_ok && k + 1 < g.n2) ? a.rho0_half[k + 1] : 0.0;
  const double al_h = cell ? a.alpha0_half[k] : 0.0, al_f = cell ? a.alpha0[k] : 0.0;

  // x windows: face f = c0 - 1 reads phi[f-R+1 .. f+R]
  float dl[3][ND];
  double ph[3][NX];  // phi[f-HI .. f+R]
  double nxt[3], hv[3][T::HPT], tcur[3], ccur[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double wv[2 * R];
#pragma unroll
    for (int m = 0; m < 2 * R; ++m) wv[m] = own_ok ? a.vel[c][(c0 - R + m) * g.is + jk] : 0.0;
#pragma unroll
    for (int m = 0; m < ND; ++m) dl[c][m] = (float)(wv[m + 1] - wv[m]);
#pragma unroll
    for (int n = 0; n < NX; ++n) ph[c][n] = wv[R - 1 - HI + n];
    nxt[c] = own_ok ? a.vel[c][(c0 + R) * g.is + jk] : 0.0;
#pragma unroll
    for (int q = 0; q < T::HPT; ++q) hv[c][q] = hg[q] >= 0 ? a.vel[c][(c0 - 1) * g.is + hg[q]] : 0.0;
    tcur[c] = (cell && (!RK || c == 2)) ? a.tend[c][c0 * g.is + jk] : 0.0;
    ccur[c] = (RK && cell && a.stage > 0) ? a.copy[c][c0 * g.is + jk] : 0.0;
  }
  double fxp[3] = {0.0, 0.0, 0.0};

  for (long long f = c0 - 1; f < c1; ++f) {
    // (a) the plane at x = f
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      plane[c][me] = ph[c][HI];
#pragma unroll
      for (int q = 0; q < T::HPT; ++q)
        if (hg[q] >= 0) plane[c][hs[q]] = hv[c][q];
    }
    // (b) loads for the next steps
    double lead[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      lead[c] = nxt[c];
      if (f + 1 < c1) {
#pragma unroll
        for (int q = 0; q < T::HPT; ++q)
          if (hg[q] >= 0) hv[c][q] = a.vel[c][(f + 1) * g.is + hg[q]];
      }
      if (f + 2 < c1 && own_ok) nxt[c] = a.vel[c][(f + 2 + R) * g.is + jk];
    }
    __syncthreads();
    const double* PU = plane[0];
    const double* PV = plane[1];
    const double* PW = plane[2];
    // (c) x faces f+1/2
    double Fx[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double p[NI];
#pragma unroll
      for (int m = 0; m < NI; ++m)
        p[m] = (c == 0) ? ph[0][m] : ((c == 1) ? PU[me + (m - HI) * NKP] : PU[me + (m - HI)]);
      const double va = interp_n<ORDER>(p);
      const bool pos = va >= 0.0;
      const float r = weno_delta<ORDER>(pos, dl[c]);
      Fx[c] = va * ((pos ? ph[c][HI] : ph[c][HI + 1]) + (double)r) * ((c == 2) ? rho_f : rho_h);
      asm volatile("" ::: "memory");  // one component's shared-memory reads at a time: fewer live registers
    }
    // x terms of the tendencies now, so that fewer values live across the barrier
    double tx[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      tx[c] = fma(-((c == 2) ? al_f : al_h) * g.dxi0, Fx[c] - fxp[c], tcur[c]);
      fxp[c] = Fx[c];
    }
    // (d) y faces j+1/2 (to shared memory) and z faces k+1/2
    double dFz[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double* P = plane[c];
      {
        double v[2 * R];
#pragma unroll
        for (int m = 0; m < 2 * R; ++m) v[m] = P[me + (m - R + 1) * NKP];
        float d[ND];
#pragma unroll
        for (int m = 0; m < ND; ++m) d[m] = (float)(v[m + 1] - v[m]);
        double p[NI];
#pragma unroll
        for (int m = 0; m < NI; ++m)
          p[m] = (c == 0) ? ph[1][m] : ((c == 1) ? PV[me + (m - HI) * NKP] : PV[me + (m - HI)]);
        const double va = interp_n<ORDER>(p);
        const bool pos = va >= 0.0;
        const float r = weno_delta<ORDER>(pos, d);
        fy[c][w][lane] = va * ((pos ? v[R - 1] : v[R]) + (double)r) * ((c == 2) ? rho_f : rho_h);
      }
      asm volatile("" ::: "memory");
      {
        double v[2 * R];
#pragma unroll
        for (int m = 0; m < 2 * R; ++m) v[m] = P[me + (m - R + 1)];
        float d[ND];
#pragma unroll
        for (int m = 0; m < ND; ++m) d[m] = (float)(v[m + 1] - v[m]);
        double p[NI];
#pragma unroll
        for (int m = 0; m < NI; ++m)
          p[m] = (c == 0) ? ph[2][m] : ((c == 1) ? PW[me + (m - HI) * NKP] : PW[me + (m - HI)]);
        const double va = interp_n<ORDER>(p);
        const bool pos = va >= 0.0;
        const float r = weno_delta<ORDER>(pos, d);
        const double Fz = va * ((pos ? v[R - 1] : v[R]) + (double)r) * ((c == 2) ? rho_h1 : rho_f);
        dFz[c] = Fz - __shfl_up_sync(0xffffffffu, Fz, 1);
      }
      asm volatile("" ::: "memory");
    }
    __syncthreads();
    // (e) tendencies of the cells at x = f
    const bool upd = cell && f >= c0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long at = f * g.is + jk;
      if (upd) {
        const double al = (c == 2) ? al_f : al_h;
        double t = fma(-al * g.dxi1, fy[c][w][lane] - fy[c][w - 1][lane], tx[c]);
        t = fma(-al * g.dxi2, dFz[c], t);
        if constexpr (RK) {
          const double val = ph[c][HI];
          double nv;
          if (a.stage == 0) {
            a.copy[c][at] = val;
            nv = add_rn(val, mul_rn(t, a.dt));
          } else if (a.stage == 1) {
            nv = add_rn(mul_rn(0.75, ccur[c]), mul_rn(0.25, add_rn(val, mul_rn(t, a.dt))));
          } else {
            nv = add_rn(mul_rn(1.0 / 3.0, ccur[c]), mul_rn(2.0 / 3.0, add_rn(val, mul_rn(t, a.dt))));
          }
          a.vnew[c][at] = nv;
        } else {
          a.tend[c][at] = t;
        }
      }
      if (cell && f + 1 < c1) {
        if (!RK || c == 2) tcur[c] = a.tend[c][at + g.is];
        if (RK && a.stage > 0) ccur[c] = a.copy[c][at + g.is];
      }
    }
    // (f) advance the x windows by one cell
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int m = 0; m < ND - 1; ++m) dl[c][m] = dl[c][m + 1];
      dl[c][ND - 1] = (float)(lead[c] - ph[c][NX - 1]);
#pragma unroll
      for (int n = 0; n < NX - 1; ++n) ph[c][n] = ph[c][n + 1];
      ph[c][NX - 1] = lead[c];
    }
  }
}

constexpr int kChunk = 64;  // cells per marching thread along x / y, at most (march_chunk)

// Cells per block along the marching direction.  The grid runs in waves of
// sms x per_sm resident blocks and a block takes ~chunk + lead steps (lead:
// its window fill), so the chunk in [8, max_chunk] with the fewest
// wave-steps is taken (ties: the longer chunk).  A fixed 64 left the last
// wave nearly empty at 512x512x256 (2520 blocks of the momentum pass on 148
// SMs: 17.03 waves) and most SMs idle on small grids (15 blocks at
// 64x64x75).  The results do not depend on the chunk: a face on a chunk
// boundary is evaluated by both blocks with the same arithmetic.
inline int march_chunk(long long n_march, long long other_blocks, int per_sm, int lead, int max_chunk) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long slots = (long long)sms * (per_sm > 0 ? per_sm : 1);
  int best = max_chunk;
  long long best_cost = -1;
  for (int c = 8; c <= max_chunk; ++c) {
    const long long blocks = other_blocks * ((n_march + c - 1) / c);
    const long long cost = (blocks + slots - 1) / slots * (c + lead);
    if (best_cost < 0 || cost <= best_cost) {
      best_cost = cost;
      best = c;
    }
  }
  return best;
}

template <class K>
inline int resident_blocks(K kernel, int threads, size_t smem = 0) {
  int n = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess || n < 1) n = 1;
  return n;
}

template <int ORDER, bool F32, int NS>
cudaError_t launch_scalar_group(const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                                const double* const vel[3], cudaStream_t st) {
  constexpr int R = St<ORDER>::R;
  const long long nl0 = g.n0 - 2 * g.gw, nl1 = g.n1 - 2 * g.gw, nl2 = g.n2 - 2 * g.gw;
  dim3 blk(32, 4);
  {
    ScalarArgs a = base;
    a.vel = vel[0];
    for (int q = 0; q < NS; ++q) a.flux[q] = flux_dir[0] ? flux_dir[0][q] : nullptr;
    const long long other = (long long)ceil_div(nl2, 32) * ceil_div(nl1, 4);
    if constexpr (F32 && NS == 1) {
      if (a.fused) {
        const int c = march_chunk(nl0, other, resident_blocks(scalar_march_f32<0, ORDER, true>, 128), 2 * R, kChunk);
        scalar_march_f32<0, ORDER, true><<<dim3(ceil_div(nl2, 32), ceil_div(nl1, 4), ceil_div(nl0, c)), blk, 0, st>>>(
            g, a, c);
      } else {
        const int c = march_chunk(nl0, other, resident_blocks(scalar_march_f32<0, ORDER, false>, 128), 2 * R, kChunk);
        scalar_march_f32<0, ORDER, false><<<dim3(ceil_div(nl2, 32), ceil_div(nl1, 4), ceil_div(nl0, c)), blk, 0, st>>>(
            g, a, c);
      }
    } else {
      const int c = march_chunk(nl0, other, resident_blocks(scalar_march<0, ORDER, F32, NS>, 128), 2 * R, kChunk);
      scalar_march<0, ORDER, F32, NS><<<dim3(ceil_div(nl2, 32), ceil_div(nl1, 4), ceil_div(nl0, c)), blk, 0, st>>>(
          g, a, c);
    }
    pb_note_launch();
  }
  {
    ScalarArgs a = base;
    a.vel = vel[1];
    for (int q = 0; q < NS; ++q) a.flux[q] = flux_dir[1] ? flux_dir[1][q] : nullptr;
    const long long other = (long long)ceil_div(nl2, 32) * ceil_div(nl0, 4);
    if constexpr (F32 && NS == 1) {
      const int c = march_chunk(nl1, other, resident_blocks(scalar_march_f32<1, ORDER, false>, 128), 2 * R, kChunk);
      scalar_march_f32<1, ORDER, false><<<dim3(ceil_div(nl2, 32), ceil_div(nl0, 4), ceil_div(nl1, c)), blk, 0, st>>>(
          g, a, c);
    } else {
      const int c = march_chunk(nl1, other, resident_blocks(scalar_march<1, ORDER, F32, NS>, 128), 2 * R, kChunk);
      scalar_march<1, ORDER, F32, NS><<<dim3(ceil_div(nl2, 32), ceil_div(nl0, 4), ceil_div(nl1, c)), blk, 0, st>>>(
          g, a, c);
    }
    pb_note_launch();
  }
  {
    ScalarArgs a = base;
    a.vel = vel[2];
    for (int q = 0; q < NS; ++q) a.flux[q] = flux_dir[2] ? flux_dir[2][q] : nullptr;
    const dim3 grd(ceil_div(nl2, 31), ceil_div(nl1, 4), (unsigned)nl0);
    if constexpr (F32 && NS == 1) {
      if (a.fused)
        scalar_z_f32<ORDER, true><<<grd, 128, 0, st>>>(g, a);
      else
        scalar_z_f32<ORDER, false><<<grd, 128, 0, st>>>(g, a);
    } else {
      scalar_z<ORDER, F32, NS><<<grd, 128, 0, st>>>(g, a);
    }
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
      a.vnew[0] = base.vnew[q];
      a.copy[0] = base.copy[q];
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
  constexpr int R = St<ORDER>::R;
  if constexpr (F32) {  // precision form: one pass for the three advecting directions
    using T = MomTile<ORDER>;
    const int c = march_chunk(nl0, (long long)ceil_div(nl2, 31) * ceil_div(nl1, T::TJ), 1, R + 1, 128);
    momentum_tile<ORDER, false><<<dim3(ceil_div(nl2, 31), ceil_div(nl1, T::TJ), ceil_div(nl0, c)), T::NT, 0,
                                  st>>>(g, a, c);
    pb_note_launch();
    return cudaGetLastError();
  } else {
  const int c0 = march_chunk(nl0, (long long)ceil_div(nl2, 32) * ceil_div(nl1, 4),
                             resident_blocks(momentum_march<0, ORDER, F32>, 128), 2 * R, kChunk);
  momentum_march<0, ORDER, F32><<<dim3(ceil_div(nl2, 32), ceil_div(nl1, 4), ceil_div(nl0, c0)), blk, 0,
                                  st>>>(g, a, c0);
  pb_note_launch();
  const int c1 = march_chunk(nl1, (long long)ceil_div(nl2, 32) * ceil_div(nl0, 4),
                             resident_blocks(momentum_march<1, ORDER, F32>, 128), 2 * R, kChunk);
  momentum_march<1, ORDER, F32><<<dim3(ceil_div(nl2, 32), ceil_div(nl0, 4), ceil_div(nl1, c1)), blk, 0,
                                  st>>>(g, a, c1);
  pb_note_launch();
  momentum_z<ORDER, F32><<<dim3(ceil_div(nl2, 31), ceil_div(nl1, 4), (unsigned)nl0), 128, 0, st>>>(g, a);
  pb_note_launch();
  return cudaGetLastError();
  }
}

// The precision form's momentum pass with the SSP-RK3 stage fused in.
template <int ORDER>
cudaError_t launch_momentum_rk3(const Geo& g, const MomArgs& a, cudaStream_t st) {
  const long long nl0 = g.n0 - 2 * g.gw, nl1 = g.n1 - 2 * g.gw, nl2 = g.n2 - 2 * g.gw;
  using T = MomTile<ORDER>;
  const int c = march_chunk(nl0, (long long)ceil_div(nl2, 31) * ceil_div(nl1, T::TJ), 1, T::R + 1, 128);
  momentum_tile<ORDER, true><<<dim3(ceil_div(nl2, 31), ceil_div(nl1, T::TJ), ceil_div(nl0, c)), T::NT, 0, st>>>(
      g, a, c);
  pb_note_launch();
  return cudaGetLastError();
}

}  // namespace

// FP64 plain form (advection_f64.cu) and FP32 precision form (advection.cu).
cudaError_t scalar_fp64(int order, int ns, const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                        const double* const vel[3], cudaStream_t st);
cudaError_t scalar_fp32(int order, int ns, const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                        const double* const vel[3], cudaStream_t st);
cudaError_t momentum_fp64(int order, const Geo& g, const MomArgs& a, cudaStream_t st);
cudaError_t momentum_fp32(int order, const Geo& g, const MomArgs& a, cudaStream_t st);
cudaError_t momentum_rk3_fp32(int order, const Geo& g, const MomArgs& a, cudaStream_t st);

}  // namespace pbadv
