// Momentum advection, precision form, with the y-z planes of u, v, w staged
// in shared memory by TMA: the same block shape, face evaluation and
// arithmetic as momentum_tile (advection_kernels.cuh), so the results are
// bit for bit the same, but no thread loads or stores a plane.
//
// Each block keeps a ring of D = R + 3 slots, each holding the block's
// window (TJ + 2R rows x NKB levels, NKB = 31 + 2R + 1 rounded up to even
// for the 16-byte alignment of the box's first level) of u, v and w at one
// x.  Slot s % D holds the plane at x = c0 - 1 + s; one elected thread
// issues its three box copies (cp.async.bulk.tensor, completion counted on
// the slot's mbarrier) D steps ahead of its use, and refills a slot right
// after the block barrier that ends the last step reading it.  A step reads
// the plane at its own x (y and z faces, and the x faces' advecting
// velocities) and, for the x window, the thread's own value R + 1 planes
// ahead.  One block barrier per step: the y face fluxes that the warp above
// reads go to one of two buffers by step parity.
#pragma once

#include "advection_kernels.cuh"
#include "tma.cuh"

namespace pbadv {
namespace {

template <int ORDER>
struct MomRing {
  using T = MomTile<ORDER>;
  static constexpr int R = T::R;
  static constexpr int NR = T::NR;                         // rows j0-R .. j0+TJ+R-1
  static constexpr int NKB = (T::NK + 2) / 2 * 2;          // levels: NK + 1, rounded up to even
  static constexpr int PLANE = (NR * NKB * 8 + 127) / 128 * 128 / 8;  // doubles, 128-byte multiple
  static constexpr int SLOT = 3 * PLANE;                   // u, v, w
  static constexpr int D = R + 3;                          // slots
  static constexpr unsigned BOX_BYTES = NR * NKB * 8;      // one component's box
  static constexpr size_t FY = 2 * 3 * T::NW * 32;         // doubles of the y-face buffers
  static constexpr size_t SMEM = (size_t)D * SLOT * 8 + FY * 8 + D * 8 + 128;
};

template <int ORDER, bool RK>
__global__ void __launch_bounds__(MomTile<ORDER>::NT, 1)
    momentum_tma(Geo g, MomArgs a, int chunk, const __grid_constant__ CUtensorMap mu,
                 const __grid_constant__ CUtensorMap mv, const __grid_constant__ CUtensorMap mw) {
  using T = MomTile<ORDER>;
  using Q = MomRing<ORDER>;
  constexpr int R = T::R, NI = T::NI, HI = T::HI, NX = T::NX, NKB = Q::NKB, D = Q::D;
  constexpr int ND = 2 * R - 1;
  extern __shared__ __align__(128) unsigned char smraw[];
  double* ring = reinterpret_cast<double*>(smraw);                        // [D][3][PLANE]
  double* fyb = ring + (size_t)D * Q::SLOT;                                // [2][3][NW][32]
  uint64_t* bar = reinterpret_cast<uint64_t*>(fyb + Q::FY);                // [D]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long k0 = g.gw + (long long)blockIdx.x * 31;
  const long long j0 = g.gw + (long long)blockIdx.y * T::TJ;
  const long long k = k0 - 1 + lane, j = j0 - 1 + w;
  const long long c0 = g.gw + (long long)blockIdx.z * chunk;
  const long long c1 = min(c0 + (long long)chunk, g.n0 - g.gw);
  const bool own_ok = j < g.n1 && k < g.n2;
  const bool cell = w >= 1 && lane >= 1 && j <= g.n1 - g.gw - 1 && k <= g.n2 - g.gw - 1;
  // box origin: first level rounded down to even, the window's rows
  const int zb = (int)((k0 - R) & ~1LL), yb = (int)(j0 - R);
  const int sh = (int)(k0 - R - zb);
  const int me = (w - 1 + R) * NKB + (lane - 1 + R) + sh;  // this thread's cell in a plane
  const int jk = (int)(j * g.js + k);
  const int nsteps = (int)(c1 - c0 + 1);  // x = c0 - 1 .. c1 - 1
  const int nplanes = nsteps + R + 1;     // the last step's lead is R + 1 planes ahead

  auto issue = [&](int s) {  // plane s (x = c0 - 1 + s) into slot s % D
    double* dst = ring + (size_t)(s % D) * Q::SLOT;
    uint64_t* b = bar + (s % D);
    const int x = (int)(c0 - 1 + s);
    pbtma::mbar_arrive_expect_tx(b, 3 * Q::BOX_BYTES);
    pbtma::tma_plane(dst, &mu, zb, yb, x, b);
    pbtma::tma_plane(dst + Q::PLANE, &mv, zb, yb, x, b);
    pbtma::tma_plane(dst + 2 * Q::PLANE, &mw, zb, yb, x, b);
  };
  if (threadIdx.x == 0) {
    for (int q = 0; q < D; ++q) pbtma::mbar_init(bar + q, 1);
    pbtma::mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int s = 0; s < D && s < nplanes; ++s) issue(s);

  const double rho_h = own_ok ? a.rho0_half[k] : 0.0;
  const double rho_f = own_ok ? a.rho0[k] : 0.0;
  const double rho_h1 = (own_ok && k + 1 < g.n2) ? a.rho0_half[k + 1] : 0.0;
  const double al_h = cell ? a.alpha0_half[k] : 0.0, al_f = cell ? a.alpha0[k] : 0.0;

  // x windows: face f = c0 - 1 reads phi[f-R+1 .. f+R]
  float dl[3][ND];
  double ph[3][NX];  // phi[f-HI .. f+R]
  double tcur[3], ccur[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double wv[2 * R];
#pragma unroll
    for (int m = 0; m < 2 * R; ++m) wv[m] = own_ok ? a.vel[c][(c0 - R + m) * g.is + jk] : 0.0;
#pragma unroll
    for (int m = 0; m < ND; ++m) dl[c][m] = (float)(wv[m + 1] - wv[m]);
#pragma unroll
    for (int n = 0; n < NX; ++n) ph[c][n] = wv[R - 1 - HI + n];
    tcur[c] = (cell && (!RK || c == 2)) ? a.tend[c][c0 * g.is + jk] : 0.0;
    ccur[c] = (RK && cell && a.stage > 0) ? a.copy[c][c0 * g.is + jk] : 0.0;
  }
  double fxp[3] = {0.0, 0.0, 0.0};

  for (int s = 0; s < nsteps; ++s) {
    const long long f = c0 - 1 + s;
    const int sl = s + R + 1;  // the plane of the x window's next value
    pbtma::mbar_wait(bar + (s % D), (unsigned)((s / D) & 1), a.err);
    pbtma::mbar_wait(bar + (sl % D), (unsigned)((sl / D) & 1), a.err);
    const double* P0 = ring + (size_t)(s % D) * Q::SLOT;
    const double* PL = ring + (size_t)(sl % D) * Q::SLOT;
    const double* PU = P0;
    const double* PV = P0 + Q::PLANE;
    const double* PW = P0 + 2 * Q::PLANE;
    double* fy = fyb + (s & 1) * (3 * T::NW * 32);
    double lead[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) lead[c] = PL[c * Q::PLANE + me];
    // (c) x faces f+1/2
    double Fx[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double p[NI];
#pragma unroll
      for (int m = 0; m < NI; ++m)
        p[m] = (c == 0) ? ph[0][m] : ((c == 1) ? PU[me + (m - HI) * NKB] : PU[me + (m - HI)]);
      const double va = interp_n<ORDER>(p);
      const bool pos = va >= 0.0;
      const float r = weno_delta<ORDER>(pos, dl[c]);
      Fx[c] = va * ((pos ? ph[c][HI] : ph[c][HI + 1]) + (double)r) * ((c == 2) ? rho_f : rho_h);
      asm volatile("" ::: "memory");
    }
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
      const double* P = P0 + c * Q::PLANE;
      {
        double v[2 * R];
#pragma unroll
        for (int m = 0; m < 2 * R; ++m) v[m] = P[me + (m - R + 1) * NKB];
        float d[ND];
#pragma unroll
        for (int m = 0; m < ND; ++m) d[m] = (float)(v[m + 1] - v[m]);
        double p[NI];
#pragma unroll
        for (int m = 0; m < NI; ++m)
          p[m] = (c == 0) ? ph[1][m] : ((c == 1) ? PV[me + (m - HI) * NKB] : PV[me + (m - HI)]);
        const double va = interp_n<ORDER>(p);
        const bool pos = va >= 0.0;
        const float r = weno_delta<ORDER>(pos, d);
        fy[(c * T::NW + w) * 32 + lane] = va * ((pos ? v[R - 1] : v[R]) + (double)r) * ((c == 2) ? rho_f : rho_h);
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
          p[m] = (c == 0) ? ph[2][m] : ((c == 1) ? PW[me + (m - HI) * NKB] : PW[me + (m - HI)]);
        const double va = interp_n<ORDER>(p);
        const bool pos = va >= 0.0;
        const float r = weno_delta<ORDER>(pos, d);
        const double Fz = va * ((pos ? v[R - 1] : v[R]) + (double)r) * ((c == 2) ? rho_h1 : rho_f);
        dFz[c] = Fz - __shfl_up_sync(0xffffffffu, Fz, 1);
      }
      asm volatile("" ::: "memory");
    }
    __syncthreads();  // every read of plane s is done; the y faces are written
    if (threadIdx.x == 0 && s + D < nplanes) issue(s + D);
    // (e) tendencies of the cells at x = f
    const bool upd = cell && f >= c0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long at = f * g.is + jk;
      if (upd) {
        const double al = (c == 2) ? al_f : al_h;
        double t = fma(-al * g.dxi1, fy[(c * T::NW + w) * 32 + lane] - fy[(c * T::NW + w - 1) * 32 + lane], tx[c]);
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

// Launch of momentum_tma for grids whose fields allow TMA plane copies.
template <int ORDER, bool RK>
cudaError_t launch_momentum_tma(const Geo& g, const MomArgs& a, cudaStream_t st) {
  using T = MomTile<ORDER>;
  using Q = MomRing<ORDER>;
  const long long nl0 = g.n0 - 2 * g.gw, nl1 = g.n1 - 2 * g.gw, nl2 = g.n2 - 2 * g.gw;
  CUtensorMap m[3];
  for (int c = 0; c < 3; ++c)
    if (pb_make_plane_map(&m[c], a.vel[c], g, Q::NKB, Q::NR)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(momentum_tma<ORDER, RK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)Q::SMEM);
  if (e != cudaSuccess) return e;
  const int c = march_chunk(nl0, (long long)ceil_div(nl2, 31) * ceil_div(nl1, T::TJ), 1, T::R + 1, 128);
  momentum_tma<ORDER, RK><<<dim3(ceil_div(nl2, 31), ceil_div(nl1, T::TJ), ceil_div(nl0, c)), T::NT, Q::SMEM,
                            st>>>(g, a, c, m[0], m[1], m[2]);
  pb_note_launch();
  return cudaGetLastError();
}

}  // namespace
}  // namespace pbadv
