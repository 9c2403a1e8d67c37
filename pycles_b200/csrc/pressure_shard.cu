// Pressure solve of a domain split across GPUs in x-slabs (full y and z per
// GPU), in phases between which the caller moves data between GPUs.
//
// The reference splits the domain over MPI ranks and moves the spectral
// data between pencils with MPI_Alltoallv (ParallelMPI.pyx:542-1068,
// PressureFFTParallel.pyx:150-219).  Here each GPU holds an x-slab; the
// solve runs as
//
//   divergence       on the x-slab (w minus its horizontal mean), written to
//                    the ghosted divergence field and to a dense array;
//   [all-to-all]     dense x-slab -> z-slab (every column, a range of levels);
//   fft_forward      x- and y-FFT of every level of the z-slab (the same
//                    kernels as the single-GPU solve) -> W[k][j][m];
//   [all-to-all]     W z-slab -> row slab (every level, a range of rows j);
//   fft_columns      the Thomas solve of every (kx, ky) column of the rows;
//   [all-to-all]     back to the z-slab;
//   fft_inverse      inverse y- and x-FFT -> dense pressure of the z-slab;
//   [all-to-all]     back to the x-slab; ghost fill and x-halo exchange;
//   correct          the pressure correction of the x-slab's velocities.
//
// The spectral arithmetic is the single-GPU solve's: the same kernels on the
// same values, so a sharded solve differs from a one-GPU solve only through
// the horizontal mean, whose per-GPU sums (in the reference's order within a
// GPU) are added across GPUs as the reference's MPI_Allreduce adds its
// ranks' sums (ParallelMPI.pyx:229-230).
#include "pb_common.cuh"

namespace {

template <bool PLAIN>
__global__ void __launch_bounds__(256) divergence_kernel(Geo g, PArgs a, double* __restrict__ dense) {
  const long long nz = g.n2 - 2 * g.gw, ny = g.n1 - 2 * g.gw;
  const long long k = g.gw + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long j = g.gw + blockIdx.y, i = g.gw + blockIdx.z;
  if (k >= g.n2 - g.gw) return;
  const long long ijk = i * g.is + j * g.js + k;
  const double d = divergence_at<PLAIN>(g, a, ijk, k);
  a.div[ijk] = d;
  if (dense) dense[((i - g.gw) * ny + (j - g.gw)) * nz + (k - g.gw)] = d;
}

__global__ void __launch_bounds__(256) residual_kernel(Geo g, PArgs a, double* __restrict__ dense) {
  const long long nz = g.n2 - 2 * g.gw, ny = g.n1 - 2 * g.gw;
  const long long k = g.gw + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long j = g.gw + blockIdx.y, i = g.gw + blockIdx.z;
  if (k >= g.n2 - g.gw) return;
  const long long ijk = i * g.is + j * g.js + k;
  dense[((i - g.gw) * ny + (j - g.gw)) * nz + (k - g.gw)] = residual_at(g, a, ijk, k, k - g.gw, nz);
}

dim3 interior_grid(const Geo& g) {
  return dim3(ceil_div(g.n2 - 2 * g.gw, 256), (unsigned)(g.n1 - 2 * g.gw), (unsigned)(g.n0 - 2 * g.gw));
}

bool interior_grid_ok(const pb_dims* d) { return d->n[0] <= 65535 && d->n[1] <= 65535; }

void bind_tables(PArgs& a, const pb_dims* slab, const void* ws) {
  const PLayout L = playout(slab);
  const char* base = static_cast<const char*>(ws);
  a.twx = reinterpret_cast<const double2*>(base + L.twx);
  a.twy = reinterpret_cast<const double2*>(base + L.twy);
  a.twxf = reinterpret_cast<const float2*>(base + L.twxf);
  a.twyf = reinterpret_cast<const float2*>(base + L.twyf);
  a.kx2 = reinterpret_cast<const double*>(base + L.kx2);
  a.ky2 = reinterpret_cast<const double*>(base + L.ky2);
}

}  // namespace

extern "C" long long pb_pressure_spectral_offset(const pb_dims* dims) {
  if (pb_check_dims(dims)) return -1;
  return playout(dims).spec;
}

extern "C" int pb_horizontal_sums(const pb_dims* dims, const double* field, double* sums, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!field || !sums) return PB_ERR_ARG;
  const Geo g = make_geo(dims);
  const size_t sm = 2 * (size_t)kSerialTile * kSerialLd * sizeof(double);
  PB_CUDA_TRY(cudaFuncSetAttribute(hmean_serial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  hmean_serial<<<ceil_div(g.n2, 32), kSerialWarps * 32, sm, as_stream(stream)>>>(g, field, sums, 1.0);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_pressure_divergence(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                      const double* alpha0, const double* alpha0_half, const double* u,
                                      const double* v, const double* w, const double* mean, double* divergence,
                                      double* div_dense, int precision, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w || !mean || !divergence) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  if (!interior_grid_ok(dims)) return PB_ERR_UNSUPPORTED;
  const Geo g = make_geo(dims);
  cudaStream_t st = as_stream(stream);
  PArgs a{};
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.alpha0 = alpha0;
  a.alpha0_half = alpha0_half;
  a.u = const_cast<double*>(u);
  a.v = const_cast<double*>(v);
  a.w = const_cast<double*>(w);
  a.mean = const_cast<double*>(mean);
  a.div = divergence;
  const long long nghost = g.npg - dims->n[0] * dims->n[1] * dims->n[2];
  if (nghost > 0) {
    zero_ghosts<<<stream_blocks(nghost), 256, 0, st>>>(g, divergence, nghost);
    pb_note_launch();
  }
  if (precision == PB_FP64)
    divergence_kernel<true><<<interior_grid(g), 256, 0, st>>>(g, a, div_dense);
  else
    divergence_kernel<false><<<interior_grid(g), 256, 0, st>>>(g, a, div_dense);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_pressure_residual(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                    const double* pressure, const double* divergence, double* resid_dense,
                                    void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !pressure || !divergence || !resid_dense) return PB_ERR_ARG;
  if (!interior_grid_ok(dims)) return PB_ERR_UNSUPPORTED;
  const Geo g = make_geo(dims);
  PArgs a{};
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.p = const_cast<double*>(pressure);
  a.div = const_cast<double*>(divergence);
  residual_kernel<<<interior_grid(g), 256, 0, as_stream(stream)>>>(g, a, resid_dense);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_pressure_fft_forward(const pb_dims* slab, void* workspace, long long workspace_bytes,
                                       const double* src_dense, int precision, void* stream) {
  int rc = pb_check_dims(slab);
  if (rc) return rc;
  if (!workspace || !src_dense) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  const PLayout L = playout(slab);
  if (workspace_bytes < L.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) return PB_ERR_WORKSPACE;
  if (!fft_sizes_ok(slab)) return PB_ERR_UNSUPPORTED;
  const Geo g = make_geo(slab);
  PArgs a{};
  bind_tables(a, slab, workspace);
  a.spec = static_cast<char*>(workspace) + L.spec;
  a.src_dense = src_dense;
  cudaStream_t st = as_stream(stream);
  return precision == PB_FP64 ? fft_forward<double2>(g, a, kSrcDense, st) : fft_forward<float2>(g, a, kSrcDense, st);
}

extern "C" int pb_pressure_fft_columns(const pb_dims* rows, const double* rho0, const double* rho0_half,
                                       const pb_dims* slab, const void* slab_workspace, void* spec, double* scratch,
                                       int j0, int precision, void* stream) {
  int rc = pb_check_dims(rows);
  if (rc) return rc;
  if ((rc = pb_check_dims(slab))) return rc;
  if (!rho0 || !rho0_half || !slab_workspace || !spec || !scratch) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  // the rows' columns are the slab's: the same x extent and horizontal grid
  if (rows->n[0] != slab->n[0] || rows->gw != slab->gw || j0 < 0 || j0 + rows->n[1] > slab->n[1])
    return PB_ERR_ARG;
  const Geo g = make_geo(rows);
  PArgs a{};
  bind_tables(a, slab, slab_workspace);
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.spec = spec;
  a.scr = scratch;
  a.j0 = j0;
  cudaStream_t st = as_stream(stream);
  return precision == PB_FP64 ? fft_columns<double2>(g, a, st) : fft_columns<float2>(g, a, st);
}

extern "C" int pb_pressure_fft_inverse(const pb_dims* slab, void* workspace, long long workspace_bytes,
                                       double* dst_dense, int precision, void* stream) {
  int rc = pb_check_dims(slab);
  if (rc) return rc;
  if (!workspace || !dst_dense) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  const PLayout L = playout(slab);
  if (workspace_bytes < L.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) return PB_ERR_WORKSPACE;
  if (!fft_sizes_ok(slab)) return PB_ERR_UNSUPPORTED;
  const Geo g = make_geo(slab);
  PArgs a{};
  bind_tables(a, slab, workspace);
  a.spec = static_cast<char*>(workspace) + L.spec;
  a.dst_dense = dst_dense;
  cudaStream_t st = as_stream(stream);
  return precision == PB_FP64 ? fft_inverse<double2>(g, a, kDstDense, st) : fft_inverse<float2>(g, a, kDstDense, st);
}

extern "C" int pb_pressure_correct(const pb_dims* dims, const double* pressure, double* u, double* v, double* w,
                                   const double* mean, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!pressure || !u || !v || !w || !mean) return PB_ERR_ARG;
  const Geo g = make_geo(dims);
  correction<<<stream_blocks(g.npg), 256, 0, as_stream(stream)>>>(g, pressure, u, v, w, mean);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
