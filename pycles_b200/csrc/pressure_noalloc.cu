// Pressure solve for callers that cannot allocate device memory.
//
// pb_pressure_solve needs a caller-provided workspace.  Some callers cannot
// make one: code running where cudaMalloc is not allowed or not wanted --
// in a loop that cannot afford the device-wide synchronisation a cudaMalloc
// or cudaFree may bring, under an allocator policy that forbids new device
// allocations after start-up, or from a host language binding with no device
// allocator of its own.  This variant keeps
// its scratch in a fixed, file-scope device array instead, so the caller
// passes only the inputs and outputs.
//
// * The array holds PB_PRESSURE_NOALLOC_MAX_BYTES (64 MiB); every GPU that
//   loads the library keeps it until the process exits.  Grids whose scratch
//   (pb_pressure_workspace_bytes) exceeds it are rejected with
//   PB_ERR_WORKSPACE.
// * Host code may not use the array's name as a device address, so the first
//   call on each device (with that device current) takes the address with
//   cudaGetSymbolAddress and fills the grid constants (wave numbers,
//   twiddles).  That set-up is synchronous; it runs again when the grid
//   changes, and then it first waits for the whole device
//   (cudaDeviceSynchronize), so that a solve of the previous grid still
//   queued on any stream finishes with the constants it was launched with.
//   Make the first call for a grid before any stream capture.
// * All calls on a device share the one array and it keeps the last call's
//   contents.  Every scratch word the solve reads is written earlier in the
//   same call, so nothing needs clearing; but calls that overlap on the GPU
//   (different streams, no ordering between them) race on the array.
// * Host threads are serialised: a call holds a lock from its set-up until
//   its kernels are enqueued, so no other thread's re-initialisation can
//   change the constants in between.
#include <mutex>

#include "pb_common.cuh"

static __device__ __align__(256) unsigned char pb_pressure_scratch[PB_PRESSURE_NOALLOC_MAX_BYTES];

namespace {

constexpr int kMaxDevices = 64;

struct NoallocSlot {
  void* addr = nullptr;
  bool have_dims = false;
  pb_dims dims;
};

NoallocSlot g_noalloc[kMaxDevices];
std::mutex g_noalloc_mutex;

bool same_dims(const pb_dims& a, const pb_dims& b) {
  for (int i = 0; i < 3; ++i)
    if (a.n[i] != b.n[i] || a.nlg[i] != b.nlg[i] || a.dx[i] != b.dx[i] || a.indx_lo[i] != b.indx_lo[i])
      return false;
  return a.gw == b.gw;
}

}  // namespace

extern "C" int pb_pressure_solve_noalloc(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                         const double* alpha0, const double* alpha0_half, double* u, double* v,
                                         double* w, double* divergence, double* dynamic_pressure, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w || !divergence || !dynamic_pressure)
    return PB_ERR_ARG;
  const long long need = pb_pressure_workspace_bytes(dims);
  if (need < 0 || need > PB_PRESSURE_NOALLOC_MAX_BYTES) return PB_ERR_WORKSPACE;
  if (!fft_sizes_ok(dims)) return PB_ERR_UNSUPPORTED;
  int dev = 0;
  PB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return PB_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoallocSlot& slot = g_noalloc[dev];
  if (slot.addr == nullptr) {
    void* p = nullptr;
    PB_CUDA_TRY(cudaGetSymbolAddress(&p, pb_pressure_scratch));
    slot.addr = p;
  }
  if (!slot.have_dims || !same_dims(slot.dims, *dims)) {
    // the constants are rewritten by synchronous copies on the legacy
    // stream, which do not wait for non-blocking streams: drain the device
    // first so that no queued solve of the previous grid reads new values
    slot.have_dims = false;
    PB_CUDA_TRY(cudaDeviceSynchronize());
    rc = pb_pressure_init(dims, slot.addr, PB_PRESSURE_NOALLOC_MAX_BYTES);
    if (rc) return rc;
    PB_CUDA_TRY(cudaDeviceSynchronize());
    slot.dims = *dims;
    slot.have_dims = true;
  }
  return pressure_solve_impl(dims, rho0, rho0_half, alpha0, alpha0_half, u, v, w, divergence, dynamic_pressure,
                             static_cast<char*>(slot.addr), PB_FP64, 0, as_stream(stream));
}
