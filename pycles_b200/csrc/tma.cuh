// Tensor-memory-accelerator (TMA) plane copies and the mbarriers that signal
// their completion, for kernels that stage y-z planes of a field in shared
// memory.
//
// A field is a flat ghosted FP64 array [i][j][k] (k contiguous).  Its tensor
// map describes it as a 3-D tensor {k: nlg2, j: nlg1, i: nlg0} and copies
// boxes of {box_k, box_j, 1} elements: one y-z plane window at one x.  The
// hardware wants the row strides (nlg2 * 8 bytes, nlg1 * nlg2 * 8 bytes) and
// the base address on 16-byte boundaries, the box's inner extent a multiple
// of 16 bytes and the inner start coordinate even (k0 * 8 bytes on a 16-byte
// boundary); callers check pb_tma_plane_ok first.  Elements outside the array
// are filled with zeros, so a box may hang over any edge.
//
// No multicast: each block loads its own planes from this GPU's memory.
// Every wait is bounded; a wait that gives up sets PB_ERR_TIMEOUT in the
// device error word and the kernel carries on (its results are then
// invalid), so no barrier is ever left waiting.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pb_common.cuh"

#define PB_ERR_TIMEOUT 0x8u  // a bounded wait for an asynchronous copy gave up

// Host: tensor map of one field for plane boxes {box_k, box_j, 1}; returns 0
// on success.
int pb_make_plane_map(CUtensorMap* map, const double* field, const Geo& g, int box_k, int box_j);

// Whether the field's layout and address allow TMA plane copies.
inline bool pb_tma_plane_ok(const Geo& g, const void* field) {
  return (g.n2 % 2) == 0 && (reinterpret_cast<uintptr_t>(field) & 15) == 0;
}

namespace pbtma {

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of the given parity; false (and the error bit
// set) if it did not complete.  Each try_wait suspends the thread for a
// hardware time slice, so the bound is of the order of a second.
constexpr int kMaxTries = 1 << 21;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned int* err) {
  for (int t = 0; t < kMaxTries; ++t)
    if (mbar_try_wait(bar, parity)) return true;
  pb_flag_at(err, PB_ERR_TIMEOUT);
  return false;
}

// One box {box_k, box_j, 1} at (k0, j0, i) of the map into shared memory
// (128-byte aligned), completing `bytes` of the barrier's transaction count.
__device__ __forceinline__ void tma_plane(void* dst, const CUtensorMap* map, int k0, int j0, int i, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(k0), "r"(j0), "r"(i), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace pbtma
