// Tensor-memory-access (TMA) and mbarrier helpers for sm_100a, written as
// inline PTX, plus the host-side encoder of tiled tensor maps.
//
// Only plain tiled loads global -> shared of this GPU's own buffers are used
// (cp.async.bulk.tensor ... .tile.mbarrier::complete_tx::bytes, no cluster
// multicast); completion is signalled on a shared-memory mbarrier whose
// transaction count the issuing thread sets to the bytes of the boxes it
// requests (out-of-bounds box elements are zero-filled and still counted).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace tb {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Make the initialised barriers visible to the async proxy (the TMA unit).
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same buffers.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also adds `bytes` to the barrier's expected transactions.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// One plain arrival (release semantics at CTA scope).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase with the given parity to complete.  Bounded: after
// `limit` unsuccessful polls (each try_wait itself suspends for a
// hardware-defined time) the wait gives up and returns false, so a lost
// transfer ends the kernel with an error instead of hanging the GPU.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Bring a tensor map (a kernel parameter) into the TMA descriptor cache
// before the first load that uses it.
__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// 3-D tiled TMA load of the box at (x, y, z) of `map` into shared memory.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// Acquire / release accesses of a flag word in global memory (inter-CTA
// hand-offs inside one launch).
__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------- host

// Encode a 3-D FP32 tiled tensor map over a pitched array: dims (nx, ny, nz)
// elements, rows `pitch` floats apart (pitch * 4 must be a multiple of 16),
// planes ny * pitch floats apart; box (bx, by, 1).  Elements outside the dims
// read as zero.  Returns false (status recorded) on failure.
bool encode_map_3d(CUtensorMap *map, const float *base, int64_t nx, int64_t ny, int64_t nz,
                   int64_t pitch, int bx, int by);

}  // namespace tb
