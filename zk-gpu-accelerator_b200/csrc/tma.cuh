// tma.cuh — tensor-memory-accelerator (TMA) tile loads and shared-memory
// mbarriers for sm_100a, as inline PTX, and the host-side tensor-map encoder.
//
// A tiled load (cp.async.bulk.tensor) copies a box of a tensor described by a
// 128-byte tensor map from global into shared memory without the issuing
// threads touching the data; the copy reports its bytes to an mbarrier, whose
// phase completes when the expected byte count has arrived. Only this GPU's
// own memory is ever described by these maps, and every load here lands in the
// issuing CTA's own shared memory only.
//
// Alignment rules the callers keep: the global base address 16-byte aligned,
// every stride a multiple of 16 bytes, the box's inner extent a multiple of
// 16 bytes, and the innermost coordinate times the element size a multiple of
// 16 bytes (a misaligned innermost coordinate is not caught by the encoder).
#pragma once
#include <cuda.h>  // CUtensorMap and its enums (types only: the driver is reached through the runtime)
#include <cuda_runtime.h>

#include <cstdint>

namespace zkb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async proxy (the TMA unit).
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy accesses (a TMA load into a buffer that threads wrote).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of transfers for the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
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

// Waits for the phase of `bar` with parity `parity` to complete; gives up and
// returns false after `limit` polls (each poll may suspend the thread for a
// short, hardware-chosen time), so that no wait can hang the kernel.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
  }
  return false;
}

// Tiled loads of one box at the given coordinates (innermost first).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// ---- host ------------------------------------------------------------------

// Encodes a tiled tensor map of 64-bit words: rank 2..5, dims[0] innermost
// (contiguous words), strides_bytes[i] the byte stride of dims[i + 1], box the
// box extent per dimension. No interleave, no swizzle, no out-of-bounds fill.
// Returns a ZKB status (ZKB_ECUDA with a message when the driver refuses).
int encode_tensor_map_u64(CUtensorMap* map, const void* base, int rank, const uint64_t* dims,
                          const uint64_t* strides_bytes, const uint32_t* box);

}  // namespace zkb
