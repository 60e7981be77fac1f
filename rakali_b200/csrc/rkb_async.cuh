// Asynchronous copies into shared memory (sm_100a): mbarriers, bulk copies
// and TMA tile loads, with bounded waits.
#pragma once
#include <cstdint>

#include "rkb_common.cuh"

namespace rkb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for a phase of `bar` for at most `limit` cycles; warp-uniform result.
// The default limit (kWaitCyclesDefault, ~1 s) polls with try_wait, which
// may suspend the thread in hardware while the copy is in flight.  A shorter
// limit (set from the host to test this error path) polls with the
// non-blocking test_wait and only while the limit has not passed, so the
// limit alone decides when the wait gives up: one shorter than a clock read
// gives up at once.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  bool ok = false;
  if (limit >= kWaitCyclesDefault) {
    ok = mbar_try_wait(bar, parity);
    if (!ok) {
      const long long t0 = clock64();
      while (!(ok = mbar_try_wait(bar, parity)))
        if (clock64() - t0 > limit) break;
    }
  } else {
    const long long t0 = clock64();
    while (clock64() - t0 <= limit)
      if ((ok = mbar_test_wait(bar, parity))) break;
  }
  return __all_sync(0xffffffffu, ok);
}

// Named CTA barrier `id` (1..15) of `count` threads (a multiple of 32), as a
// producer (arrive: does not wait) or a consumer (sync: waits for `count`
// arrivals including its own warp's); orders the producers' prior memory
// accesses before the consumers' later ones.  Warp-uniform.
__device__ __forceinline__ void named_arrive(int id, int count) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// TMA load of one box of a 2D tensor map (a CUtensorMap in parameter, constant
// or global memory) at element coordinates (x, y) into shared memory,
// completing on `bar`.  The box lands row after row, x fastest; elements
// outside the map's extent read as zero.  x times the element size must be a
// multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

}  // namespace rkb
