// TMA (cp.async.bulk.tensor) tile loads completed on shared-memory mbarriers, sm_100a.
// Loads are plain: each CTA fetches its own boxes from this GPU's memory.  Every wait is bounded: after kWaitPolls
// polls the waiter gives up and the caller reports a timeout instead of hanging.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ausm {

constexpr unsigned kWaitPolls = 1u << 16;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// orders this thread's earlier generic-proxy shared-memory accesses before later
// async-proxy (TMA) accesses
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 2-D tiled load of the box at element coordinates (x, y) of the tensor map into dst.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// Programmatic dependent launch: a kernel launched with the programmatic-serialization
// attribute may start while the previous kernel in its stream is still running.  It
// reads nothing that kernel (or a later-finishing one before it) writes until
// grid_dep_wait() returns; grid_dep_launch() lets the next such kernel start early.
// Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity: at most `polls` polls (none for
// polls = 0); false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned polls = kWaitPolls) {
  for (unsigned it = 0; it < polls; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Polls of a tile's first wait for each of its boxes (kWaitPolls).  Tests lower it
// (ausm_debug_set_wait_polls, to 0: the wait gives up at once) to drive the timeout
// path without a fault: the tile then reports AUSM_ERR_TIMEOUT and still waits, with
// the full bound, for its copies to land before the CTA exits.  One copy per
// translation unit that launches TMA stage kernels, each with its own setter.
static __constant__ unsigned c_wait_polls = kWaitPolls;

}  // namespace ausm
