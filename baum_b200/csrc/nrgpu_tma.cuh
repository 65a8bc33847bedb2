// nrgpu_tma.cuh -- staging of 3-D field tiles into shared memory with the
// tensor memory accelerator (cp.async.bulk.tensor, sm_90+; used on sm_100a)
// and the mbarriers that signal them.
//
// A tile of TX x TY x TZ inner points is computed by one block of
// TX*TY*TZ threads, one point each.  Every field it reads is brought in as
// one box of (TX+2H) x (TY+2H) x (TZ+2H) points, the tile plus a halo of H
// points per side, by a single TMA load issued by one thread; the copy
// engine fills coordinates outside the array with zeros (those taps are
// never used: the order ladder and the shifted advection stencils keep every
// tap inside the box).  The loads are plain 3-D tiled loads from this GPU's
// own memory; each block loads its own boxes.
//
// Every wait on an mbarrier is bounded: after kTmaWaitCycles clock cycles
// it gives up and returns false, and the caller records the failure in the
// level's status word instead of spinning forever.
#pragma once
#include <cuda.h>
#include "nrgpu_common.cuh"

namespace tma {

// about 2 s at the B200's clock
constexpr long long kTmaWaitCycles = 4000000000LL;

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async proxy (the copy engine)
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces the bytes the pending copies will deliver
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// wait until the phase with the given parity has completed; false when the
// wait ran out of time
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kTmaWaitCycles) return false;
  return true;
}

// 3-D tiled load of one box into shared memory, completing on bar
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace tma
