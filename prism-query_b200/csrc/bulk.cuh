// bulk.cuh — the Blackwell bulk-copy engine's L2 prefetch for kernels that
// stream a column once in tiles: a CTA asks the engine to bring a LATER
// tile into L2 (cp.async.bulk.prefetch.L2), so the CTA that takes that tile
// one resident wave later finds its input in L2 instead of waiting on DRAM.
// The prefetch occupies no shared memory, registers or L1 and nothing waits
// on it.
#pragma once

#include "common.cuh"

namespace prism {

// `bytes` (a multiple of 16, src 16-byte aligned) into L2
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

}  // namespace prism
