// Shared device helpers for the DMOLP B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define DMOLP_FULL_MASK 0xffffffffu

namespace dmolp {

constexpr int kWarp = 32;
constexpr int kBlock = 256;                 // threads per block for the warp-per-vertex kernels
constexpr int kWarpsPerBlock = kBlock / kWarp;
constexpr int kRadixBits = 8;               // digit width of the segmented radix select
constexpr int kRadix = 1 << kRadixBits;
constexpr int kMaxIter = 500;               // the reference's max_iter (src/phase2/phase2.cpp:263)
constexpr int kSelHistBuffers = 3;          // the radix select's global histograms rotate over three buffers

// 5-bit bit reversal: the position at which the reference's 32-lane shuffle-down tree prefers a lane
// among equal scores (lane with the smaller reversed index wins).
__device__ __forceinline__ uint32_t brev5(uint32_t x) { return __brev(x) >> 27; }

// Append under a predicate with one atomic per warp; returns the slot (or -1 when !pred).
// Must be called by all threads of the active mask.
__device__ __forceinline__ int warp_append(int *counter, bool pred) {
    const unsigned active = __activemask();
    const unsigned m = __ballot_sync(active, pred);
    if (!m) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(active, base, leader);
    return pred ? base + __popc(m & ((1u << lane) - 1)) : -1;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(DMOLP_FULL_MASK, x, o);
    return x;
}

// Read-only, streaming load of a neighbour id (bypasses L1 allocation; CSR is read once per pass).
__device__ __forceinline__ int32_t ld_stream(const int32_t *p) { return __ldcs(p); }

}  // namespace dmolp
