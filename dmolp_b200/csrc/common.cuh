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

// Degree bins of the LP window selection (k <= kDegSelMaxK).  A record's degree d falls in a superbin s
// and a fine bin f inside it: s = d for d < 64 (one degree each); 64 + (d - 64) / 64 for d < 2048 (64
// degrees, f = the offset); for d >= 2048 one superbin per octave, s = 95 + floor(log2 d) - 11, and f = the
// six bits of d below its leading one (1/64 octave).  Ascending (s, f) is ascending degree; records that share
// a fine bin below 2048 share their degree.
constexpr int kDegSelMaxK = 64;
constexpr int kDsSingle = 64;                         // superbins of one degree
constexpr int kDsCoarse0 = kDsSingle + 31;            // first superbin of degrees >= 2048
constexpr int kDsBins = kDsCoarse0 + 20;              // superbins per label (degrees < 2^31)
constexpr int kDsFine = 64;                           // fine bins per superbin
constexpr int kDsExactMax = 2048;                     // degrees below this have a fine bin of their own

__device__ __forceinline__ int2 dsel_bin(int d) {
    if (d < kDsSingle) return make_int2(d, 0);
    if (d < kDsExactMax) return make_int2(kDsSingle + ((d - kDsSingle) >> 6), (d - kDsSingle) & 63);
    const int j = 31 - __clz(d);
    return make_int2(kDsCoarse0 + (j - 11), (d >> (j - 6)) & 63);
}

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

// One value per thread summed over the block; thread 0 adds the sum to *dst.  One atomic per block instead
// of one per warp: atomics on one address queue at one L2 slice, and the warps of a kernel finish together.
// Every thread of the block must call it (two block barriers); blockDim.x <= 1024.
template <typename T>
__device__ __forceinline__ void block_atomic_add(unsigned long long v, T *dst) {
    __shared__ unsigned long long s_w[32];
    v = warp_sum_u64(v);
    __syncthreads();  // s_w is free (an earlier call's sums were read)
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_w[w];
        if (t) atomicAdd(dst, (T)t);
    }
}

// Read-only, streaming load of a neighbour id (bypasses L1 allocation; CSR is read once per pass).
__device__ __forceinline__ int32_t ld_stream(const int32_t *p) { return __ldcs(p); }

}  // namespace dmolp
