// Segmented radix select: per segment, mark the `need` records with the smallest unique 64-bit keys.
//
// MSD radix select, 8-bit digits from the top of the key.  Each pass: (1) histogram of the current digit
// per segment over the active records (shared-memory histograms when nseg*256 counters fit, global
// otherwise); (2) one block per segment finds the digit d* where the running count crosses `need`;
// (3) records below d* are selected, records equal to d* stay active for the next digit, the rest drop.
// The first pass runs over all records; later passes over a compacted active list, so the work after the
// first digit is proportional to the records tied on the prefix.  Keys are unique, so the last digit
// always resolves.  Used for the LP boundary window (key = degree or max-degree, then id) and for the
// phase-1 theta selection (key = raw degree, then id).
#include "kernels.cuh"

namespace dmolp {
namespace {

constexpr int kSmemSegMax = 64;  // 64 segments * 256 digits * 4 B = 64 KiB of shared histogram

__global__ void k_sel_hist(const int32_t *__restrict__ seg, const uint64_t *__restrict__ key,
                           const int *__restrict__ n_dev, const int32_t *__restrict__ list, const int *__restrict__ nlist,
                           int nseg, int shift, unsigned int *__restrict__ ghist, const int *__restrict__ stopped) {
    if (stopped && *stopped) return;
    extern __shared__ unsigned int shist[];
    const bool use_smem = nseg <= kSmemSegMax;
    const int n = list ? *nlist : *n_dev;
    if (use_smem) {
        for (int i = threadIdx.x; i < nseg * kRadix; i += blockDim.x) shist[i] = 0;
        __syncthreads();
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int r = list ? list[i] : i;
        const int p = seg[r];
        if (p < 0) continue;  // empty record slot
        const int d = (int)((key[r] >> shift) & (kRadix - 1));
        if (use_smem) atomicAdd(&shist[p * kRadix + d], 1u);
        else atomicAdd(&ghist[p * kRadix + d], 1u);
    }
    if (use_smem) {
        __syncthreads();
        for (int i = threadIdx.x; i < nseg * kRadix; i += blockDim.x)
            if (shist[i]) atomicAdd(&ghist[i], shist[i]);
    }
}

// One block (256 threads = one per digit) per segment.
__global__ void k_sel_scan(unsigned int *__restrict__ ghist, int32_t *__restrict__ need,
                           int32_t *__restrict__ sel_below, int32_t *__restrict__ keep_digit,
                           const int *__restrict__ stopped) {
    if (stopped && *stopped) return;
    __shared__ unsigned int warp_tot[kRadix / 32];
    __shared__ int s_dstar;
    const int p = blockIdx.x, d = threadIdx.x, lane = d & 31, w = d >> 5;
    const unsigned int c = ghist[p * kRadix + d];
    ghist[p * kRadix + d] = 0;  // ready for the next pass
    // inclusive scan of c over the 256 digits
    unsigned int x = c;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(DMOLP_FULL_MASK, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    if (d == 0) s_dstar = -1;
    __syncthreads();
    unsigned int before = 0;
    for (int i = 0; i < w; ++i) before += warp_tot[i];
    const unsigned int incl = x + before, excl = incl - c;
    unsigned int total = 0;
    for (int i = 0; i < kRadix / 32; ++i) total += warp_tot[i];
    const int nd = need[p];
    if (nd <= 0) {
        if (d == 0) {
            sel_below[p] = 0;
            keep_digit[p] = -1;
        }
        return;
    }
    if ((unsigned int)nd >= total) {  // every active record of the segment is selected
        if (d == 0) {
            sel_below[p] = kRadix;
            keep_digit[p] = -1;
            need[p] = 0;
        }
        return;
    }
    if (excl < (unsigned int)nd && (unsigned int)nd <= incl) s_dstar = d;
    __syncthreads();
    if (d == s_dstar) {
        const unsigned int r = (unsigned int)nd - excl;
        if (r == c) {
            sel_below[p] = d + 1;
            keep_digit[p] = -1;
            need[p] = 0;
        } else {
            sel_below[p] = d;
            keep_digit[p] = d;
            need[p] = (int)r;
        }
    }
}

__global__ void k_sel_partition(const int32_t *__restrict__ seg, const uint64_t *__restrict__ key,
                                const int *__restrict__ n_dev, const int32_t *__restrict__ list,
                                const int *__restrict__ nlist, int shift, const int32_t *__restrict__ sel_below,
                                const int32_t *__restrict__ keep_digit, uint8_t *__restrict__ sel,
                                int32_t *__restrict__ out, int *__restrict__ nout, const int *__restrict__ stopped) {
    if (stopped && *stopped) return;
    const int n = list ? *nlist : *n_dev;
    const int base = blockIdx.x * blockDim.x;
    for (int i0 = base; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        bool keep = false;
        int r = 0;
        if (i < n) {
            r = list ? list[i] : i;
            const int p = seg[r];
            if (p >= 0) {  // skip empty record slots
                const int d = (int)((key[r] >> shift) & (kRadix - 1));
                if (d < sel_below[p]) sel[r] = 1;
                else keep = (d == keep_digit[p]);
            }
        }
        const int slot = warp_append(nout, keep);
        if (keep) out[slot] = r;
    }
}

__global__ void k_zero_int(int *p) { *p = 0; }

}  // namespace

void select_smallest(dmolp_ctx *c, const int32_t *seg, const uint64_t *key, const int *n_dev, int nseg, int keybits,
                     uint8_t *sel, const int *stopped) {
    const int npass = (keybits + kRadixBits - 1) / kRadixBits;
    const int top = npass * kRadixBits;
    const int grid = c->num_sms * 4;
    const size_t smem = nseg <= kSmemSegMax ? (size_t)nseg * kRadix * sizeof(unsigned int) : 0;
    int *nact = &c->b.cnt->nactive[0];
    for (int pass = 0; pass < npass; ++pass) {
        const int shift = top - kRadixBits * (pass + 1);
        const int32_t *in_list = pass == 0 ? nullptr : c->b.active[(pass - 1) & 1];
        const int *in_n = pass == 0 ? nullptr : nact + ((pass - 1) & 1);
        int32_t *out_list = c->b.active[pass & 1];
        int *out_n = nact + (pass & 1);
        k_sel_hist<<<grid, 512, smem, c->stream>>>(seg, key, n_dev, in_list, in_n, nseg, shift, c->b.hist, stopped);
        k_sel_scan<<<nseg, kRadix, 0, c->stream>>>(c->b.hist, c->b.need, c->b.sel_below, c->b.keep_digit, stopped);
        k_zero_int<<<1, 1, 0, c->stream>>>(out_n);
        k_sel_partition<<<grid, 256, 0, c->stream>>>(seg, key, n_dev, in_list, in_n, shift, c->b.sel_below,
                                                     c->b.keep_digit, sel, out_list, out_n, stopped);
        c->launches += 4;
    }
}

void select_prepare() {
    cudaFuncSetAttribute(k_sel_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kSmemSegMax * kRadix * sizeof(unsigned int)));
}

}  // namespace dmolp
