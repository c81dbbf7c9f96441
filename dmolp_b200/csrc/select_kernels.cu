// Segmented radix select: per segment, mark the `need` records with the smallest unique 64-bit keys.
//
// MSD radix select, 8-bit digits from the top of the key.  A pass is two launches:
//   hist       per-segment histogram of the current digit over the active records (shared-memory
//              histograms when nseg*256 counters fit, global otherwise); the last block to finish (a
//              completion counter) scans every segment's 256 bins, one warp per segment, and finds the digit
//              d* where the running count crosses `need`
//   partition  records below d* are selected, records equal to d* stay active for the next digit
// The first pass runs over all record slots; later passes over the compacted active list, so the work after
// the first digit is proportional to the records tied on the prefix.  Keys are unique, so the last digit
// always resolves; once no segment needs records, later passes return at once.  Used for the LP boundary
// window (key = degree or max-degree, then id) and the phase-1 theta selection (key = raw degree, then id).
#include "kernels.cuh"

namespace dmolp {
namespace {

constexpr int kSmemSegMax = 64;  // 64 segments * 256 digits * 4 B = 64 KiB of shared histogram
constexpr int kHistThreads = 512;

struct SelArgs {
    const int32_t *seg;
    const uint64_t *key;
    const int *n_dev;
    const int32_t *list;  // null in the first pass: all records
    const int *nlist;
    int32_t *out;
    int *nout;
    int nseg, shift, pass;
    unsigned int *ghist;
    int32_t *need, *sel_below, *keep_digit;
    uint8_t *sel;
    LpControl *ctl;
    const int *stopped;
};

__device__ __forceinline__ bool sel_skip(const SelArgs &a) {
    if (a.stopped && *a.stopped) return true;
    return a.pass > 0 && a.ctl->sel_open == 0;
}

// The last block: per segment, the digit where the running count crosses need[p]; clears the histogram.
__device__ void scan_segments(const SelArgs &a) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int open = 0;
    for (int p = w; p < a.nseg; p += nw) {
        unsigned int c[8];
        unsigned int sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            unsigned int *h = a.ghist + p * kRadix + lane * 8 + j;
            c[j] = __ldcg(h);
            *h = 0;
            sum += c[j];
        }
        unsigned int incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
            if (lane >= o) incl += y;
        }
        const unsigned int total = __shfl_sync(DMOLP_FULL_MASK, incl, 31);
        const int nd = a.need[p];
        if (nd <= 0) {
            if (lane == 0) {
                a.sel_below[p] = 0;
                a.keep_digit[p] = -1;
            }
            continue;
        }
        if ((unsigned int)nd >= total) {  // every active record of the segment is selected
            if (lane == 0) {
                a.sel_below[p] = kRadix;
                a.keep_digit[p] = -1;
                a.need[p] = 0;
            }
            continue;
        }
        unsigned int run = incl - sum;  // exclusive prefix of this lane's 8 bins
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const unsigned int excl = run, inc = run + c[j];
            if (excl < (unsigned int)nd && (unsigned int)nd <= inc) {
                const int d = lane * 8 + j;
                const unsigned int r = (unsigned int)nd - excl;
                if (r == c[j]) {
                    a.sel_below[p] = d + 1;
                    a.keep_digit[p] = -1;
                    a.need[p] = 0;
                } else {
                    a.sel_below[p] = d;
                    a.keep_digit[p] = d;
                    a.need[p] = (int)r;
                    ++open;
                }
            }
            run = inc;
        }
    }
    __shared__ int s_open;
    if (threadIdx.x == 0) s_open = 0;
    __syncthreads();
    if (open) atomicAdd(&s_open, open);
    __syncthreads();
    if (threadIdx.x == 0) {
        a.ctl->sel_open = s_open;
        a.ctl->sel_pass = a.pass;
        *a.nout = 0;
    }
}

__global__ void __launch_bounds__(kHistThreads) k_sel_hist(SelArgs a) {
    if (sel_skip(a)) return;
    extern __shared__ unsigned int shist[];
    __shared__ int s_last;
    const bool use_smem = a.nseg <= kSmemSegMax;
    const int n = a.list ? *a.nlist : *a.n_dev;
    if (use_smem) {
        for (int i = threadIdx.x; i < a.nseg * kRadix; i += blockDim.x) shist[i] = 0;
        __syncthreads();
    }
    // Keys crowd into few bins (a digit of small degrees is mostly 0): lanes with the same bin are merged
    // with __match_any_sync and add once.
    const int lane = threadIdx.x & 31;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        int bin = -(lane + 1);  // unique non-bin value for idle lanes and empty slots
        if (i < n) {
            const int r = a.list ? a.list[i] : i;
            const int p = a.seg[r];
            if (p >= 0) bin = p * kRadix + (int)((a.key[r] >> a.shift) & (kRadix - 1));
        }
        const unsigned m = __match_any_sync(DMOLP_FULL_MASK, bin);
        if (bin >= 0 && lane == __ffs(m) - 1) {
            if (use_smem) atomicAdd(&shist[bin], (unsigned)__popc(m));
            else atomicAdd(&a.ghist[bin], (unsigned)__popc(m));
        }
    }
    if (use_smem) {
        __syncthreads();
        for (int i = threadIdx.x; i < a.nseg * kRadix; i += blockDim.x)
            if (shist[i]) atomicAdd(&a.ghist[i], shist[i]);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&a.ctl->sel_done, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) a.ctl->sel_done = 0;
    scan_segments(a);
}

__global__ void k_sel_partition(SelArgs a) {
    if ((a.stopped && *a.stopped) || a.ctl->sel_pass != a.pass) return;
    const int n = a.list ? *a.nlist : *a.n_dev;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        bool keep = false;
        int r = 0;
        if (i < n) {
            r = a.list ? a.list[i] : i;
            const int p = a.seg[r];
            if (p >= 0) {  // skip empty record slots
                const int d = (int)((a.key[r] >> a.shift) & (kRadix - 1));
                if (d < a.sel_below[p]) a.sel[r] = 1;
                else keep = (d == a.keep_digit[p]);
            }
        }
        const int slot = warp_append(a.nout, keep);
        if (keep) a.out[slot] = r;
    }
}

__global__ void k_sel_begin(LpControl *ctl) { ctl->sel_pass = -1; }

}  // namespace

void select_smallest(dmolp_ctx *c, const int32_t *seg, const uint64_t *key, const int *n_dev, int nseg, int keybits,
                     uint8_t *sel, const int *stopped) {
    const int npass = (keybits + kRadixBits - 1) / kRadixBits;
    const int top = npass * kRadixBits;
    const int grid = c->num_sms * 2;
    const size_t smem = nseg <= kSmemSegMax ? (size_t)nseg * kRadix * sizeof(unsigned int) : 0;
    int *nact = &c->b.cnt->nactive[0];
    SelArgs a;
    a.seg = seg;
    a.key = key;
    a.n_dev = n_dev;
    a.nseg = nseg;
    a.ghist = c->b.hist;
    a.need = c->b.need;
    a.sel_below = c->b.sel_below;
    a.keep_digit = c->b.keep_digit;
    a.sel = sel;
    a.ctl = c->b.ctrl;
    a.stopped = stopped;
    k_sel_begin<<<1, 1, 0, c->stream>>>(c->b.ctrl);
    c->launches += 1;
    for (int pass = 0; pass < npass; ++pass) {
        a.pass = pass;
        a.shift = top - kRadixBits * (pass + 1);
        a.list = pass == 0 ? nullptr : c->b.active[(pass - 1) & 1];
        a.nlist = pass == 0 ? nullptr : nact + ((pass - 1) & 1);
        a.out = c->b.active[pass & 1];
        a.nout = nact + (pass & 1);
        k_sel_hist<<<grid, kHistThreads, smem, c->stream>>>(a);
        k_sel_partition<<<grid, 256, 0, c->stream>>>(a);
        c->launches += 2;
    }
}

void select_prepare() {
    cudaFuncSetAttribute(k_sel_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kSmemSegMax * kRadix * sizeof(unsigned int)));
}

}  // namespace dmolp
