// Segmented radix select: per segment, mark the `need` records with the smallest unique 64-bit keys.
//
// MSD radix select, 8-bit digits from the top of the key, all passes in ONE cooperative launch (one block
// per SM, all resident) with one grid barrier per pass:
//   histogram  each block histograms the current digit over ITS OWN active records (a slice of the active
//              list that only it reads and writes) in shared memory, and adds the bins into the pass's
//              global histogram
//   -- grid barrier --
//   decide     every block reads the global histogram of every segment and derives the same digit
//              decisions (the digit d* where the running count crosses `need`) into its shared memory
//   partition  the block's records below d* are selected; records equal to d* stay in its slice for the
//              next digit
// The global histograms rotate over three buffers: the one read in pass p-1 is cleared after the barrier of
// pass p (nobody reads it any more) and is written again only in pass p+2, after the next barrier.  Records
// start in per-block ranges of the record slots, so no block ever needs another's records and no global
// append counter is contended.  Keys are unique, so the last digit always resolves; once no segment needs
// records the kernel ends.  Data blocks hand to one another is read with L1-bypassing loads.  Used for the
// LP boundary window (key = degree or max-degree, then id) and the phase-1 theta selection (key = raw
// degree, then id).
#include "../../include/dmolp_b200.h"
#include "kernels.cuh"
#include "lp_device.cuh"

namespace dmolp {
namespace {

constexpr int kSmemSegMax = 64;  // 64 segments * 256 digits * 4 B = 64 KiB of shared histogram
constexpr int kSelThreads = 1024;
constexpr int kPartU = 2;  // records per thread and step of the partition
constexpr int kSelTail = 4096;  // at most this many records left: block 0 finishes the digits alone
constexpr size_t kTailBytes = (size_t)kSelTail * (sizeof(uint64_t) + 4 * sizeof(int));
constexpr unsigned int kBarrierSpins = 1u << 22;  // a generous bound; then give up and flag

struct SelArgs {
    const int32_t *seg;
    const uint64_t *key;
    const int *n_dev;
    int32_t *act0, *act1;  // active records, by pass parity; block b owns [b*cap, (b+1)*cap) of each
    int nseg, npass, top;
    unsigned int *ghist;   // kSelHistBuffers x nseg x 256
    const int32_t *need;
    uint8_t *sel;
    LpControl *ctl;
    const int *stopped;
    SplitArgs sp;  // used when has_split: selected slots go straight to the LP window
    int has_split;
    int hist_ready;  // the first digit's histogram is already in buffer 0
    int tail_ok;     // shared histograms and the tail region (kTailBytes) are in the dynamic shared memory
};

// Sense-counting grid barrier (all blocks are resident: cooperative launch).  A wait that runs past
// kBarrierSpins sets ctl->wait_timeout and returns, so the kernel always ends.
__device__ __forceinline__ void grid_sync(LpControl *ctl) {
    __threadfence();  // each thread's own global writes and reductions are visible before the arrival
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *gen = &ctl->bar_gen;
        const unsigned int g = *gen;
        __threadfence();
        if (atomicAdd(&ctl->bar_count, 1u) == gridDim.x - 1) {
            atomicExch(&ctl->bar_count, 0u);
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            for (unsigned int i = 0; *gen == g; ++i) {
                if (i >= kBarrierSpins) {
                    atomicExch(&ctl->wait_timeout, 1);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
}

__device__ __forceinline__ void zero_share(unsigned int *buf, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) buf[i] = 0;
}

// Adds a record's bin (or nothing: bin < 0, unique per lane) to the block's histogram, merging lanes of the
// same bin with __match_any_sync.  All 32 lanes call it.
__device__ __forceinline__ void hist_add(int bin, bool use_smem, unsigned int *shist, unsigned int *gh) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __match_any_sync(DMOLP_FULL_MASK, bin);
    if (bin >= 0 && lane == __ffs(m) - 1) {
        if (use_smem) atomicAdd(&shist[bin], (unsigned)__popc(m));
        else atomicAdd(&gh[bin], (unsigned)__popc(m));
    }
}

__device__ __forceinline__ void hist_flush(bool use_smem, const unsigned int *shist, unsigned int *gh, int nbins) {
    if (!use_smem) return;
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x)
        if (shist[i]) atomicAdd(&gh[i], shist[i]);
}

// Digit decisions of one pass, the same in every block that runs them: per segment with records still
// needed, the digit d* where the running count of cnt_at(seg * 256 + digit) crosses the need.  Records
// below d* are selected; at d* either all of them (the need is met) or the segment stays open with the
// rest of its need, *s_open counting open segments and *s_tied the records they keep.  Warps per segment.
template <typename C>
__device__ __forceinline__ void decide_digits(int nseg, int *s_need, int *s_below, int *s_keep, int *s_open,
                                              int *s_tied, C cnt_at) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int p = wid; p < nseg; p += nw) {
        const int nd = s_need[p];
        if (nd <= 0) {
            if (lane == 0) {
                s_below[p] = 0;
                s_keep[p] = -1;
            }
            continue;
        }
        unsigned int c[8];
        unsigned int sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c[j] = cnt_at(p * kRadix + lane * 8 + j);
            sum += c[j];
        }
        unsigned int incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
            if (lane >= o) incl += y;
        }
        const unsigned int total = __shfl_sync(DMOLP_FULL_MASK, incl, 31);
        if ((unsigned int)nd >= total) {  // every active record of the segment is selected
            if (lane == 0) {
                s_below[p] = kRadix;
                s_keep[p] = -1;
                s_need[p] = 0;
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
                    s_below[p] = d + 1;
                    s_keep[p] = -1;
                    s_need[p] = 0;
                } else {
                    s_below[p] = d;
                    s_keep[p] = d;
                    s_need[p] = (int)r;
                    atomicAdd(s_open, 1);
                    atomicAdd(s_tied, (int)c[j]);
                }
            }
            run = inc;
        }
    }
}

// The LP window out of the selection (all 32 lanes call it): U records per lane, take[u] marking the
// selected ones, whose key holds vertex and degree (SplitArgs).  Stamps them, adds their degrees to te and
// appends them to the window and their decision-class lists.  With a staging area (stage: 4 lists x
// kStage ids of this warp in shared memory, scnt: their fill), the appends collect there and a list is
// written out with one atomic when it would overflow (stage_flush does the rest at the end); without it,
// each list's appends of the call are reserved by one atomic (lane j for list j).
constexpr int kStage = 128;
static_assert((size_t)(kSelThreads / 32) * 4 * kStage * sizeof(int) <= kTailBytes, "the staging lives in the tail region");
__device__ __forceinline__ int *list_ptr(const SelArgs &a, int j) { return j == 0 ? a.sp.win : a.sp.dec[j - 1]; }
__device__ __forceinline__ int *list_ctr(const SelArgs &a, int j) { return j == 0 ? a.sp.nwin : &a.sp.ndec[j - 1]; }

__device__ __forceinline__ void stage_flush_list(const SelArgs &a, int j, int *stage, int n) {
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0 && n) base = atomicAdd(list_ctr(a, j), n);
    base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
    int *dst = list_ptr(a, j) + base;
    for (int i = lane; i < n; i += 32) dst[i] = stage[i];
}

// The warp's staged ids of all four lists written out (all lanes).
__device__ __forceinline__ void stage_flush(const SelArgs &a, int *stage, int *scnt) {
    __syncwarp();
    for (int j = 0; j < 4; ++j) stage_flush_list(a, j, stage + j * kStage, scnt[j]);
    __syncwarp();
    if ((threadIdx.x & 31) < 4) scnt[threadIdx.x & 31] = 0;
    __syncwarp();
}

template <int U>
__device__ __forceinline__ void emit_window(const SelArgs &a, const bool *take, const uint64_t *key, const int *p,
                                            uint64_t vmask, unsigned long long &te, int *stage = nullptr,
                                            int *scnt = nullptr) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1;
    int v[U], cls[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        v[u] = 0;
        cls[u] = -1;
        if (take[u]) {
            v[u] = (int)(key[u] & vmask);
            const int dk = (int)(key[u] >> a.sp.ibits);
            const int deg = __ldg(a.sp.RE + p[u]) > 1.0 ? a.sp.maxdeg - dk : dk;
            a.sp.sstamp[v[u]] = a.sp.t;
            te += (unsigned long long)deg;
            cls[u] = dec_class(deg, p[u], a.sp.eff);
        }
    }
    // list j (0 window, 1-3 classes 0-2)
    unsigned ml[4][U];
    int tl[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        tl[j] = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            ml[j][u] = __ballot_sync(DMOLP_FULL_MASK, j == 0 ? take[u] : cls[u] == j - 1);
            tl[j] += __popc(ml[j][u]);
        }
    }
    if (stage) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!tl[j]) continue;  // warp-uniform
            int *sj = stage + j * kStage;
            int c0 = scnt[j];
            if (c0 + tl[j] > kStage) {
                __syncwarp();
                stage_flush_list(a, j, sj, c0);
                c0 = 0;
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const bool mine = j == 0 ? take[u] : cls[u] == j - 1;
                if (mine) sj[c0 + __popc(ml[j][u] & below)] = v[u];
                c0 += __popc(ml[j][u]);
            }
            __syncwarp();
            if (lane == 0) scnt[j] = c0;
            __syncwarp();
        }
        return;
    }
    int cnt = 0;  // lane j: list j's appends of the call
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (lane == j) cnt = tl[j];
    int base = 0;
    if (lane < 4 && cnt) base = atomicAdd(list_ctr(a, lane), cnt);
    int bl[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) bl[j] = __shfl_sync(DMOLP_FULL_MASK, base, j);
#pragma unroll
    for (int u = 0; u < U; ++u) {
        if (take[u]) {
            a.sp.win[bl[0] + __popc(ml[0][u] & below)] = v[u];
            const int c = cls[u];
            const unsigned mc = c == 0 ? ml[1][u] : (c == 1 ? ml[2][u] : ml[3][u]);
            const int bc = c == 0 ? bl[1] : (c == 1 ? bl[2] : bl[3]);
            a.sp.dec[c][bc + __popc(mc & below)] = v[u];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) bl[j] += __popc(ml[j][u]);
    }
}

// Block 0 alone: the remaining digits [q0, npass) of the n <= kSelTail records of `list` (their id, segment
// and key copied to shared memory), with shared histograms, the same decisions and a compaction per pass.
__device__ void select_tail(const SelArgs &a, int q0, const int32_t *list, unsigned int *shist, int *s_need,
                            int *s_below, int *s_keep, uint8_t *region, uint64_t vmask, unsigned long long &te) {
    __shared__ int t_open, t_cnt, t_tied;
    uint64_t *t_key = reinterpret_cast<uint64_t *>(region);
    int *t_r = reinterpret_cast<int *>(t_key + kSelTail);
    int *t_seg = t_r + kSelTail, *t_i0 = t_seg + kSelTail, *t_i1 = t_i0 + kSelTail;
    const int nseg = a.nseg, nbins = nseg * kRadix;
    int n = __ldcg(&a.ctl->sel_tail);  // the pass's tied count, <= kSelTail
    n = n < kSelTail ? n : kSelTail;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int r = __ldcg(list + i);
        t_r[i] = r;
        t_seg[i] = a.seg[r];
        t_key[i] = a.key[r];
        t_i0[i] = i;
    }
    int m = n;
    int *cur = t_i0, *nxt = t_i1;
    for (int q = q0; q < a.npass; ++q) {
        const int shift = a.top - kRadixBits * (q + 1);
        for (int i = threadIdx.x; i < nbins; i += blockDim.x) shist[i] = 0u;
        if (threadIdx.x == 0) {
            t_open = 0;
            t_cnt = 0;
            t_tied = 0;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const int j = cur[i];
            atomicAdd(&shist[t_seg[j] * kRadix + (int)((t_key[j] >> shift) & (kRadix - 1))], 1u);
        }
        __syncthreads();
        decide_digits(nseg, s_need, s_below, s_keep, &t_open, &t_tied, [&](int i) { return shist[i]; });
        __syncthreads();
        const bool more = t_open > 0 && q + 1 < a.npass;
        for (int i0 = 0; i0 < m; i0 += blockDim.x) {
            const int i = i0 + threadIdx.x;
            bool take = false;
            uint64_t key = 0;
            int p = 0;
            if (i < m) {
                const int j = cur[i];
                p = t_seg[j];
                key = t_key[j];
                const int d = (int)((key >> shift) & (kRadix - 1));
                if (d < s_below[p]) {
                    a.sel[t_r[j]] = 1;
                    take = true;
                } else if (more && d == s_keep[p]) {
                    nxt[atomicAdd(&t_cnt, 1)] = j;
                }
            }
            if (a.has_split) emit_window<1>(a, &take, &key, &p, vmask, te);  // all lanes take part
        }
        __syncthreads();
        m = t_cnt;
        int *x = cur;
        cur = nxt;
        nxt = x;
        __syncthreads();
        if (!more) break;
    }
}

__global__ void __launch_bounds__(kSelThreads, 1) k_select(SelArgs a) {
    if (a.stopped && *a.stopped) return;  // the same for every block: all return, no barrier is left open
    extern __shared__ unsigned int smem[];
    const int nseg = a.nseg, nbins = nseg * kRadix;
    const bool use_smem = nseg <= kSmemSegMax;
    unsigned int *shist = smem;
    int *s_need = reinterpret_cast<int *>(smem + (use_smem ? nbins : 0));
    int *s_below = s_need + nseg, *s_keep = s_below + nseg;
    uint8_t *s_tail = reinterpret_cast<uint8_t *>(((uintptr_t)(s_keep + nseg) + 15) & ~(uintptr_t)15);
    __shared__ int s_open, s_cnt, s_tied;
    // window appends staged per warp (4 lists x kStage ids) in the tail region, which the tail uses only
    // after every warp has flushed; without that region the appends go straight out
    __shared__ int s_scnt[kSelThreads / 32][4];
    int *w_stage = nullptr, *w_scnt = nullptr;
    if (a.tail_ok && a.has_split) {
        w_stage = reinterpret_cast<int *>(s_tail) + (threadIdx.x >> 5) * 4 * kStage;
        w_scnt = s_scnt[threadIdx.x >> 5];
        if ((threadIdx.x & 31) < 4) w_scnt[threadIdx.x & 31] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->sel_tail = 0;  // read only after a grid barrier
    const int lane = threadIdx.x & 31;
    for (int p = threadIdx.x; p < nseg; p += blockDim.x) {
        if (a.has_split) {  // need[p] = min(n_p, ceil(e^(-t/5) * n_p))   (gpu_lp_boundary.cu:244, 296-297)
            const int n = a.sp.npart[p];
            const int m = (int)ceil(__dmul_rn(*a.sp.ratio, (double)n));
            s_need[p] = m > n ? n : m;
        } else {
            s_need[p] = a.need[p];
        }
    }
    if (use_smem)
        for (int i = threadIdx.x; i < nbins; i += blockDim.x) shist[i] = 0;
    const int n0 = *a.n_dev;
    const int cap = (n0 + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * cap;
    int my_n = max(0, min(n0, lo + cap) - lo);  // pass 0: record slots [lo, lo + my_n)
    __syncthreads();
    // ---- histogram of the first digit over this block's record slots (unless the records' writer built it) ----
    if (!a.hist_ready) {
        const int shift = a.top - kRadixBits;
        for (int i0 = 0; i0 < my_n; i0 += blockDim.x) {
            const int i = i0 + threadIdx.x;
            int bin = -(lane + 1);  // unique non-bin value for idle lanes and empty slots
            if (i < my_n) {
                const int r = lo + i;
                const int p = a.seg[r];
                const uint64_t key = a.key[r];  // loaded with seg (an empty slot's stale key is not used)
                if (p >= 0 && s_need[p] > 0) bin = p * kRadix + (int)((key >> shift) & (kRadix - 1));
            }
            hist_add(bin, use_smem, shist, a.ghist);
        }
        hist_flush(use_smem, shist, a.ghist, nbins);
    }
    unsigned long long te = 0;  // degrees of the selected vertices (has_split)
    const uint64_t vmask = a.has_split ? (1ull << a.sp.ibits) - 1 : 0;
    int pass = 0;
    for (; pass < a.npass; ++pass) {
        const int shift = a.top - kRadixBits * (pass + 1);
        const int32_t *src = pass ? (((pass - 1) & 1) ? a.act1 : a.act0) + lo : nullptr;
        int32_t *dst = ((pass & 1) ? a.act1 : a.act0) + lo;
        unsigned int *gh = a.ghist + (size_t)(pass % kSelHistBuffers) * nbins;
        unsigned int *gh_next = a.ghist + (size_t)((pass + 1) % kSelHistBuffers) * nbins;
        grid_sync(a.ctl);  // this pass's histogram is complete
        if (pass > 0)      // read by every block in the previous pass, before the barrier just passed
            zero_share(a.ghist + (size_t)((pass - 1) % kSelHistBuffers) * nbins, nbins);
        if (threadIdx.x == 0) {
            s_open = 0;
            s_cnt = 0;
            s_tied = 0;
        }
        if (use_smem)  // the block's histogram of the next digit
            for (int i = threadIdx.x; i < nbins; i += blockDim.x) shist[i] = 0;
        __syncthreads();
        // ---- digit decisions, the same in every block ----
        decide_digits(nseg, s_need, s_below, s_keep, &s_open, &s_tied, [&](int i) { return __ldcg(gh + i); });
        __syncthreads();
        const bool more = s_open > 0 && pass + 1 < a.npass;
        // few records left: this pass's kept records go to one list and block 0 finishes alone
        const bool tail = more && a.tail_ok && s_tied <= kSelTail;
        int32_t *tail_list = (pass & 1) ? a.act1 : a.act0;
        const int shift_next = shift - kRadixBits;
        // ---- partition of this block's records, and the next digit's histogram of the records kept;
        //      kPartU records per thread and step, their loads and their appends' atomics issued together ----
        for (int i0 = 0; i0 < my_n; i0 += kPartU * blockDim.x) {
            bool keep[kPartU], take[kPartU];
            int r[kPartU], bin[kPartU], p[kPartU];
            uint64_t key[kPartU];
#pragma unroll
            for (int u = 0; u < kPartU; ++u) {
                const int i = i0 + u * (int)blockDim.x + (int)threadIdx.x;
                r[u] = i < my_n ? (src ? src[i] : lo + i) : -1;
            }
#pragma unroll
            for (int u = 0; u < kPartU; ++u) {
                p[u] = r[u] >= 0 ? a.seg[r[u]] : -1;
                key[u] = r[u] >= 0 ? a.key[r[u]] : 0;
            }
#pragma unroll
            for (int u = 0; u < kPartU; ++u) {
                keep[u] = take[u] = false;
                bin[u] = -(lane + 1) - 32 * u;  // unique non-bin value per lane and record
                if (p[u] >= 0) {  // skip empty record slots
                    const int d = (int)((key[u] >> shift) & (kRadix - 1));
                    if (d < s_below[p[u]]) {
                        a.sel[r[u]] = 1;
                        take[u] = true;
                    } else if (more && d == s_keep[p[u]]) {
                        keep[u] = true;
                        if (!tail) bin[u] = p[u] * kRadix + (int)((key[u] >> shift_next) & (kRadix - 1));
                    }
                }
            }
            const unsigned below = (1u << lane) - 1;
            {  // kept records to this block's slice (one shared atomic for the step) or to the tail list
                unsigned m[kPartU];
                int tot = 0;
#pragma unroll
                for (int u = 0; u < kPartU; ++u) {
                    m[u] = __ballot_sync(DMOLP_FULL_MASK, keep[u]);
                    tot += __popc(m[u]);
                }
                int base = 0;
                if (tot && lane == 0) base = tail ? atomicAdd(&a.ctl->sel_tail, tot) : atomicAdd(&s_cnt, tot);
                base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
                int32_t *out = tail ? tail_list : dst;
#pragma unroll
                for (int u = 0; u < kPartU; ++u) {
                    if (keep[u]) out[base + __popc(m[u] & below)] = r[u];
                    base += __popc(m[u]);
                }
            }
            if (more && !tail)
#pragma unroll
                for (int u = 0; u < kPartU; ++u) hist_add(bin[u], use_smem, shist, gh_next);
            if (a.has_split) emit_window<kPartU>(a, take, key, p, vmask, te, w_stage, w_scnt);  // all lanes
        }
        if (tail) {
            // the tail list is complete and this pass's histogram read by every block: clear it; block 0
            // runs the remaining digits over the list in shared memory, the others are done
            if (w_stage) stage_flush(a, w_stage, w_scnt);
            __syncthreads();  // the tail region is free
            grid_sync(a.ctl);
            zero_share(gh, nbins);
            if (blockIdx.x == 0) select_tail(a, pass + 1, tail_list, shist, s_need, s_below, s_keep, s_tail, vmask, te);
            break;
        }
        if (more) hist_flush(use_smem, shist, gh_next, nbins);
        __syncthreads();
        my_n = s_cnt;
        __syncthreads();  // every thread has read s_cnt before the next pass resets it
        if (!more) {
            if (w_stage) stage_flush(a, w_stage, w_scnt);
            // the last pass's histogram is still set: clear it once every block has read it
            grid_sync(a.ctl);
            zero_share(gh, nbins);
            break;
        }
    }
    if (a.has_split) {
        te = warp_sum_u64(te);
        if (lane == 0 && te) atomicAdd(a.sp.te, te);
    }
}

}  // namespace

void select_smallest(dmolp_ctx *c, const int32_t *seg, const uint64_t *key, const int *n_dev, int nseg, int keybits,
                     uint8_t *sel, const int *stopped, const SplitArgs *split, bool first_hist_ready) {
    const int npass = (keybits + kRadixBits - 1) / kRadixBits;
    const bool smem_hist = nseg <= kSmemSegMax;
    // shared histograms, needs / decisions, and (with shared histograms) the tail region, 16-byte aligned
    const size_t smem = (smem_hist ? (size_t)nseg * kRadix * sizeof(unsigned int) : 0) + 3 * (size_t)nseg * sizeof(int) +
                        (smem_hist ? 16 + kTailBytes : 0);
    SelArgs a;
    a.seg = seg;
    a.key = key;
    a.n_dev = n_dev;
    a.act0 = c->b.active[0];
    a.act1 = c->b.active[1];
    a.nseg = nseg;
    a.npass = npass;
    a.top = npass * kRadixBits;
    a.ghist = c->b.hist;
    a.need = c->b.need;
    a.sel = sel;
    a.ctl = c->b.ctrl;
    a.stopped = stopped;
    a.has_split = split != nullptr;
    a.hist_ready = first_hist_ready ? 1 : 0;
    a.tail_ok = smem_hist ? 1 : 0;
    if (split) a.sp = *split;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)c->num_sms);  // one block per SM, all resident (cooperative launch)
    cfg.blockDim = dim3(kSelThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_select, a);
    if (e != cudaSuccess && c->launch_error == cudaSuccess) c->launch_error = e;  // reported by the entry point
    c->launches += 1;
}

void select_prepare() {
    cudaFuncSetAttribute(k_select, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kSmemSegMax * kRadix * sizeof(unsigned int) + 3 * DMOLP_MAX_K * sizeof(int) + 16 +
                               kTailBytes));
}

}  // namespace dmolp
