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
    unsigned int polls;  // grid barrier wait limit
};

// Sense-counting grid barrier (all blocks are resident: cooperative launch).  Returns false when the wait
// ran past `polls` polls of the generation word, or another block's barrier already gave up: then
// ctl->wait_timeout holds 1 + the id of the first barrier that gave up, the loop is stopped, and the caller's
// block leaves the kernel at once (every block that waits at a later barrier leaves too), so the kernel
// always ends; the host reports the timeout and clears the barrier state.
__device__ __forceinline__ bool grid_sync(LpControl *ctl, unsigned int polls, int id) {
    __shared__ int s_pass;
    __threadfence();  // each thread's own global writes and reductions are visible before the arrival
    __syncthreads();
    if (threadIdx.x == 0) {
        int pass = 1;
        volatile unsigned int *gen = &ctl->bar_gen;
        volatile int *gave_up = &ctl->wait_timeout;
        const unsigned int g = *gen;
        __threadfence();
        if (atomicAdd(&ctl->bar_count, 1u) == gridDim.x - 1) {
            atomicExch(&ctl->bar_count, 0u);
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            for (unsigned int i = 0; *gen == g; ++i) {
                if (i >= polls || *gave_up) {
                    atomicCAS(&ctl->wait_timeout, 0, 1 + id);
                    atomicExch(&ctl->stopped, 1);  // the iteration's later kernels return at once
                    pass = 0;
                    break;
                }
            }
        }
        __threadfence();
        s_pass = pass;
    }
    __syncthreads();
    return s_pass != 0;
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
__device__ __forceinline__ int *list_ptr(const SplitArgs &sp, int j) { return j == 0 ? sp.win : sp.dec[j - 1]; }
__device__ __forceinline__ int *list_ctr(const SplitArgs &sp, int j) { return j == 0 ? sp.nwin : &sp.ndec[j - 1]; }

__device__ __forceinline__ void stage_flush_list(const SplitArgs &sp, int j, int *stage, int n) {
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0 && n) base = atomicAdd(list_ctr(sp, j), n);
    base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
    int *dst = list_ptr(sp, j) + base;
    for (int i = lane; i < n; i += 32) dst[i] = stage[i];
}

// The warp's staged ids of all four lists written out (all lanes).
__device__ __forceinline__ void stage_flush(const SplitArgs &sp, int *stage, int *scnt) {
    __syncwarp();
    for (int j = 0; j < 4; ++j) stage_flush_list(sp, j, stage + j * kStage, scnt[j]);
    __syncwarp();
    if ((threadIdx.x & 31) < 4) scnt[threadIdx.x & 31] = 0;
    __syncwarp();
}

template <int U>
__device__ __forceinline__ void emit_window(const SplitArgs &sp, const bool *take, const uint64_t *key, const int *p,
                                            uint64_t vmask, unsigned long long &te, unsigned long long &ws,
                                            int *stage = nullptr,
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
            const int dk = (int)(key[u] >> sp.ibits);
            const int deg = __ldg(sp.RE + p[u]) > 1.0 ? sp.maxdeg - dk : dk;
            sp.sstamp[v[u]] = sp.t;
            te += (unsigned long long)deg;
            ws += window_mix(v[u]);
            cls[u] = dec_class(deg, p[u], sp.eff);
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
                stage_flush_list(sp, j, sj, c0);
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
    if (lane < 4 && cnt) base = atomicAdd(list_ctr(sp, lane), cnt);
    int bl[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) bl[j] = __shfl_sync(DMOLP_FULL_MASK, base, j);
#pragma unroll
    for (int u = 0; u < U; ++u) {
        if (take[u]) {
            sp.win[bl[0] + __popc(ml[0][u] & below)] = v[u];
            const int c = cls[u];
            const unsigned mc = c == 0 ? ml[1][u] : (c == 1 ? ml[2][u] : ml[3][u]);
            const int bc = c == 0 ? bl[1] : (c == 1 ? bl[2] : bl[3]);
            sp.dec[c][bc + __popc(mc & below)] = v[u];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) bl[j] += __popc(ml[j][u]);
    }
}

// Block 0 alone: the remaining digits [q0, npass) of the n <= kSelTail records of `list` (their id, segment
// and key copied to shared memory), with shared histograms, the same decisions and a compaction per pass.
__device__ void select_tail(const SelArgs &a, int q0, const int32_t *list, unsigned int *shist, int *s_need,
                            int *s_below, int *s_keep, uint8_t *region, uint64_t vmask, unsigned long long &te,
                            unsigned long long &ws) {
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
            if (a.has_split) emit_window<1>(a.sp, &take, &key, &p, vmask, te, ws);  // all lanes take part
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
    unsigned long long te = 0, ws = 0;  // degrees and window_mix sum of the selected vertices (has_split)
    const uint64_t vmask = a.has_split ? (1ull << a.sp.ibits) - 1 : 0;
    int pass = 0;
    for (; pass < a.npass; ++pass) {
        const int shift = a.top - kRadixBits * (pass + 1);
        const int32_t *src = pass ? (((pass - 1) & 1) ? a.act1 : a.act0) + lo : nullptr;
        int32_t *dst = ((pass & 1) ? a.act1 : a.act0) + lo;
        unsigned int *gh = a.ghist + (size_t)(pass % kSelHistBuffers) * nbins;
        unsigned int *gh_next = a.ghist + (size_t)((pass + 1) % kSelHistBuffers) * nbins;
        if (!grid_sync(a.ctl, a.polls, 1 + pass)) return;  // this pass's histogram is complete
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
            if (a.has_split) emit_window<kPartU>(a.sp, take, key, p, vmask, te, ws, w_stage, w_scnt);  // all lanes
        }
        if (tail) {
            // the tail list is complete and this pass's histogram read by every block: clear it; block 0
            // runs the remaining digits over the list in shared memory, the others are done
            if (w_stage) stage_flush(a.sp, w_stage, w_scnt);
            __syncthreads();  // the tail region is free
            if (!grid_sync(a.ctl, a.polls, 9)) return;
            zero_share(gh, nbins);
            if (blockIdx.x == 0) select_tail(a, pass + 1, tail_list, shist, s_need, s_below, s_keep, s_tail, vmask, te, ws);
            break;
        }
        if (more) hist_flush(use_smem, shist, gh_next, nbins);
        __syncthreads();
        my_n = s_cnt;
        __syncthreads();  // every thread has read s_cnt before the next pass resets it
        if (!more) {
            if (w_stage) stage_flush(a.sp, w_stage, w_scnt);
            // the last pass's histogram is still set: clear it once every block has read it
            if (!grid_sync(a.ctl, a.polls, 10)) return;
            zero_share(gh, nbins);
            break;
        }
    }
    if (a.has_split) {
        te = warp_sum_u64(te);
        ws = warp_sum_u64(ws);
        if (lane == 0 && te) atomicAdd(a.sp.te, te);
        if (lane == 0 && ws) atomicAdd(a.sp.wsum, ws);
    }
}

// ------------------------------------------------------------------------------------------------------
// Degree-bin window selection (LP, at most kDegSelMaxK labels).
//
// Per label p the window takes need_p = min(n_p, ceil(e^(-t/5) n_p)) of the label's n_p boundary records:
// the smallest degrees first, or the largest first when RE[p] > 1, ids ascending among equal degrees
// (gpu_lp_boundary.cu:244, 282-300).  The boundary test has counted every label's records per degree
// superbin (dsel_bin, Buffers::dsup).  One cooperative launch, one block per SM, ONE grid barrier:
//   0. every block finds, per label, the superbin where the running count in the label's order reaches
//      need_p; records of the superbins before it are taken, the rest of that superbin is partial;
//   1. each warp walks its own contiguous range of record slots in order: taken records go to the window;
//      records of a partial superbin of degree < 2048 go to the warp's list (label and key, in slot order)
//      and into the block's fine-bin counts (stored per block in dcntb, summed into dfine); the keys of those
//      of degree >= 2048 to their label's segment of a tail list (segments sized by the superbin counts) and
//      into dfine;
//   -- grid barrier --
//   2. every block finds, per label, the fine bin of the partial superbin where the count reaches the rest
//      of the need.  Below degree 2048 a fine bin is a single degree, and record slots hold the vertices of
//      one degree in ascending id order (slots follow the degree classes, ids ascending inside a class), so
//      a record of the partial fine bin is taken when fewer than the rest of the need precede it: in the
//      blocks before this one (dcntb), in the warps before this one, in its warp's list before it.  Above,
//      block p sorts label p's tail keys of the partial fine bin (degree, then id) and takes the first ones.
// ------------------------------------------------------------------------------------------------------
constexpr int kDsThreads = 1024;
constexpr int kDsWarps = kDsThreads / 32;
constexpr int kDsU = 2;          // record slots per lane and step of the first walk
constexpr int kDsTieCap = 4096;  // a label's coarse tied records ranked in shared memory (more: from global)

struct DegSelArgs {
    const int32_t *seg;        // bown: label of a boundary record, -1 for an empty slot
    const uint64_t *key;       // bkey: (dk << ibits) | v
    const int *n_dev;          // record slots
    int32_t *lists;            // the warps' lists of partial-superbin records below degree 2048: labels ...
    uint64_t *lkeys;           // ... and keys (the same positions)
    uint64_t *tail;            // keys of partial-superbin records of degree >= 2048, one segment per label
    int *tcnt, *tcnt_next;     // [nseg] tail records per label (this iteration / the next one's, cleared here)
    unsigned int *dsup;        // [nseg * kDsBins] from the boundary test; cleared here after the barrier
    unsigned int *dfine;       // [nseg * kDsFine] fine counts of this iteration's partial superbins
    unsigned int *dfine_next;  // the other parity's buffer, cleared here for the next iteration
    unsigned int *dcntb;       // [gridDim.x * nseg * kDsFine]
    int nseg;
    unsigned int polls;
    LpControl *ctl;
    const int *stopped;
    SplitArgs sp;
};

// Dynamic shared memory of k_select_deg for nseg labels.
__host__ __device__ constexpr size_t ds_smem_bytes(int nseg) {
    return (size_t)kDsTieCap * 8 + (size_t)10 * nseg * 4 + (size_t)nseg * kDsFine * 4 +
           (size_t)2 * kDsWarps * nseg * 4 + (size_t)kDsWarps * 4 * kStage * 4;
}

// Order position of superbin / fine bin x in a label's order (descending degree when dir).
__device__ __forceinline__ int ds_ord(int x, int n, int dir) { return dir ? n - 1 - x : x; }

// Running-count crossing over `per` consecutive order positions per lane (all lanes): the position where
// the count reaches need (0 < need < total), the records before it and its count.
template <int PER, typename C>
__device__ __forceinline__ void ds_cross(int need, C cnt_at, int lane, int &pos, int &before, int &count) {
    unsigned int c[PER], sum = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        c[j] = cnt_at(lane * PER + j);
        sum += c[j];
    }
    unsigned int incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
        if (lane >= o) incl += y;
    }
    unsigned int run = incl - sum;
    int fpos = -1, fbefore = 0, fcount = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        if (run < (unsigned)need && (unsigned)need <= run + c[j]) {
            fpos = lane * PER + j;
            fbefore = (int)run;
            fcount = (int)c[j];
        }
        run += c[j];
    }
    const unsigned m = __ballot_sync(DMOLP_FULL_MASK, fpos >= 0);
    const int src = m ? __ffs(m) - 1 : 0;
    pos = __shfl_sync(DMOLP_FULL_MASK, fpos, src);
    before = __shfl_sync(DMOLP_FULL_MASK, fbefore, src);
    count = __shfl_sync(DMOLP_FULL_MASK, fcount, src);
}

__global__ void __launch_bounds__(kDsThreads, 1) k_select_deg(DegSelArgs a) {
    if (a.stopped && *a.stopped) return;  // the same for every block: all return, no barrier is left open
    extern __shared__ __align__(16) unsigned char ds_smem[];
    const int nseg = a.nseg, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1;
    uint64_t *s_tkey = reinterpret_cast<uint64_t *>(ds_smem);       // [kDsTieCap] keys of this block's coarse ties
    int *s_otake = reinterpret_cast<int *>(s_tkey + kDsTieCap);     // [nseg] superbin order positions below this are taken
    int *s_opart = s_otake + nseg;       // [nseg] order position of the partial superbin, -1 none
    int *s_rem = s_opart + nseg;         // [nseg] records still needed from the partial superbin
    int *s_dir = s_rem + nseg;           // [nseg] 1: largest degree first (RE > 1)
    int *s_kind = s_dir + nseg;          // [nseg] partial superbin: 0 none, 1 one degree, 2 < 2048, 3 coarse
    int *s_toff = s_kind + nseg;         // [nseg] the label's segment of the tail list
    int *s_ftake = s_toff + nseg;        // [nseg] fine order positions below this are taken
    int *s_fpart = s_ftake + nseg;       // [nseg] fine order position of the partial fine bin, -1 none
    int *s_frem = s_fpart + nseg;        // [nseg] records still needed from the partial fine bin
    int *s_pre = s_frem + nseg;          // [nseg] the partial fine bin's records in the blocks before this one
    unsigned int *s_f = reinterpret_cast<unsigned int *>(s_pre + nseg);  // [nseg * kDsFine] this block's
    int *s_wc = reinterpret_cast<int *>(s_f + nseg * kDsFine);  // [kDsWarps * nseg] partial fine bin per warp
    int *s_wrun = s_wc + kDsWarps * nseg;                       // [kDsWarps * nseg] running rank per warp
    int *s_stage = s_wrun + kDsWarps * nseg;                    // [kDsWarps * 4 * kStage] window appends
    __shared__ int s_scnt[kDsWarps][4];
    __shared__ int s_ntie, s_walk1, s_bstar, s_before;
    __shared__ unsigned int s_wsum[kDsWarps];
    __shared__ int s_soff[kDsWarps][4], s_sbase[4];
    __shared__ unsigned long long s_te[kDsWarps], s_ws[kDsWarps];
    int *w_stage = s_stage + wid * 4 * kStage, *w_scnt = s_scnt[wid];
    if (lane < 4) w_scnt[lane] = 0;
    for (int i = threadIdx.x; i < nseg * kDsFine; i += blockDim.x) s_f[i] = 0u;
    for (int i = threadIdx.x; i < kDsWarps * nseg; i += blockDim.x) s_wc[i] = 0;
    if (threadIdx.x == 0) {
        s_ntie = 0;
        s_walk1 = 0;
    }
    // the other parity's fine and tail counts were used by the previous iteration's selection: clear them
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nseg * kDsFine; i += gridDim.x * blockDim.x)
        a.dfine_next[i] = 0u;
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < nseg; i += blockDim.x) a.tcnt_next[i] = 0;
    // ---- 0. per label: the superbin where the need is reached ----
    const double ratio = *a.sp.ratio;
    for (int p = wid; p < nseg; p += kDsWarps) {
        const int n = a.sp.npart[p];
        const int m = (int)ceil(__dmul_rn(ratio, (double)n));  // ceil(e^(-t/5) n), gpu_lp_boundary.cu:296-297
        const int need = m > n ? n : m;
        const int dir = __ldg(a.sp.RE + p) > 1.0 ? 1 : 0;
        int take = need >= n ? kDsBins : 0, part = -1, rem = 0, kind = 0, tsize = 0;
        if (need > 0 && need < n) {
            int pos, before, count;
            ds_cross<(kDsBins + 31) / 32>(need, [&](int o) {
                return o < kDsBins ? __ldcg(a.dsup + p * kDsBins + ds_ord(o, kDsBins, dir)) : 0u;
            }, lane, pos, before, count);
            if (pos < 0) {  // inconsistent counts (never expected): take nothing more
                take = 0;
            } else if (need - before == count) {
                take = pos + 1;
            } else {
                take = pos;
                part = pos;
                rem = need - before;
                const int sb = ds_ord(pos, kDsBins, dir);
                kind = sb < kDsSingle ? 1 : (sb < kDsCoarse0 ? 2 : 3);
                if (kind == 3) tsize = count;
            }
        }
        if (lane == 0) {
            s_otake[p] = take;
            s_opart[p] = part;
            s_rem[p] = rem;
            s_dir[p] = dir;
            s_kind[p] = kind;
            s_toff[p] = tsize;  // the segment sizes, turned into offsets below
        }
    }
    __syncthreads();
    if (wid == 0) {  // exclusive prefix of the tail segment sizes (nseg <= 64: two per lane)
        const int x0 = lane < nseg ? s_toff[lane] : 0, x1 = lane + 32 < nseg ? s_toff[lane + 32] : 0;
        int incl = x0 + x1;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - x0 - x1;
        __syncwarp();
        if (lane < nseg) s_toff[lane] = excl;
        if (lane + 32 < nseg) s_toff[lane + 32] = excl + x0;
    }
    __syncthreads();
    // ---- 1. each warp walks its own contiguous range of record slots ----
    const int n0 = *a.n_dev;
    const int cap = (n0 + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * cap;
    const int my_n = max(0, min(n0, lo + cap) - lo);
    const int wcap = (my_n + kDsWarps - 1) / kDsWarps;
    const int wlo = lo + min(my_n, wid * wcap), whi = lo + min(my_n, (wid + 1) * wcap);
    int32_t *wlist = a.lists + wlo;  // at most whi - wlo entries: label, and the key in lkeys
    uint64_t *wkey = a.lkeys + wlo;
    int wl = 0;                      // the warp's list length (warp-uniform)
    const int ibits = a.sp.ibits, maxdeg = a.sp.maxdeg;
    const uint64_t vmask = (1ull << ibits) - 1;
    unsigned long long te = 0, ws = 0;
    auto bins_of = [&](uint64_t key, int p, int &o, int &fo) {
        const int dir = s_dir[p];
        const int dk = (int)(key >> ibits);
        const int2 bf = dsel_bin(dir ? maxdeg - dk : dk);
        o = ds_ord(bf.x, kDsBins, dir);
        fo = ds_ord(bf.y, kDsFine, dir);
        return bf;
    };
    // the next step's slots are loaded while this step's are processed
    int np_[kDsU];
    uint64_t nkey[kDsU];
#pragma unroll
    for (int u = 0; u < kDsU; ++u) {
        const int r = wlo + u * 32 + lane;
        np_[u] = r < whi ? a.seg[r] : -1;
        nkey[u] = r < whi ? a.key[r] : 0;
    }
    for (int r0 = wlo; r0 < whi; r0 += 32 * kDsU) {
        int p[kDsU], fb[kDsU];
        uint64_t key[kDsU];
        bool take[kDsU], part[kDsU];
#pragma unroll
        for (int u = 0; u < kDsU; ++u) {
            p[u] = np_[u];
            key[u] = nkey[u];
            const int r = r0 + 32 * kDsU + u * 32 + lane;
            np_[u] = r < whi ? a.seg[r] : -1;
            nkey[u] = r < whi ? a.key[r] : 0;
        }
#pragma unroll
        for (int u = 0; u < kDsU; ++u) {
            take[u] = part[u] = false;
            fb[u] = -1;
            if (p[u] >= 0) {
                int o, fo;
                const int2 bf = bins_of(key[u], p[u], o, fo);
                if (o < s_otake[p[u]]) {
                    take[u] = true;
                } else if (o == s_opart[p[u]]) {
                    part[u] = true;
                    fb[u] = p[u] * kDsFine + bf.y;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kDsU; ++u) {
            // fine counts; a partial superbin of one degree has a single fine bin, so its records are also
            // counted per warp (the ties' ranks need no second walk of the list)
            const bool coarse = part[u] && s_kind[p[u]] == 3;
            if (part[u]) {
                atomicAdd(&s_f[fb[u]], 1u);
                if (s_kind[p[u]] == 1) atomicAdd(&s_wc[wid * nseg + p[u]], 1);
            }
            // records below degree 2048 to the warp's list, in slot order; coarse ones to their label's
            // tail segment (one global atomic per label group of the warp)
            const unsigned mp = __ballot_sync(DMOLP_FULL_MASK, part[u] && !coarse);
            if (part[u] && !coarse) {
                wlist[wl + __popc(mp & below)] = p[u];
                wkey[wl + __popc(mp & below)] = key[u];
            }
            wl += __popc(mp);
            if (__any_sync(DMOLP_FULL_MASK, coarse)) {
                const unsigned mc = __match_any_sync(DMOLP_FULL_MASK, coarse ? p[u] : -1 - lane);
                int q = 0;
                if (coarse && lane == __ffs(mc) - 1) q = atomicAdd(&a.tcnt[p[u]], __popc(mc));
                q = __shfl_sync(DMOLP_FULL_MASK, q, coarse ? __ffs(mc) - 1 : lane);
                if (coarse) a.tail[s_toff[p[u]] + q + __popc(mc & below)] = key[u];
            }
        }
        emit_window<kDsU>(a.sp, take, key, p, vmask, te, ws, w_stage, w_scnt);  // all lanes
    }
    __syncthreads();
    // this block's fine counts: kept per block for the prefixes, summed for the fine decisions
    for (int i = threadIdx.x; i < nseg * kDsFine; i += blockDim.x) {
        const unsigned int v = s_f[i];
        a.dcntb[(size_t)blockIdx.x * nseg * kDsFine + i] = v;
        if (v) atomicAdd(&a.dfine[i], v);
    }
    if (!grid_sync(a.ctl, a.polls, 0)) return;
    // every block has read the superbin counts: clear them for the next boundary test
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nseg * kDsBins; i += gridDim.x * blockDim.x) a.dsup[i] = 0u;
    // ---- 2. per label with a partial superbin: the fine bin where the rest of the need is reached ----
    for (int p = wid; p < nseg; p += kDsWarps) {
        int take = 0, part = -1, rem = 0, pre = 0;
        const int kind = s_kind[p];
        if (kind != 0) {
            const int dir = s_dir[p];
            const int need = s_rem[p];
            int pos, before, count;
            ds_cross<kDsFine / 32>(need, [&](int fo) {
                return __ldcg(a.dfine + p * kDsFine + ds_ord(fo, kDsFine, dir));
            }, lane, pos, before, count);
            if (pos < 0) {
                take = 0;
            } else if (need - before == count) {
                take = pos + 1;
            } else {
                take = pos;
                part = pos;
                rem = need - before;
                if (kind != 3) {  // one degree: its records in the blocks before this one
                    const int f = ds_ord(pos, kDsFine, dir);
                    for (int b = lane; b < (int)blockIdx.x; b += 32)
                        pre += (int)__ldcg(a.dcntb + (size_t)b * nseg * kDsFine + p * kDsFine + f);
                    for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(DMOLP_FULL_MASK, pre, o);
                    if (lane == 0 && kind == 2) s_walk1 = 1;  // the warps' counts need a walk of the lists
                }
            }
        }
        if (lane == 0) {
            s_ftake[p] = take;
            s_fpart[p] = part;
            s_frem[p] = rem;
            s_pre[p] = pre;
        }
    }
    __syncthreads();
    // a record of the warp's list: its label, key, fine order position, and whether it is an exact tie
    auto list_rec = [&](int i, int &p, uint64_t &key, int &fo, bool &tie) {
        p = -1;
        key = 0;
        fo = -1;
        tie = false;
        if (i < wl) {
            p = wlist[i];
            key = wkey[i];
            int o;
            bins_of(key, p, o, fo);
            tie = fo == s_fpart[p];
        }
    };
    if (s_walk1) {  // exact ties of multi-degree superbins: this warp's count per label
        for (int i0 = 0; i0 < wl; i0 += 32) {
            int p, fo;
            uint64_t key;
            bool tie;
            list_rec(i0 + lane, p, key, fo, tie);
            tie = tie && s_kind[p] == 2;
            const unsigned m = __match_any_sync(DMOLP_FULL_MASK, tie ? p : -1 - lane);
            if (tie && lane == __ffs(m) - 1) s_wc[wid * nseg + p] += __popc(m);
            __syncwarp();
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kDsWarps * nseg; i += blockDim.x) {
        const int w = i / nseg, p = i - w * nseg;
        int base = s_pre[p];
        for (int x = 0; x < w; ++x) base += s_wc[x * nseg + p];
        s_wrun[i] = base;
    }
    __syncthreads();
    for (int i0 = 0; i0 < wl; i0 += 32) {
        int p, fo;
        uint64_t key;
        bool tie;
        list_rec(i0 + lane, p, key, fo, tie);
        bool take = p >= 0 && fo < s_ftake[p];
        const unsigned m = __match_any_sync(DMOLP_FULL_MASK, tie ? p : -1 - lane);
        if (tie) take = s_wrun[wid * nseg + p] + __popc(m & below) < s_frem[p];
        __syncwarp();
        if (tie && lane == __ffs(m) - 1) s_wrun[wid * nseg + p] += __popc(m);
        __syncwarp();
        emit_window<1>(a.sp, &take, &key, &p, vmask, te, ws, w_stage, w_scnt);  // all lanes
    }
    // ---- labels with a partial superbin of degree >= 2048: their tail segments ----
    // Every block takes its slice of every such segment's records of fine bins before the partial one.
    for (int p = 0; p < nseg; ++p) {
        if (s_kind[p] != 3) continue;  // block-uniform
        const int nt = __ldcg(a.tcnt + p);
        const int ch = (nt + (int)gridDim.x - 1) / (int)gridDim.x;
        const int lo = (int)blockIdx.x * ch, hi = min(nt, lo + ch);
        const uint64_t *seg_tail = a.tail + s_toff[p];
        const int ftake = s_ftake[p];
        for (int i0 = lo; i0 < hi; i0 += blockDim.x) {  // block-uniform trip count
            const int i = i0 + (int)threadIdx.x;
            bool take = false;
            uint64_t key = 0;
            int pp = p;
            if (i < hi) {
                key = __ldcg(seg_tail + i);
                int o, fo;
                bins_of(key, p, o, fo);
                take = fo < ftake;
            }
            emit_window<1>(a.sp, &take, &key, &pp, vmask, te, ws, w_stage, w_scnt);  // all lanes
        }
    }
    // Block p (p, p + gridDim.x, ...) takes label p's records of the partial fine bin.  It spans 2^jw degrees
    // (octave j, jw = j - 6); its records are counted per sub-bin of the label's order (one degree each while
    // jw <= 10, else 2^(jw-10) degrees), a block scan finds the sub-bin where the rest of the need is reached,
    // the sub-bins before it are taken, and only that sub-bin's records are sorted by key (degree, then id)
    // -- at these degrees usually a handful.
    for (int p = blockIdx.x; p < nseg; p += gridDim.x) {
        if (s_kind[p] != 3) continue;  // block-uniform
        const int nt = __ldcg(a.tcnt + p);
        const uint64_t *seg_tail = a.tail + s_toff[p];
        const int fpart = s_fpart[p], frem = s_frem[p], dir = s_dir[p];
        const int jw = ds_ord(s_opart[p], kDsBins, dir) - kDsCoarse0 + 5;  // superbin kDsCoarse0 + j - 11
        const int sh = jw > 10 ? jw - 10 : 0;
        const int nsub = 1 << (jw - sh);  // <= 1024 = blockDim.x
        auto sub_of = [&](uint64_t key) {
            const int dk = (int)(key >> ibits);
            const int x = (dir ? maxdeg - dk : dk) & ((1 << jw) - 1);
            return (dir ? (1 << jw) - 1 - x : x) >> sh;
        };
        unsigned int *s_sub = reinterpret_cast<unsigned int *>(s_tkey);  // counts first, the tied keys later
        __syncthreads();  // s_ntie and the shared tie keys are free
        for (int i = threadIdx.x; i < nsub; i += blockDim.x) s_sub[i] = 0u;
        if (threadIdx.x == 0) {
            s_ntie = 0;
            s_bstar = -1;
            s_before = 0;
        }
        __syncthreads();
        // pass 1: the partial fine bin's records counted per sub-bin (four keys per thread in flight)
        for (int i0 = 0; i0 < nt; i0 += 4 * blockDim.x) {
            uint64_t k4[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = i0 + q * (int)blockDim.x + (int)threadIdx.x;
                k4[q] = i < nt ? __ldcg(seg_tail + i) : ~0ull;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (k4[q] == ~0ull) continue;
                int o, fo;
                bins_of(k4[q], p, o, fo);
                if (fo == fpart) atomicAdd(&s_sub[sub_of(k4[q])], 1u);
            }
        }
        __syncthreads();
        {  // the sub-bin where the running count reaches frem (block scan, one sub-bin per thread)
            const unsigned int c = (int)threadIdx.x < nsub ? s_sub[threadIdx.x] : 0u;
            unsigned int incl = c;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) s_wsum[wid] = incl;
            __syncthreads();
            if (wid == 0) {
                unsigned int x = s_wsum[lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned int y = __shfl_up_sync(DMOLP_FULL_MASK, x, o);
                    if (lane >= o) x += y;
                }
                s_wsum[lane] = x;
            }
            __syncthreads();
            incl += wid ? s_wsum[wid - 1] : 0u;
            if (c && incl - c < (unsigned)frem && (unsigned)frem <= incl) {
                s_bstar = (int)threadIdx.x;
                s_before = (int)(incl - c);
            }
        }
        __syncthreads();
        const int bstar = s_bstar, rem2 = frem - s_before;  // bstar < 0: inconsistent counts (never expected)
        // pass 2: sub-bins before bstar are taken, bstar's records collected
        for (int i0 = 0; i0 < nt; i0 += blockDim.x) {
            const int i = i0 + (int)threadIdx.x;
            bool take = false;
            uint64_t key = 0;
            int pp = p;
            if (i < nt && bstar >= 0) {
                key = __ldcg(seg_tail + i);
                int o, fo;
                bins_of(key, p, o, fo);
                if (fo == fpart) {
                    const int sb2 = sub_of(key);
                    if (sb2 < bstar) {
                        take = true;
                    } else if (sb2 == bstar) {
                        const int q = atomicAdd(&s_ntie, 1);
                        if (q < kDsTieCap) s_tkey[q] = key;
                    }
                }
            }
            emit_window<1>(a.sp, &take, &key, &pp, vmask, te, ws, w_stage, w_scnt);  // all lanes
        }
        __syncthreads();
        const int m = s_ntie;
        if (bstar < 0) {
            // nothing more from this label
        } else if (m <= kDsTieCap) {
            // the sub-bin's records sorted by key (bitonic, padded to a power of two): the first rem2 are taken
            int n2 = 1;
            while (n2 < m) n2 <<= 1;
            for (int i = m + (int)threadIdx.x; i < n2; i += blockDim.x) s_tkey[i] = ~0ull;
            for (int size = 2; size <= n2; size <<= 1) {
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    __syncthreads();
                    for (int i = threadIdx.x; i < (n2 >> 1); i += blockDim.x) {
                        const int lo = 2 * stride * (i / stride) + (i % stride), hi = lo + stride;
                        const uint64_t x = s_tkey[lo], y = s_tkey[hi];
                        if ((x > y) == ((lo & size) == 0)) {
                            s_tkey[lo] = y;
                            s_tkey[hi] = x;
                        }
                    }
                }
            }
            __syncthreads();
            const int nt2 = rem2 < m ? rem2 : m;
            for (int i0 = 0; i0 < nt2; i0 += blockDim.x) {
                const int i = i0 + (int)threadIdx.x;
                bool take = i < nt2;
                uint64_t key = take ? s_tkey[i] : 0;
                int pp = p;
                emit_window<1>(a.sp, &take, &key, &pp, vmask, te, ws, w_stage, w_scnt);  // all lanes
            }
        } else {  // more ties than the shared keys hold: each ranked against the sub-bin in global memory
            for (int i0 = 0; i0 < nt; i0 += blockDim.x) {
                const int i = i0 + (int)threadIdx.x;
                bool take = false;
                uint64_t key = 0;
                int pp = p;
                if (i < nt) {
                    key = __ldcg(seg_tail + i);
                    int o, fo;
                    bins_of(key, p, o, fo);
                    if (fo == fpart && sub_of(key) == bstar) {
                        int rank = 0;
                        for (int j = 0; j < nt; ++j) {
                            const uint64_t kj = __ldcg(seg_tail + j);
                            int oj, foj;
                            bins_of(kj, p, oj, foj);
                            rank += foj == fpart && sub_of(kj) == bstar && kj < key;
                        }
                        take = rank < rem2;
                    }
                }
                emit_window<1>(a.sp, &take, &key, &pp, vmask, te, ws, w_stage, w_scnt);  // all lanes
            }
        }
    }
    // ---- end: the warps' staged appends and the block's sums, one atomic per list and per sum for the block
    //      (one per warp would queue ~4,700 atomics on each of six counters) ----
    __syncthreads();  // every warp's stage and counts are final
    if (threadIdx.x < 4) {
        const int j = threadIdx.x;
        int tot = 0;
        for (int w = 0; w < kDsWarps; ++w) {
            s_soff[w][j] = tot;
            tot += s_scnt[w][j];
        }
        s_sbase[j] = tot ? atomicAdd(list_ctr(a.sp, j), tot) : 0;
    }
    te = warp_sum_u64(te);
    ws = warp_sum_u64(ws);
    if (lane == 0) {
        s_te[wid] = te;
        s_ws[wid] = ws;
    }
    __syncthreads();
    for (int j = 0; j < 4; ++j) {
        const int n = w_scnt[j];
        int *dst = list_ptr(a.sp, j) + s_sbase[j] + s_soff[wid][j];
        for (int i = lane; i < n; i += 32) dst[i] = w_stage[j * kStage + i];
    }
    if (threadIdx.x == 0) {
        unsigned long long tt = 0, ww = 0;
        for (int w = 0; w < kDsWarps; ++w) {
            tt += s_te[w];
            ww += s_ws[w];
        }
        if (tt) atomicAdd(a.sp.te, tt);
        if (ww) atomicAdd(a.sp.wsum, ww);
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
    a.polls = c->wait_polls;
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

bool select_window_deg(dmolp_ctx *c, int nseg, const SplitArgs &split, const int *stopped) {
    if (nseg > kDegSelMaxK) return false;
    DegSelArgs a;
    a.seg = c->b.bown;
    a.key = c->b.bkey;
    a.n_dev = &c->b.cnt->npos;
    a.lists = c->b.active[0];
    a.lkeys = c->b.dlkey;
    a.tail = c->b.dtkey;
    a.tcnt = c->b.dtcnt + (split.t & 1) * kDegSelMaxK;
    a.tcnt_next = c->b.dtcnt + ((split.t + 1) & 1) * kDegSelMaxK;
    a.dsup = c->b.dsup;
    a.dfine = c->b.dfine[split.t & 1];
    a.dfine_next = c->b.dfine[(split.t + 1) & 1];
    a.dcntb = c->b.dcntb;
    a.nseg = nseg;
    a.polls = c->wait_polls;
    a.ctl = c->b.ctrl;
    a.stopped = stopped;
    a.sp = split;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)c->num_sms);  // one block per SM, all resident (cooperative launch)
    cfg.blockDim = dim3(kDsThreads);
    cfg.dynamicSmemBytes = ds_smem_bytes(nseg);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_select_deg, a);
    if (e != cudaSuccess && c->launch_error == cudaSuccess) c->launch_error = e;  // reported by the entry point
    c->launches += 1;
    return true;
}

int select_binary_version() {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_select) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return fa.binaryVersion;
}

void select_prepare() {
    cudaFuncSetAttribute(k_select_deg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ds_smem_bytes(kDegSelMaxK));
    cudaFuncSetAttribute(k_select, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kSmemSegMax * kRadix * sizeof(unsigned int) + 3 * DMOLP_MAX_K * sizeof(int) + 16 +
                               kTailBytes));
}

}  // namespace dmolp
