// Phase-2 label propagation on the resident CSR.  One iteration t (1-based) is a fixed sequence of
// launches with device-side counts, so it needs no host round trip and can be enqueued ahead or captured:
//
//   begin      penalties from the last statistics (calculatePenalties, src/phase2/phase2.cpp:158-209),
//              counter reset
//   cand       candidates = previous window plus its neighbours, deduplicated by an iteration stamp
//              (expandBoundaryNodes, src/phase2/gpu_lp_boundary.cu:195-240); at t = 1 every vertex
//   scan       one pass over each candidate's neighbours computing BOTH the boundary test
//              (gpu_lp_boundary.cu:251-270) and the penalised-argmax decision of boundaryLPKernel_unified
//              (gpu_lp_boundary.cu:354-426); boundary candidates become selection records
//   need/select  per label, the ceil(e^(-t/5) n) records with the smallest (degree asc|desc, id) key
//              (gpu_lp_boundary.cu:244, 277-301), by segmented radix select
//   commit     selected records become the next window; moved vertices take their new label (Jacobi:
//              every decision read the labels as they were at the start of the iteration)
//   mid/stats/end  the fused edge-cut + balance pass (computePartitionStats / computeEdgeCut,
//              phase2.cpp:55-117, 214-253) and the stopping rules of run_phase2 (phase2.cpp:309-415)
//
// Floating point: penalties and scores use __d*_rn intrinsics, which the compiler never contracts into
// FMAs, so every value is the IEEE double of the reference's expression in its evaluation order.
#include <cfloat>

#include "../../include/dmolp_b200.h"
#include "kernels.cuh"

namespace dmolp {
namespace {

constexpr int kGridPerSm = 4;

// ------------------------------------------------------------------------------------ begin
// Single block.  Thread 0 computes the penalties sequentially (k <= 1024 values); the block resets the
// per-iteration counters.
__global__ void k_lp_begin(Buffers b, int k, int t, long long narcs) {
    LpControl *ctl = b.ctrl;
    if (ctl->stopped) return;
    LpCounters *cn = b.cnt;
    for (int p = threadIdx.x; p < k; p += blockDim.x) b.npart[p] = 0;
    if (threadIdx.x == 0) {
        cn->ncand = 0;
        cn->nbnd = 0;
        cn->nwin[t & 1] = 0;
        cn->nchanged = 0;
        ctl->stop_now = 0;
        ctl->skip_stats = 0;
        LpRecordDev &r = b.rec[t - 1];
        r.iteration = t;
        r.window = r.candidates = r.changes = 0;
        r.boundary = 0;
        r.edge_cut = ctl->prev_cut;
        r.te_prev = t == 1 ? (unsigned long long)narcs : 0ull;
        r.te_cand = r.te_sel = r.te_stats = 0;

        // ---- statistics -> expected values (phase2.cpp:110-115) ----
        long long tv = 0, te = 0;
        for (int p = 0; p < k; ++p) {
            tv += (long long)b.vc[p];
            te += (long long)(b.intra[p] / 2);
        }
        const double ev = __ddiv_rn((double)tv, (double)k);
        const double ee = te > 0 ? __ddiv_rn((double)te, (double)k) : 1.0;
        // ---- calculatePenalties (phase2.cpp:166-203) ----
        double rv_mean = 0.0, re_mean = 0.0;
        for (int p = 0; p < k; ++p) {
            const double rv = ev > 0 ? __ddiv_rn((double)(long long)b.vc[p], ev) : 1.0;
            const double re = ee > 0 ? __ddiv_rn((double)(long long)(b.intra[p] / 2), ee) : 1.0;
            b.RE[p] = re;
            b.tpen[p] = rv;  // RV kept here until the penalties overwrite it below
            rv_mean = __dadd_rn(rv_mean, rv);
            re_mean = __dadd_rn(re_mean, re);
        }
        rv_mean = __ddiv_rn(rv_mean, (double)k);
        re_mean = __ddiv_rn(re_mean, (double)k);
        double rv_var = 0.0, re_var = 0.0;
        for (int p = 0; p < k; ++p) {
            const double dv = __dsub_rn(b.tpen[p], rv_mean), de = __dsub_rn(b.RE[p], re_mean);
            rv_var = __dadd_rn(rv_var, __dmul_rn(dv, dv));
            re_var = __dadd_rn(re_var, __dmul_rn(de, de));
        }
        rv_var = __ddiv_rn(rv_var, (double)k);
        re_var = __ddiv_rn(re_var, (double)k);
        const double total_var = __dadd_rn(rv_var, re_var);
        const double imb_rv = total_var > 0 ? __ddiv_rn(rv_var, total_var) : 0.0;
        const double imb_re = total_var > 0 ? __ddiv_rn(re_var, total_var) : 0.0;
        const double g = __dadd_rn(1.0, b.logtab[t]);
        double *ph = b.penhist + (size_t)(t - 1) * DMOLP_MAX_K;
        for (int p = 0; p < k; ++p) {
            const double grv = __dmul_rn(__dsub_rn(1.0, b.tpen[p]), g);
            const double gre = __dmul_rn(__dsub_rn(1.0, b.RE[p]), g);
            const double pen = __dadd_rn(__dmul_rn(imb_rv, grv), __dmul_rn(imb_re, gre));
            ph[p] = pen;
            b.tpen[p] = __dadd_rn(1.0, pen);  // the kernel's score factor (1.0 + penalty[c])
        }
    }
}

// ------------------------------------------------------------------------------------ cand
// Warp per vertex of the previous window: stamp the vertex and its neighbours with t; a vertex whose stamp
// changes is appended once.
__global__ void k_lp_cand(Buffers b, int t, int nv) {
    if (b.ctrl->stopped) return;
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int32_t *prev = b.win[(t - 1) & 1];
    const int n = b.cnt->nwin[(t - 1) & 1];
    unsigned long long te = 0;
    for (int i = gw; i < n; i += nw) {
        const int v = prev[i];
        const int64_t s = b.off[v], e = b.off[v + 1];
        if (lane == 0) te += (unsigned long long)(e - s);
        {
            bool fresh = false;
            if (lane == 0) fresh = atomicExch(&b.stamp[v], t) != t;
            const int slot = warp_append(&b.cnt->ncand, fresh);
            if (fresh) b.cand[slot] = v;
        }
        for (int64_t j0 = s; j0 < e; j0 += 32) {
            const int64_t j = j0 + lane;
            bool fresh = false;
            int u = 0;
            if (j < e) {
                u = ld_stream(b.col + j);
                fresh = atomicExch(&b.stamp[u], t) != t;
            }
            const int slot = warp_append(&b.cnt->ncand, fresh);
            if (fresh) b.cand[slot] = u;
        }
    }
    te = warp_sum_u64(te);
    if (lane == 0 && te) atomicAdd(&b.rec[t - 1].te_prev, te);
}

// ------------------------------------------------------------------------------------ scan
// Warp per candidate.  Each warp owns an `eff`-entry shared histogram of neighbour labels.  One read of the
// neighbour labels gives the boundary flag (any neighbour labelled differently) and the decision:
//   score[c] = count[c] > 0 ? count[c] * (1 + penalty[c]) : 0          for c < eff
//   M = max score; among labels scoring M the reference's shuffle tree keeps the one whose 5-bit
//   bit-reversed lane index is smallest (earlier 32-label chunk first when eff > 32);
//   new label = M > (own < eff ? count[own] : -1e300) ? that label : own.
__global__ void k_lp_scan(Buffers b, int t, int all, int nv, int eff, int ibits, int maxdeg) {
    if (b.ctrl->stopped) return;
    extern __shared__ int shist[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int *h = shist + wib * eff;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int n = all ? nv : b.cnt->ncand;
    unsigned long long te = 0;
    for (int i = gw; i < n; i += nw) {
        const int v = all ? i : b.cand[i];
        const int own = b.label[v];
        const int64_t s = b.off[v], e = b.off[v + 1];
        for (int c = lane; c < eff; c += 32) h[c] = 0;
        __syncwarp();
        bool diff = false;
        for (int64_t j = s + lane; j < e; j += 32) {
            const int lu = b.label[ld_stream(b.col + j)];
            diff |= (lu != own);
            if ((unsigned)lu < (unsigned)eff) atomicAdd(&h[lu], 1);
        }
        __syncwarp();
        if (lane == 0) te += (unsigned long long)(e - s);
        if (__any_sync(DMOLP_FULL_MASK, diff)) {
            double best = -DBL_MAX;
            int bkey = 0x7fffffff, blab = -1;
            for (int c = lane; c < eff; c += 32) {
                const int cnt = h[c];
                const double sc = cnt > 0 ? __dmul_rn((double)cnt, b.tpen[c]) : 0.0;
                const int key = (c & ~31) | (int)brev5((unsigned)c & 31u);
                if (sc > best || (sc == best && key < bkey)) {
                    best = sc;
                    bkey = key;
                    blab = c;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(DMOLP_FULL_MASK, best, o);
                const int ok = __shfl_xor_sync(DMOLP_FULL_MASK, bkey, o);
                const int ol = __shfl_xor_sync(DMOLP_FULL_MASK, blab, o);
                if (ob > best || (ob == best && ok < bkey)) {
                    best = ob;
                    bkey = ok;
                    blab = ol;
                }
            }
            if (lane == 0) {
                const double own_raw = (unsigned)own < (unsigned)eff ? (double)h[own] : -1e300;
                const int nl = best > own_raw ? blab : own;
                const int idx = atomicAdd(&b.cnt->nbnd, 1);
                const int deg = (int)(e - s);
                const uint64_t dk = b.RE[own] > 1.0 ? (uint64_t)(maxdeg - deg) : (uint64_t)deg;
                b.bv[idx] = v;
                b.bown[idx] = own;
                b.bnew[idx] = nl;
                b.bkey[idx] = (dk << ibits) | (uint64_t)v;
                b.bsel[idx] = 0;
                atomicAdd(&b.npart[own], 1);
            }
        }
        __syncwarp();
    }
    te = warp_sum_u64(te);
    if (lane == 0 && te) atomicAdd(&b.rec[t - 1].te_cand, te);
}

// ------------------------------------------------------------------------------------ need
// need[p] = min(n_p, ceil(e^(-t/5) * n_p))   (gpu_lp_boundary.cu:244, 296-297)
__global__ void k_lp_need(Buffers b, int k, int t) {
    if (b.ctrl->stopped) return;
    const double ratio = b.ratiotab[t];
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        const int n = b.npart[p];
        int m = (int)ceil(__dmul_rn(ratio, (double)n));
        b.need[p] = m > n ? n : m;
    }
}

// ------------------------------------------------------------------------------------ commit
__global__ void k_lp_commit(Buffers b, int t, int apply) {
    if (b.ctrl->stopped) return;
    const int n = b.cnt->nbnd;
    int32_t *win = b.win[t & 1];
    unsigned long long te = 0;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        bool take = false, moved = false;
        int v = 0;
        if (i < n && b.bsel[i]) {
            take = true;
            v = b.bv[i];
            te += (unsigned long long)(b.off[v + 1] - b.off[v]);
            const int nl = b.bnew[i];
            if (apply && nl != b.bown[i]) {
                b.label[v] = nl;
                moved = true;
            }
        }
        const int slot = warp_append(&b.cnt->nwin[t & 1], take);
        if (take) win[slot] = v;
        warp_append(&b.cnt->nchanged, moved);
    }
    te = warp_sum_u64(te);
    if ((threadIdx.x & 31) == 0 && te) atomicAdd(&b.rec[t - 1].te_sel, te);
}

// ------------------------------------------------------------------------------------ mid
// Decides whether this iteration runs the statistics pass (run_phase2's breaks at phase2.cpp:309 and 387
// come before the statistics), and clears the accumulators for it.
__global__ void k_lp_mid(Buffers b, int k, int t) {
    LpControl *ctl = b.ctrl;
    if (ctl->stopped) return;
    __shared__ int s_skip;
    if (threadIdx.x == 0) {
        LpRecordDev &r = b.rec[t - 1];
        r.window = b.cnt->nwin[t & 1];
        r.candidates = t == 1 ? -1 : b.cnt->ncand;
        r.changes = b.cnt->nchanged;
        r.boundary = b.cnt->nbnd;
        int skip = 0;
        if (r.window == 0) {
            skip = 1;
            if (ctl->mode == DMOLP_LP_MODE_REF) ctl->stop_now = 1;
        } else if (r.changes == 0 && ctl->mode == DMOLP_LP_MODE_REF) {
            skip = 1;
            ctl->stop_now = 2;
        }
        ctl->skip_stats = skip;
        if (!skip) b.cnt->cut_arcs = 0;
        s_skip = skip;
    }
    __syncthreads();
    if (!s_skip)
        for (int p = threadIdx.x; p < k; p += blockDim.x) {
            b.vc[p] = 0;
            b.intra[p] = 0;
        }
}

// ------------------------------------------------------------------------------------ stats
// The fused edge-cut / balance pass: per vertex its label count, its same-label arcs and its cut arcs.
// Warp per vertex; per-block shared accumulators per label.
__global__ void k_stats(Buffers b, int k, int nv, const int *stopped, const int *skip) {
    if ((stopped && *stopped) || (skip && *skip)) return;
    extern __shared__ unsigned long long sacc[];  // [2k]: vertex counts, intra arcs
    unsigned long long *svc = sacc, *sin = sacc + k;
    for (int p = threadIdx.x; p < 2 * k; p += blockDim.x) sacc[p] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long cut = 0;
    bool bad = false;
    for (int v = gw; v < nv; v += nw) {
        const int lv = b.label[v];
        const int64_t s = b.off[v], e = b.off[v + 1];
        unsigned int same = 0, diff = 0;
        for (int64_t j = s + lane; j < e; j += 32) {
            const int lu = b.label[ld_stream(b.col + j)];
            bad |= (unsigned)lu >= (unsigned)k;
            same += (lu == lv);
            diff += (lu != lv);
        }
        for (int o = 16; o > 0; o >>= 1) {
            same += __shfl_xor_sync(DMOLP_FULL_MASK, same, o);
            diff += __shfl_xor_sync(DMOLP_FULL_MASK, diff, o);
        }
        if (lane == 0) {
            if ((unsigned)lv < (unsigned)k) {
                atomicAdd(&svc[lv], 1ull);
                if (same) atomicAdd(&sin[lv], (unsigned long long)same);
            } else {
                bad = true;
            }
            cut += diff;
        }
    }
    cut = warp_sum_u64(cut);
    if (lane == 0 && cut) atomicAdd(&b.cnt->cut_arcs, cut);
    if (__any_sync(DMOLP_FULL_MASK, bad) && lane == 0) b.ctrl->error = 1;
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        if (svc[p]) atomicAdd(&b.vc[p], svc[p]);
        if (sin[p]) atomicAdd(&b.intra[p], sin[p]);
    }
}

// ------------------------------------------------------------------------------------ end
__global__ void k_lp_end(Buffers b, int k, int t, long long narcs) {
    LpControl *ctl = b.ctrl;
    if (ctl->stopped) return;
    LpRecordDev &r = b.rec[t - 1];
    if (!ctl->skip_stats) {
        const unsigned long long arcs = b.cnt->cut_arcs;
        r.te_stats = (unsigned long long)narcs;
        if ((arcs & 1ull) || ctl->error) {
            ctl->error = 1;
            ctl->stop_now = 4;
        } else {
            const long long cur = (long long)(arcs >> 1);
            const long long prev = ctl->prev_cut;
            const double delta = prev > 0 ? fabs(__ddiv_rn((double)(cur - prev), (double)prev)) : 1.0;
            if (delta < 0.03) ctl->conv += 1;
            else ctl->conv = 0;
            ctl->prev_cut = cur;
            if (ctl->mode == DMOLP_LP_MODE_REF && ctl->conv >= 10) ctl->stop_now = 3;
        }
    }
    r.edge_cut = ctl->prev_cut;
    long long *ch = b.cnthist + (size_t)(t - 1) * 2 * DMOLP_MAX_K;
    for (int p = 0; p < k; ++p) {
        ch[p] = (long long)b.vc[p];
        ch[DMOLP_MAX_K + p] = (long long)(b.intra[p] / 2);
    }
    ctl->iters_run = t;
    if (ctl->stop_now) {
        ctl->stopped = 1;
        ctl->stop_reason = ctl->stop_now;
    }
}

__global__ void k_lp_init_end(Buffers b, int mode) {
    LpControl *ctl = b.ctrl;
    const unsigned long long arcs = b.cnt->cut_arcs;
    ctl->mode = mode;
    ctl->conv = 0;
    ctl->iters_run = 0;
    ctl->stop_reason = 0;
    ctl->stop_now = 0;
    ctl->skip_stats = 0;
    ctl->prev_cut = (long long)(arcs >> 1);
    if ((arcs & 1ull) || ctl->error) {
        ctl->error = 1;
        ctl->stopped = 1;
        ctl->stop_reason = 4;
    } else {
        ctl->stopped = 0;
    }
}

__global__ void k_reset_stats(Buffers b, int k, const int *stopped) {
    if (stopped && *stopped) return;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        b.vc[p] = 0;
        b.intra[p] = 0;
    }
    if (threadIdx.x == 0) {
        b.cnt->cut_arcs = 0;
        if (!stopped) b.ctrl->error = 0;
    }
}

// ---- single-call pieces (dmolp_window_select / dmolp_lp_apply) ----

// Records for an explicit window list (already in b.cand, count in cnt->ncand): decisions only.
__global__ void k_apply_scan(Buffers b, int n, int eff) {
    extern __shared__ int shist[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int *h = shist + wib * eff;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < n; i += nw) {
        const int v = b.cand[i];
        const int own = b.label[v];
        const int64_t s = b.off[v], e = b.off[v + 1];
        for (int c = lane; c < eff; c += 32) h[c] = 0;
        __syncwarp();
        for (int64_t j = s + lane; j < e; j += 32) {
            const int lu = b.label[b.col[j]];
            if ((unsigned)lu < (unsigned)eff) atomicAdd(&h[lu], 1);
        }
        __syncwarp();
        double best = -DBL_MAX;
        int bkey = 0x7fffffff, blab = -1;
        for (int c = lane; c < eff; c += 32) {
            const int cnt = h[c];
            const double sc = cnt > 0 ? __dmul_rn((double)cnt, b.tpen[c]) : 0.0;
            const int key = (c & ~31) | (int)brev5((unsigned)c & 31u);
            if (sc > best || (sc == best && key < bkey)) {
                best = sc;
                bkey = key;
                blab = c;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(DMOLP_FULL_MASK, best, o);
            const int ok = __shfl_xor_sync(DMOLP_FULL_MASK, bkey, o);
            const int ol = __shfl_xor_sync(DMOLP_FULL_MASK, blab, o);
            if (ob > best || (ob == best && ok < bkey)) {
                best = ob;
                bkey = ok;
                blab = ol;
            }
        }
        if (lane == 0) {
            const double own_raw = (unsigned)own < (unsigned)eff ? (double)h[own] : -1e300;
            b.bnew[i] = best > own_raw ? blab : own;
            b.bown[i] = own;
            b.bv[i] = v;
        }
        __syncwarp();
    }
}

__global__ void k_apply_commit(Buffers b, int n) {
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        bool moved = false;
        if (i < n && b.bnew[i] != b.bown[i]) {
            b.label[b.bv[i]] = b.bnew[i];
            moved = true;
        }
        const int slot = warp_append(&b.cnt->nchanged, moved);
        if (moved) b.win[0][slot] = i;  // index into bv/bnew of the moved record
    }
}

__global__ void k_zero_counters(Buffers b) {
    b.cnt->ncand = 0;
    b.cnt->nbnd = 0;
    b.cnt->nwin[0] = b.cnt->nwin[1] = 0;
    b.cnt->nchanged = 0;
}

// Set-up of a stand-alone window selection: the caller's previous window is in win[(t-1)&1].
__global__ void k_ws_begin(Buffers b, int k, int t, int nprev) {
    for (int p = threadIdx.x; p < k; p += blockDim.x) b.npart[p] = 0;
    if (threadIdx.x == 0) {
        b.cnt->ncand = 0;
        b.cnt->nbnd = 0;
        b.cnt->nchanged = 0;
        b.cnt->nwin[(t - 1) & 1] = nprev;
        b.cnt->nwin[t & 1] = 0;
        b.ctrl->stopped = 0;
        LpRecordDev &r = b.rec[t - 1];
        r.te_prev = r.te_cand = r.te_sel = r.te_stats = 0;
    }
}

int grid_for(dmolp_ctx *c) { return c->num_sms * kGridPerSm; }

}  // namespace

void lp_reset_stats(dmolp_ctx *c, int k, const int *stopped) {
    k_reset_stats<<<1, 256, 0, c->stream>>>(c->b, k, stopped);
    c->launches++;
}

void lp_stats(dmolp_ctx *c, int k, const int *stopped, const int *skip) {
    k_stats<<<grid_for(c), kBlock, 2 * k * sizeof(unsigned long long), c->stream>>>(c->b, k, (int)c->nv, stopped,
                                                                                     skip);
    c->launches++;
}

void lp_init_end(dmolp_ctx *c, int mode) {
    k_lp_init_end<<<1, 1, 0, c->stream>>>(c->b, mode);
    c->launches++;
}

// Optional timing of one kernel launch (dmolp_set_profiling): an event pair around it on the same stream.
struct ProfScope {
    dmolp_ctx *c;
    int kind, t;
    cudaEvent_t e1 = nullptr;
    ProfScope(dmolp_ctx *c_, int kind_, int t_) : c(c_), kind(kind_), t(t_) {
        if (!c->profiling) return;
        cudaEvent_t e0;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, c->stream);
        c->prof_events.push_back(e0);
        c->prof_events.push_back(e1);
        c->prof_kind.push_back(kind);
        c->prof_iter.push_back(t);
    }
    ~ProfScope() {
        if (e1) cudaEventRecord(e1, c->stream);
    }
};

void lp_iteration(dmolp_ctx *c, const LpLaunch &L, int t) {
    Buffers &b = c->b;
    const int grid = grid_for(c);
    const int *stopped = &b.ctrl->stopped;
    k_lp_begin<<<1, 256, 0, c->stream>>>(b, L.k, t, (long long)c->narcs);
    if (t > 1) k_lp_cand<<<grid, kBlock, 0, c->stream>>>(b, t, (int)c->nv);
    const size_t smem = (size_t)kWarpsPerBlock * L.eff * sizeof(int);
    {
        ProfScope ps(c, 0, t);
        k_lp_scan<<<grid, kBlock, smem, c->stream>>>(b, t, t == 1, (int)c->nv, L.eff, c->ibits, (int)c->maxdeg);
    }
    k_lp_need<<<1, 256, 0, c->stream>>>(b, L.k, t);
    c->launches += t > 1 ? 4 : 3;
    select_smallest(c, b.bown, b.bkey, &b.cnt->nbnd, L.k, c->dbits + c->ibits, b.bsel, stopped);
    k_lp_commit<<<grid, kBlock, 0, c->stream>>>(b, t, 1);
    k_lp_mid<<<1, 256, 0, c->stream>>>(b, L.k, t);
    {
        ProfScope ps(c, 1, t);
        k_stats<<<grid, kBlock, 2 * L.k * sizeof(unsigned long long), c->stream>>>(b, L.k, (int)c->nv, stopped,
                                                                                    &b.ctrl->skip_stats);
    }
    k_lp_end<<<1, 1, 0, c->stream>>>(b, L.k, t, (long long)c->narcs);
    c->launches += 4;
}

// The window of dmolp_window_select: prev list in win[(t-1)&1] with count n; RE in b.RE.
void lp_window_from_list(dmolp_ctx *c, int k, int t, const double *RE_dev, int nprev) {
    (void)RE_dev;  // already copied to b.RE by the caller
    Buffers &b = c->b;
    const int grid = grid_for(c);
    k_ws_begin<<<1, 256, 0, c->stream>>>(b, k, t, nprev);
    k_lp_cand<<<grid, kBlock, 0, c->stream>>>(b, t, (int)c->nv);
    // the scan's decisions are not used here (eff = 1 keeps its histogram tiny); only its records are
    const size_t smem = (size_t)kWarpsPerBlock * 1 * sizeof(int);
    k_lp_scan<<<grid, kBlock, smem, c->stream>>>(b, t, 0, (int)c->nv, 1, c->ibits, (int)c->maxdeg);
    k_lp_need<<<1, 256, 0, c->stream>>>(b, k, t);
    c->launches += 4;
    select_smallest(c, b.bown, b.bkey, &b.cnt->nbnd, k, c->dbits + c->ibits, b.bsel, nullptr);
    k_lp_commit<<<grid, kBlock, 0, c->stream>>>(b, t, 0);
    c->launches += 1;
}

// Decisions + commit for an explicit list already in b.cand (n entries), penalties in b.tpen.
void lp_apply_list(dmolp_ctx *c, int k, int eff, int n) {
    (void)k;
    Buffers &b = c->b;
    const int grid = grid_for(c);
    k_zero_counters<<<1, 1, 0, c->stream>>>(b);
    const size_t smem = (size_t)kWarpsPerBlock * eff * sizeof(int);
    k_apply_scan<<<grid, kBlock, smem, c->stream>>>(b, n, eff);
    k_apply_commit<<<grid, kBlock, 0, c->stream>>>(b, n);
    c->launches += 3;
}

}  // namespace dmolp
