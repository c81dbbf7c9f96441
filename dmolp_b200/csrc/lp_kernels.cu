// Phase-2 label propagation on the resident CSR.  One iteration t (1-based) is a fixed sequence of
// launches with device-side counts, so a whole run is captured once into a CUDA graph and replayed:
//
//   begin    penalties from the current statistics (calculatePenalties, src/phase2/phase2.cpp:158-209);
//            counter reset (with the previous iteration's end: one k_lp_turn between iterations)
//   mark     stamp the previous window and its neighbours with t (expandBoundaryNodes' candidate set,
//            src/phase2/gpu_lp_boundary.cu:195-240): thread per short row, warp per longer row; a hub's
//            row is walked only when the hub enters or leaves the window, keeping hubwin[u] (window hubs
//            whose rows hold u) current
//   bnd      degree-bucketed candidacy (stamp / hubwin, or a pull walk that stops at the first window
//            neighbour) and the boundary test from the maintained count of differently-labelled neighbours
//            (gpu_lp_boundary.cu:251-270); a boundary vertex becomes a selection record keyed (degree
//            asc|desc by RE[label], id), counted per label and degree superbin (k <= 64; else the first
//            radix digit of the keys is histogrammed per label)
//   select   per label the ceil(e^(-t/5) n) smallest keys (gpu_lp_boundary.cu:244, 277-301), from the
//            degree bins (k <= 64, select_kernels.cu k_select_deg) or by radix select; the selection emits
//            the next window and routes it to the decision classes
//   decide   boundaryLPKernel_unified's rule (gpu_lp_boundary.cu:354-426) for the selected vertices only:
//            persistent warps over hub row chunks, warp-class groups and thread-class groups; on symmetric
//            graphs the hubs' label counts (and, with at most 32 scored labels, every vertex's) are kept
//            current instead of recounted; a changed label is parked in newlab[] (Jacobi: nothing moves yet)
//   update   (symmetric graphs) edge cut, per-part intra arcs and vertex counts change only through the
//            movers' arcs: each arc is re-scored with both endpoints' old and new labels, weighted 2 when
//            the neighbour stays (its reverse arc is not visited) and 1 when it moves too.  Asymmetric
//            graphs run the full statistics pass instead (computePartitionStats / computeEdgeCut,
//            phase2.cpp:55-117, 214-253).
//   apply    movers take their new labels
//   end      the stopping rules of run_phase2 (phase2.cpp:309-415) and the iteration record
//
// Floating point: penalties and scores use __d*_rn intrinsics, which the compiler never contracts into
// FMAs, so every value is the IEEE double of the reference's expression in its evaluation order.
#include <cfloat>

#include "../../include/dmolp_b200.h"
#include "kernels.cuh"
#include "lp_device.cuh"

namespace dmolp {
namespace {

constexpr int kGridPerSm = 4;

// ------------------------------------------------------------------------------------ begin
// Start of iteration t (one block): counters, the iteration record, penalties.
__device__ void lp_begin(const Buffers &b, int k, int t, long long narcs, double *s_re, double *s_tp) {
    LpControl *ctl = b.ctrl;
    LpCounters *cn = b.cnt;
    for (int p = threadIdx.x; p < k; p += blockDim.x) b.npart[p] = 0;
    if (threadIdx.x == 0) {
        cn->ncand = 0;
        cn->nbnd = 0;
        cn->nwin[t & 1] = 0;
        cn->nchanged = 0;
        for (int c = 0; c < 3; ++c) {
            cn->ndec_prev[c] = t > 1 ? cn->ndec[c] : 0;
            cn->ndec[c] = 0;
        }
        cn->nchunk = 0;
        cn->nhubq = 0;
        cn->nhubw = 0;
        cn->dgrab[0] = cn->dgrab[1] = cn->dgrab[2] = 0;
        ctl->stop_now = 0;
        ctl->skip_stats = 0;
        LpRecordDev &r = b.rec[t - 1];
        r.iteration = t;
        r.window = r.candidates = r.changes = r.boundary = 0;
        r.edge_cut = ctl->prev_cut;
        // sum of degrees over the previous window = the previous iteration's selected window
        r.te_prev = t == 1 ? (unsigned long long)narcs : b.rec[t - 2].te_sel;
        r.te_cand = r.te_sel = r.te_stats = 0;
        r.arcs_bnd = r.arcs_dec = r.arcs_upd = r.arcs_mark = r.te_hubsel = 0;
        r.win_sum = 0;
    }
    // ---- statistics -> expected values and calculatePenalties (phase2.cpp:110-115, 158-209) ----
    // (RE and the penalties in shared memory while the serial sums read them, then out to global)
    if (threadIdx.x < 32) {
        warp_penalties(k, [&](int p) { return sll(b.vc[p]); }, [&](int p) { return sll(b.intra[p]) / 2; },
                       b.logtab[t], s_re, s_tp, b.penhist + (size_t)(t - 1) * DMOLP_MAX_K);
        for (int p = threadIdx.x; p < k; p += 32) {
            b.RE[p] = s_re[p];
            b.tpen[p] = s_tp[p];
        }
    }
}

// ------------------------------------------------------------------------------------ mark
// Hubs sit in many rows: reading the stamp first saves most of the (L2) stores.
__device__ __forceinline__ void stamp_once(const Buffers &b, int u, int t) {
    if (b.stamp[u] != t) b.stamp[u] = t;
}

// dmolp_window_select's marking: warp per vertex of the previous window (win list): stamp it and its
// first kChunk neighbours; the rest of a long row is queued in kChunk pieces for k_mark_chunks.
__global__ void k_mark(Buffers b, int t) {
    if (b.ctrl->stopped || b.ctrl->pull) return;
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int32_t *prev = b.win[(t - 1) & 1];
    const int n = b.cnt->nwin[(t - 1) & 1];
    unsigned long long rd = 0;
    for (int i = gw; i < n; i += nw) {
        const int v = prev[i];
        const int64_t s = b.off[v], e = b.off[v + 1];
        if (lane == 0) {
            b.stamp[v] = t;
            for (int64_t c = s + kChunk; c < e; c += kChunk) {
                const int q = atomicAdd(&b.cnt->nchunk, 1);
                b.chunkq[q] = make_int2(v, (int)(c - s));
            }
        }
        const int64_t e1 = e - s > kChunk ? s + kChunk : e;
        warp_row(b.col, s, e1, lane, [&](int u) { stamp_once(b, u, t); }, [] { return false; });
        if (lane == 0) rd += (unsigned long long)(e1 - s);
    }
    block_atomic_add(rd, &b.rec[t - 1].arcs_mark);
}

__global__ void k_mark_chunks(Buffers b, int t) {
    if (b.ctrl->stopped) return;
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int n = b.cnt->nchunk;
    unsigned long long rd = 0;
    for (int i = gw; i < n; i += nw) {
        const int2 q = b.chunkq[i];
        const int64_t s = b.off[q.x] + q.y, rowe = b.off[q.x + 1];
        const int64_t e = rowe - s > kChunk ? s + kChunk : rowe;
        warp_row(b.col, s, e, lane, [&](int u) { stamp_once(b, u, t); }, [] { return false; });
        if (lane == 0) rd += (unsigned long long)(e - s);
    }
    block_atomic_add(rd, &b.rec[t - 1].arcs_mark);
}

// The loop's marking: the previous window by decision class (dec[c], ndec_prev[c]; the lists are rewritten
// only by this iteration's selection, after the marking).  Blocks [0, g0): thread per vertex of class 0
// (rows of at most kDecSmall arcs), then the hubs (class 2), which stamp only themselves -- their
// neighbours are candidates through hubwin; blocks [g0, grid): warp per vertex of class 1.
__global__ void __launch_bounds__(256, 5) k_mark_win(Buffers b, int t, int g0) {
    if (b.ctrl->stopped || b.ctrl->pull) return;
    const LpCounters *cn = b.cnt;
    const int lane = threadIdx.x & 31;
    unsigned long long rd = 0;
    if ((int)blockIdx.x < g0) {
        const int stride = g0 * blockDim.x;
        const int n0 = cn->ndec_prev[0];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n0; i += stride) {
            const int v = b.dec[0][i];
            const int64_t s = b.off[v];
            const int deg = (int)(b.off[v + 1] - s);
            b.stamp[v] = t;
            rd += (unsigned long long)deg;
            for (int j = 0; j < deg; j += 8) {  // eight ids in flight, then their stamps stored
                int u[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) u[q] = j + q < deg ? __ldg(b.col + s + j + q) : -1;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (u[q] >= 0) b.stamp[u[q]] = t;
            }
        }
        const int n2 = cn->ndec_prev[2];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) b.stamp[b.dec[2][i]] = t;
    } else {
        const int gw = (((int)blockIdx.x - g0) * (int)blockDim.x + (int)threadIdx.x) >> 5;
        const int nw = (((int)gridDim.x - g0) * (int)blockDim.x) >> 5;
        const int n1 = cn->ndec_prev[1];
        for (int i = gw; i < n1; i += nw) {
            const int v = b.dec[1][i];
            const int64_t s = b.off[v], e = b.off[v + 1];
            if (lane == 0) {
                b.stamp[v] = t;
                rd += (unsigned long long)(e - s);
            }
            warp_row_wide(b.col, s, e, lane, [](int) { return 0; }, [&](int u, int) { b.stamp[u] = t; },
                          [] { return false; });
        }
    }
    block_atomic_add(rd, &b.rec[t - 1].arcs_mark);
}

// hubwin[u] = hubs of the previous window whose rows hold u, kept across iterations: a hub that entered
// the window (sstamp == t-1) adds one to every vertex of its row, a hub that left subtracts one.  Thread
// per hub: flip hub_in and queue the row in kHubChunk pieces.
__global__ void k_hubwin_queue(Buffers b, int t, int nhub) {
    if (b.ctrl->stopped) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nhub; i += gridDim.x * blockDim.x) {
        const int h = b.bucket[2][i];
        const int now = b.sstamp[h] == t - 1;
        if (now == b.hub_in[i]) continue;
        b.hub_in[i] = now;
        const int64_t deg = b.off[h + 1] - b.off[h];
        const int nch = (int)((deg + kHubChunk - 1) / kHubChunk);
        const int base = atomicAdd(&b.cnt->nhubw, nch);
        for (int c = 0; c < nch; ++c) b.hubwq[base + c] = make_int2(i, c * kHubChunk);
    }
}

// Warp per queued chunk: +1 (hub entered) or -1 (hub left) on every vertex of the chunk.
__global__ void k_hubwin_apply(Buffers b, int t) {
    if (b.ctrl->stopped) return;
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int n = b.cnt->nhubw;
    unsigned long long rd = 0;
    for (int i = gw; i < n; i += nw) {
        const int2 q = b.hubwq[i];
        const int h = b.bucket[2][q.x];
        const int d = b.hub_in[q.x] ? 1 : -1;
        const int64_t s = b.off[h] + q.y, rowe = b.off[h + 1];
        const int64_t e = rowe - s > kHubChunk ? s + kHubChunk : rowe;
        warp_row(b.col, s, e, lane, [&](int u) { atomicAdd(&b.hubwin[u], d); }, [] { return false; });
        if (lane == 0) rd += (unsigned long long)(e - s);
    }
    block_atomic_add(rd, &b.rec[t - 1].arcs_mark);
}

// ------------------------------------------------------------------------------------ bnd
struct BndArgs {
    int t, all, ibits, maxdeg;
    int hubwin;  // hubwin is current: hubs of the previous window make their neighbours candidates
    unsigned int *hist;  // when set: first-digit histogram of the boundary records for the selection (k <= 32)
    int hshift;          // its digit: bits [hshift, hshift + 8) of the key
    unsigned int *dsup;  // when set: degree-superbin counts of the boundary records per label (k <= 64)
    int nb0, nb1, nb2;
    int g0, g1;  // block split: [0,g0) thread class, [g0,g0+g1) warp class, rest block class
};

__device__ __forceinline__ uint64_t sel_key(const Buffers &b, int own, int deg, int v, int ibits, int maxdeg) {
    const uint64_t dk = b.RE[own] > 1.0 ? (uint64_t)(maxdeg - deg) : (uint64_t)deg;
    return (dk << ibits) | (uint64_t)v;
}

// Record slot pos (the vertex's position in ball): own label and key of a boundary vertex, -1 otherwise.
// No global append: every slot is rewritten each iteration.  (The LP selections emit the window directly;
// the selection flags bsel are read only by phase 1, which clears its own.)
__device__ __forceinline__ void put_slot(const Buffers &b, int pos, bool isb, int own, uint64_t key) {
    b.bown[pos] = isb ? own : -1;
    if (isb) b.bkey[pos] = key;
}

// Candidacy: t = 1 every vertex; push mode stamp[v] == t (set by k_mark); pull mode v is in the previous
// window (sstamp == t-1) or has a neighbour that is; in both modes hubwin[v] > 0 (a hub of the previous
// window lists v) when the hub rows are not walked.  A candidate is on the boundary when it has a
// differently-labelled neighbour: ndiff[v] > 0, a count kept exact by the statistics pass and by k_update
// (symmetric graphs) or by the full pass after every move (other graphs).  So only pull-mode candidacy
// walks rows; at t = 1 and in push mode every record slot costs a handful of per-vertex reads.
constexpr int kBndPushU = 4;  // k_bnd push mode: record slots per thread and step

__global__ void __launch_bounds__(256, 5) k_bnd(Buffers b, BndArgs a, int k) {
    if (b.ctrl->stopped) return;
    // [k] boundary records per label in this block, then [k * 256] first-digit or [k * kDsBins] superbin counts
    extern __shared__ int s_npart[];
    unsigned int *s_hist = reinterpret_cast<unsigned int *>(s_npart + k);
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_npart[p] = 0;
    const int nhist = a.dsup ? k * kDsBins : (a.hist ? k * kRadix : 0);
    for (int i = threadIdx.x; i < nhist; i += blockDim.x) s_hist[i] = 0u;
    __syncthreads();
    const bool pull = !a.all && b.ctrl->pull;
    const int tp = a.t - 1;
    const int lane = threadIdx.x & 31;
    unsigned long long te = 0, rd = 0, nc = 0, nbd = 0;
    // nd = ndiff[v] and lv = label[v], loaded by the caller ahead of the candidacy test
    auto finish = [&](int pos, int v, bool cand, int deg, int nd, int lv) {
        const bool isb = cand && nd > 0;
        int own = 0;
        if (cand) {
            ++nc;
            te += (unsigned long long)deg;
        }
        uint64_t key = 0;
        if (isb) {
            own = lv;
            ++nbd;
            atomicAdd(&s_npart[own], 1);
            key = sel_key(b, own, deg, v, a.ibits, a.maxdeg);
            if (a.dsup) atomicAdd(&s_hist[own * kDsBins + dsel_bin(deg).x], 1u);
            else if (a.hist) atomicAdd(&s_hist[own * kRadix + (int)((key >> a.hshift) & (kRadix - 1))], 1u);
        }
        put_slot(b, pos, isb, own, key);
    };
    if (!pull) {
        // ---- every record slot, thread per slot; kBndPushU slots per thread with their loads in flight
        //      together (the per-slot chain slot -> vertex state -> offsets is latency, not bandwidth) ----
        const int n = a.nb0 + a.nb1 + a.nb2;
        const int nt = (int)gridDim.x * (int)blockDim.x;
        for (int p0 = blockIdx.x * blockDim.x + threadIdx.x; p0 < n; p0 += kBndPushU * nt) {
            int v[kBndPushU], st[kBndPushU], hw[kBndPushU], nd[kBndPushU], lv[kBndPushU], deg[kBndPushU];
            bool cand[kBndPushU];
#pragma unroll
            for (int q = 0; q < kBndPushU; ++q) v[q] = p0 + q * nt < n ? b.ball[p0 + q * nt] : -1;
#pragma unroll
            for (int q = 0; q < kBndPushU; ++q) {
                st[q] = hw[q] = nd[q] = lv[q] = 0;
                if (v[q] >= 0) {
                    st[q] = b.stamp[v[q]];
                    hw[q] = a.hubwin ? b.hubwin[v[q]] : 0;
                    nd[q] = b.ndiff[v[q]];
                    lv[q] = b.label[v[q]];
                }
            }
#pragma unroll
            for (int q = 0; q < kBndPushU; ++q) {
                cand[q] = v[q] >= 0 && (a.all || st[q] == a.t || hw[q] > 0);
                deg[q] = cand[q] ? (int)(b.off[v[q] + 1] - b.off[v[q]]) : 0;
            }
#pragma unroll
            for (int q = 0; q < kBndPushU; ++q)
                if (v[q] >= 0) finish(p0 + q * nt, v[q], cand[q], deg[q], nd[q], lv[q]);
        }
    } else if ((int)blockIdx.x < a.g0) {
        // ---- pull, thread per vertex (deg <= kSmallDeg): window stamps of the row, 8 at a time ----
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nb0; i += a.g0 * blockDim.x) {
            const int v = b.bucket[0][i];
            const int st = b.sstamp[v], hw = a.hubwin ? b.hubwin[v] : 0, nd = b.ndiff[v], lv = b.label[v];
            bool cand = st == tp || hw > 0;
            const int64_t s = b.off[v];
            const int deg = (int)(b.off[v + 1] - s);
            if (!cand) {
                int j = 0;
                for (; j < deg && !cand; j += 8) {  // eight ids, then their window stamps, in flight
                    int u[8], sv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) u[q] = j + q < deg ? __ldg(b.col + s + j + q) : -1;
#pragma unroll
                    for (int q = 0; q < 8; ++q) sv[q] = u[q] >= 0 ? b.sstamp[u[q]] : tp - 1;
#pragma unroll
                    for (int q = 0; q < 8; ++q) cand |= sv[q] == tp;
                }
                rd += (unsigned long long)(j < deg ? j : deg);
            }
            finish(i, v, cand, deg, nd, lv);
        }
    } else if ((int)blockIdx.x < a.g0 + a.g1) {
        // ---- pull, 32 vertices (deg in (kSmallDeg, kLargeDeg]) per warp: each lane checks the first 8 arcs
        //      of its row; the rows still undecided are walked by the whole warp, one after another ----
        const int wpb = blockDim.x >> 5;
        const int gw = ((int)blockIdx.x - a.g0) * wpb + (threadIdx.x >> 5), nw = a.g1 * wpb;
        for (int i0 = gw * 32; i0 < a.nb1; i0 += nw * 32) {
            const int i = i0 + lane;
            const bool valid = i < a.nb1;
            int v = 0, nd = 0, lv = 0;
            int64_t s = 0, e = 0;
            bool cand = false;
            if (valid) {
                v = b.bucket[1][i];
                const int st = b.sstamp[v], hw = a.hubwin ? b.hubwin[v] : 0;
                nd = b.ndiff[v];
                lv = b.label[v];
                s = b.off[v];
                e = b.off[v + 1];
                cand = st == tp || hw > 0;
                if (!cand) {  // deg > kSmallDeg >= 8: the first eight ids exist
                    int u[8], sv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) u[q] = __ldg(b.col + s + q);
#pragma unroll
                    for (int q = 0; q < 8; ++q) sv[q] = b.sstamp[u[q]];
#pragma unroll
                    for (int q = 0; q < 8; ++q) cand |= sv[q] == tp;
                    rd += 8;
                }
            }
            for (unsigned m = __ballot_sync(DMOLP_FULL_MASK, valid && !cand); m; m &= m - 1) {
                const int j = __ffs(m) - 1;
                const int64_t sj = __shfl_sync(DMOLP_FULL_MASK, s, j) + 8, ej = __shfl_sync(DMOLP_FULL_MASK, e, j);
                bool fs = false;
                const int64_t r = warp_row_wide(b.col, sj, ej, lane, [&](int u) { return b.sstamp[u]; },
                                                [&](int, int sv) { fs |= sv == tp; },
                                                [&] { return __any_sync(DMOLP_FULL_MASK, fs); });
                const bool cj = __any_sync(DMOLP_FULL_MASK, fs);
                if (lane == j) {
                    cand = cj;
                    rd += (unsigned long long)r;
                }
            }
            if (valid) finish(a.nb0 + i, v, cand, (int)(e - s), nd, lv);
        }
    } else {
        // ---- pull, block per vertex (deg > kLargeDeg) ----
        const int gb = (int)blockIdx.x - a.g0 - a.g1, nbk = (int)gridDim.x - a.g0 - a.g1;
        for (int i = gb; i < a.nb2; i += nbk) {
            const int pos = a.nb0 + a.nb1 + i;
            const int v = b.bucket[2][i];
            const bool cand0 = b.sstamp[v] == tp || (a.hubwin && b.hubwin[v] > 0);
            const int64_t s = b.off[v], e = b.off[v + 1];
            bool cand = cand0;
            int64_t j0 = s;
            if (!cand0) {  // block-uniform
                for (j0 = s; j0 < e; j0 += blockDim.x * 4) {
                    bool fs = false;
                    int u[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int64_t j = j0 + q * blockDim.x + threadIdx.x;
                        u[q] = j < e ? __ldcs(b.col + j) : -1;
                    }
                    int sv[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) sv[q] = u[q] >= 0 ? b.sstamp[u[q]] : tp - 1;
#pragma unroll
                    for (int q = 0; q < 4; ++q) fs |= sv[q] == tp;
                    if (__syncthreads_or(fs)) {
                        cand = true;
                        j0 += blockDim.x * 4;
                        break;
                    }
                }
            }
            if (threadIdx.x == 0) {
                if (!cand0) rd += (unsigned long long)((j0 < e ? j0 : e) - s);
                finish(pos, v, cand, (int)(e - s), b.ndiff[v], b.label[v]);
            }
            __syncthreads();
        }
    }
    block_atomic_add(te, &b.rec[a.t - 1].te_cand);
    block_atomic_add(rd, &b.rec[a.t - 1].arcs_bnd);
    block_atomic_add(nc, &b.cnt->ncand);
    block_atomic_add(nbd, &b.cnt->nbnd);
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x)
        if (s_npart[p]) atomicAdd(&b.npart[p], s_npart[p]);
    unsigned int *gh = a.dsup ? a.dsup : a.hist;
    for (int i = threadIdx.x; i < nhist; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&gh[i], s_hist[i]);
}

// ------------------------------------------------------------------------------------ decide
struct DecArgs {
    int t, eff;
    int wstride;    // shared ints per warp: lane-private counters (eff <= 32), histogram, or byte counters
    int hub_ready;  // the hubs' label counts are current (kept from the movers): decide them first
    int use_hot;    // count through colh and the block's copy of the hot labels (eff <= 32)
    int kept;       // non-hub vertices decide from their kept label counts (vcnt; eff <= 32)
};

// Label of a row entry u: a vertex id (u >= 0) or, in colh, the hot vertex of rank -(u + 2), whose label
// (clamped to 255) is in the block's shared copy s_hot.
__device__ __forceinline__ int nbr_label(const int32_t *__restrict__ label, const uint8_t *s_hot, int u) {
    return u >= 0 ? label[u] : (int)s_hot[-u - 2];
}

// The block's copy of the hot labels (all threads; ends with a barrier).
__device__ __forceinline__ void load_hot(const Buffers &b, uint8_t *s_hot) {
    const uint4 *src = reinterpret_cast<const uint4 *>(b.hotlab);
    uint4 *dst = reinterpret_cast<uint4 *>(s_hot);
    for (int i = threadIdx.x; i < kHotMax / 16; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

__device__ __forceinline__ void park_move(const Buffers &b, int v, int nl) {
    b.newlab[v] = nl;
    const int q = atomicAdd(&b.cnt->nchanged, 1);
    b.mov[q] = v;
}

// Work distribution of k_decide: lane 0 takes the next item of a class with one atomic; the result is
// broadcast only when the warp needs it, so the atomic's latency overlaps the current item.
__device__ __forceinline__ int grab_issue(int *ctr, int lane) { return lane == 0 ? atomicAdd(ctr, 1) : 0; }
__device__ __forceinline__ int grab_take(int pending) { return __shfl_sync(DMOLP_FULL_MASK, pending, 0); }

// Lane-private label counts (eff <= 32) of the arcs [s, e) of col (b.col, or colh with s_hot).
__device__ __forceinline__ void count_priv(const int32_t *__restrict__ col, const int32_t *__restrict__ label,
                                           const uint8_t *s_hot, int64_t s, int64_t e, int lane, int eff, int *h) {
    warp_row_wide(col, s, e, lane, [&](int u) { return nbr_label(label, s_hot, u); }, [&](int, int l) {
        if ((unsigned)l < (unsigned)eff) h[l * 32 + ((lane + l) & 31)] += 1;
    }, [] { return false; });
}

// Label counts of the arcs [s, e) into the warp's region: lane-private counters (eff <= 32) or a shared
// histogram of eff ints (warp_count's match-aggregated atomics).
// col / s_hot: as for count_priv (the eff > 32 histogram reads b.col).
__device__ __forceinline__ void count_row(const Buffers &b, const int32_t *col, const uint8_t *s_hot, int64_t s,
                                          int64_t e, int lane, int eff, int *h) {
    if (eff <= 32) {
        priv_zero(h, eff, lane);
        __syncwarp();
        count_priv(col, b.label, s_hot, s, e, lane, eff, h);
    } else {
        for (int c = lane; c < eff; c += 32) h[c] = 0;
        __syncwarp();
        warp_count(b.col, b.label, s, e, lane, eff, h);
    }
    __syncwarp();
}

// Hub rows (deg > kLargeDeg) in queued chunks of kHubChunk arcs, (list position, first arc) in b.hubq:
// warp per chunk, its label counts added to the hub's row of b.hh.
__device__ __forceinline__ void hub_chunks(const Buffers &b, const int32_t *col, const uint8_t *s_hot,
                                           const int32_t *list, int eff, int lane, int *h, unsigned long long &rd) {
    LpCounters *cn = b.cnt;
    const int n = cn->nhubq;
    int pend = grab_issue(&cn->dgrab[2], lane);
    for (;;) {
        const int q = grab_take(pend);
        if (q >= n) break;
        pend = grab_issue(&cn->dgrab[2], lane);
        const int2 ch = b.hubq[q];
        const int v = list[ch.x];
        const int64_t s = b.off[v] + ch.y, rowe = b.off[v + 1];
        const int64_t e = rowe - s > kHubChunk ? s + kHubChunk : rowe;
        count_row(b, col, s_hot, s, e, lane, eff, h);
        int32_t *row = b.hh + (size_t)b.hidx[v] * DMOLP_MAX_K;
        if (eff <= 32) {
            const int cnt = priv_total(h, eff, lane);
            if (cnt) atomicAdd(&row[lane], cnt);
        } else {
            for (int c = lane; c < eff; c += 32)
                if (h[c]) atomicAdd(&row[c], h[c]);
        }
        if (lane == 0) rd += (unsigned long long)(e - s);
        __syncwarp();
    }
}

// Decision of selected hub dec[2][i] from its row of label counts (warp; argmax over labels < eff); the
// hubs' arcs are summed for the next iteration's push / pull choice.
__device__ __forceinline__ void hub_decide(const Buffers &b, int i, int eff, int t, int lane) {
    const int v = b.dec[2][i];
    const int own = b.label[v];
    const int32_t *row = b.hh + (size_t)b.hidx[v] * DMOLP_MAX_K;
    double best;
    int blab;
    warp_argmax(eff, b.tpen, lane, [&](int c) { return row[c]; }, best, blab);
    if (lane == 0) {
        const double own_raw = (unsigned)own < (unsigned)eff ? (double)row[own] : -1e300;
        const int nl = best > own_raw ? blab : own;
        if (nl != own) park_move(b, v, nl);
        atomicAdd(&b.rec[t - 1].te_hubsel, (unsigned long long)(b.off[v + 1] - b.off[v]));
    }
}

// Persistent warps take the selected window's work largest items first: hub row chunks (none queued when
// the hub counts are kept current), then groups of warp-class vertices (metadata of the group loaded by
// its lanes in one step), then groups of 32 thread-class vertices (lane per vertex).
__global__ void __launch_bounds__(256, 4) k_decide(Buffers b, DecArgs a) {
    if (b.ctrl->stopped) return;
    extern __shared__ int shist[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int eff = a.eff;
    const bool priv = eff <= 32;
    int *h = shist + wib * a.wstride;
    uint8_t *s_hot = nullptr;
    const int32_t *col = b.col;
    if (a.use_hot) {  // block-uniform
        s_hot = reinterpret_cast<uint8_t *>(shist + kWarpsPerBlock * a.wstride);
        load_hot(b, s_hot);
        col = b.colh;
    }
    LpCounters *cn = b.cnt;
    unsigned long long rd = 0;

    if (a.hub_ready) {
        // ---- hub decisions from their kept label counts: warp per selected hub ----
        const int n = cn->ndec[2];
        int pend = grab_issue(&cn->dgrab[2], lane);
        for (;;) {
            const int q = grab_take(pend);
            if (q >= n) break;
            pend = grab_issue(&cn->dgrab[2], lane);
            hub_decide(b, q, eff, a.t, lane);
        }
    } else {
        hub_chunks(b, col, s_hot, b.dec[2], eff, lane, h, rd);
    }

    if (a.kept) {
        // ---- every other selected vertex from its kept label counts (vcnt): thread per vertex, 32 per
        //      item, the rule of warp_argmax over labels < eff in one thread.  The items cost the same, so
        //      warps stride over them (a shared claim counter would serialise one atomic per 32 vertices) ----
        const int n0 = cn->ndec[0], n = n0 + cn->ndec[1];
        const int ng = (n + 31) >> 5;
        const int nw = (int)gridDim.x * (int)(blockDim.x >> 5);
        for (int g = (int)blockIdx.x * (int)(blockDim.x >> 5) + wib; g < ng; g += nw) {  // warp-uniform
            const int i = g * 32 + lane;
            int v = 0, nl = 0;
            bool mv = false;
            if (i < n) {
                v = i < n0 ? b.dec[0][i] : b.dec[1][i - n0];
                const int own = b.label[v];
                const uint4 *src = reinterpret_cast<const uint4 *>(b.vcnt + (size_t)v * 32);
                // the 16 count words staged in the lane's row of the warp's shared counters (stride 17:
                // no bank conflicts), the labels with a nonzero count as a mask
                uint32_t *sw = reinterpret_cast<uint32_t *>(h) + lane * 17;
                uint32_t nz = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint4 x = src[q];
                    const uint32_t xw[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        sw[4 * q + r] = xw[r];
                        const uint32_t m2 = __vcmpne2(xw[r], 0u);  // 0xFFFF per nonzero half
                        nz |= ((m2 & 1u) | ((m2 >> 15) & 2u)) << (2 * (4 * q + r));
                    }
                }
                const uint32_t effm = eff >= 32 ? ~0u : (1u << eff) - 1u;
                nz &= effm;
                // argmax of (score, tie key) over labels < eff: the labels with neighbours first; those with
                // none score exactly 0 and can only win when nothing scored above 0
                double best = -DBL_MAX;
                int bkey = 0x7fffffff, blab = -1, own_cnt = 0;
                for (uint32_t m = nz; m; m &= m - 1) {
                    const int c = __ffs(m) - 1;
                    const int cnt = (int)((sw[c >> 1] >> ((c & 1) * 16)) & 0xFFFFu);
                    const double sc = __dmul_rn((double)cnt, __ldg(b.tpen + c));
                    const int key = tiekey(c);
                    if (better(sc, key, best, bkey)) {
                        best = sc;
                        bkey = key;
                        blab = c;
                    }
                    if (c == own) own_cnt = cnt;
                }
                const uint32_t zm = ~nz & effm;
                if (zm && !(best > 0.0)) {
                    for (uint32_t m = zm; m; m &= m - 1) {
                        const int c = __ffs(m) - 1;
                        const int key = tiekey(c);
                        if (better(0.0, key, best, bkey)) {
                            best = 0.0;
                            bkey = key;
                            blab = c;
                        }
                    }
                }
                const double own_raw = (unsigned)own < (unsigned)eff ? (double)own_cnt : -1e300;
                nl = best > own_raw ? blab : own;
                mv = nl != own;
            }
            // the warp's movers appended with one atomic (one per mover would serialise on the counter)
            const unsigned mm = __ballot_sync(DMOLP_FULL_MASK, mv);
            if (mm) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&b.cnt->nchanged, __popc(mm));
                base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
                if (mv) {
                    b.newlab[v] = nl;
                    b.mov[base + __popc(mm & ((1u << lane) - 1))] = v;
                }
            }
        }
    } else {
        // ---- warp per vertex, groups of G consecutive list entries per item ----
        {
            const int n = cn->ndec[1];
            const int nwarps = (int)gridDim.x * (int)(blockDim.x >> 5);
            int G = n / (nwarps * 4);
            G = G < 1 ? 1 : (G > 8 ? 8 : G);
            const int ng = (n + G - 1) / G;
            int pend = grab_issue(&cn->dgrab[1], lane);
            for (;;) {
                const int g = grab_take(pend);
                if (g >= ng) break;
                pend = grab_issue(&cn->dgrab[1], lane);
                const int i0 = g * G, m = n - i0 < G ? n - i0 : G;
                int gv = 0, gown = 0;
                int64_t gs = 0, ge = 0;
                if (lane < m) {
                    gv = b.dec[1][i0 + lane];
                    gown = b.label[gv];
                    gs = b.off[gv];
                    ge = b.off[gv + 1];
                }
                for (int j = 0; j < m; ++j) {
                    const int v = __shfl_sync(DMOLP_FULL_MASK, gv, j);
                    const int own = __shfl_sync(DMOLP_FULL_MASK, gown, j);
                    const int64_t s = __shfl_sync(DMOLP_FULL_MASK, gs, j), e = __shfl_sync(DMOLP_FULL_MASK, ge, j);
                    count_row(b, col, s_hot, s, e, lane, eff, h);
                    double best;
                    int blab, own_cnt;
                    if (priv) {
                        const int cnt = priv_total(h, eff, lane);
                        warp_argmax(eff, b.tpen, lane, [&](int) { return cnt; }, best, blab);
                        own_cnt = __shfl_sync(DMOLP_FULL_MASK, cnt, own & 31);
                    } else {
                        warp_argmax(eff, b.tpen, lane, [&](int c) { return h[c]; }, best, blab);
                        own_cnt = (unsigned)own < (unsigned)eff ? h[own] : 0;
                    }
                    if (lane == 0) {
                        rd += (unsigned long long)(e - s);
                        const double own_raw = (unsigned)own < (unsigned)eff ? (double)own_cnt : -1e300;
                        const int nl = best > own_raw ? blab : own;
                        if (nl != own) park_move(b, v, nl);
                    }
                    __syncwarp();
                }
            }
        }

        // ---- thread per vertex: deg <= kDecSmall, own label scored, eff <= kDecSmallK.  Label counts are
        //      bytes in this lane's column of the warp's region (word w of lane L at [w * 32 + L]: four labels
        //      per word, conflict-free); a 64-bit mask lists the labels seen, and only those are scored -- an
        //      absent label scores 0 <= count[own] and cannot win ----
        {
            const int n = cn->ndec[0];
            const int ng = (n + 31) >> 5;
            uint32_t *cw = reinterpret_cast<uint32_t *>(h) + lane;
            if (ng > 0)
                for (int w = 0; w < kDecSmallK / 4; ++w) cw[w * 32] = 0u;
            int pend = grab_issue(&cn->dgrab[0], lane);
            for (;;) {
                const int g = grab_take(pend);
                if (g >= ng) break;
                pend = grab_issue(&cn->dgrab[0], lane);
                const int i = g * 32 + lane;
                if (i >= n) continue;
                const int v = b.dec[0][i];
                const int own = b.label[v];
                const int64_t s = b.off[v];
                const int deg = (int)(b.off[v + 1] - s);
                rd += deg;
                unsigned long long seen = 0ull;
                for (int j = 0; j < deg; j += 8) {
                    int u[8], l[8];
    #pragma unroll
                    for (int q = 0; q < 8; ++q) u[q] = j + q < deg ? __ldg(col + s + j + q) : kNoArc;
    #pragma unroll
                    for (int q = 0; q < 8; ++q) l[q] = u[q] != kNoArc ? nbr_label(b.label, s_hot, u[q]) : -1;
    #pragma unroll
                    for (int q = 0; q < 8; ++q)
                        if ((unsigned)l[q] < (unsigned)eff) {
                            cw[(l[q] >> 2) * 32] += 1u << ((l[q] & 3) * 8);
                            seen |= 1ull << l[q];
                        }
                }
                const int own_cnt = (int)((cw[(own >> 2) * 32] >> ((own & 3) * 8)) & 0xFFu);
                double best = -DBL_MAX;
                int bkey = 0x7fffffff, blab = -1;
                for (unsigned long long m = seen; m; m &= m - 1) {
                    const int c = __ffsll((long long)m) - 1;
                    const int cnt = (int)((cw[(c >> 2) * 32] >> ((c & 3) * 8)) & 0xFFu);
                    const double sc = __dmul_rn((double)cnt, b.tpen[c]);
                    const int key = tiekey(c);
                    if (better(sc, key, best, bkey)) {
                        best = sc;
                        bkey = key;
                        blab = c;
                    }
                }
                for (unsigned long long m = seen; m; m &= m - 1) cw[((__ffsll((long long)m) - 1) >> 2) * 32] = 0u;
                if (blab >= 0 && best > (double)own_cnt && blab != own) park_move(b, v, blab);
            }
        }
    }
    // per warp (no block barrier: the decisions' dynamic shared memory already takes the whole 48 KB)
    rd = warp_sum_u64(rd);
    if (lane == 0 && rd) atomicAdd(&b.rec[a.t - 1].arcs_dec, rd);
}

// Hub rows queued in kHubChunk pieces for hub_chunks, with each hub's count row cleared: the selected hubs
// (list = dec[2], n = ndec[2]) before k_decide, or every hub (list = bucket[2]) at the start of a run.
__device__ __forceinline__ void hub_queue(const Buffers &b, const int32_t *list, int n, int eff) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < n; i += nw) {
        const int v = list[i];
        int32_t *row = b.hh + (size_t)b.hidx[v] * DMOLP_MAX_K;
        for (int c = lane; c < eff; c += 32) row[c] = 0;
        const int64_t deg = b.off[v + 1] - b.off[v];
        const int nch = (int)((deg + kHubChunk - 1) / kHubChunk);
        int base = 0;
        if (lane == 0) base = atomicAdd(&b.cnt->nhubq, nch);
        base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
        for (int c = lane; c < nch; c += 32) b.hubq[base + c] = make_int2(i, c * kHubChunk);
    }
}

__global__ void k_hub_prep(Buffers b, int eff) {
    if (b.ctrl->stopped) return;
    hub_queue(b, b.dec[2], b.cnt->ndec[2], eff);
}

__global__ void k_hub_index(Buffers b, int nhub) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nhub; i += gridDim.x * blockDim.x)
        b.hidx[b.bucket[2][i]] = i;
}

// Hub decisions after k_decide summed the chunks of their rows: warp per hub.
__global__ void k_hub_final(Buffers b, int eff, int t) {
    if (b.ctrl->stopped) return;
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int n = b.cnt->ndec[2];
    for (int i = gw; i < n; i += nw) hub_decide(b, i, eff, t, lane);
}

// ------------------------------------------------------------------------------------ update
// Warp per mover v (old label a = label[v], new label c = newlab[v]).  For each arc (v,u), with u's old
// label lo = label[u] and new label ln (newlab[u] if u moves, else lo), the arc leaves the cut count
// [a != lo] and the intra count of a if a == lo, and enters them with (c, ln).  Weight 2 when u stays:
// the reverse arc (u,v) changes the same way but is never visited; weight 1 when u moves (or u == v):
// (u,v) is visited from u's side.  Vertex counts move by one.  A hub neighbour u sees v's label go from
// a to c: its row of label counts (labels < eff) moves by one.
constexpr int kUpdLaneRow = 32;  // k_update: rows of at most this many arcs are walked by one lane ...
constexpr int kUpdLaneMin = 8;   // ... when there are at least this many movers per warp

__global__ void __launch_bounds__(256, 2) k_update(Buffers b, int k, int eff, int t, int keep) {
    if (b.ctrl->stopped) return;
    extern __shared__ unsigned long long sacc[];  // [2k]: vertex-count deltas, intra-arc deltas
    for (int p = threadIdx.x; p < 2 * k; p += blockDim.x) sacc[p] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int n = b.cnt->nchanged;
    long long dcut = 0;
    unsigned long long rd = 0;
    // arc (v, u) of a mover v from label a to c, u's labels g = (old, pending or -1, hub index or -1)
    auto arc = [&](int u, int3 g, int a, int c, long long &in_c, long long &out_a, int &dv) {
        const int lo = g.x;
        const int nu = g.y;
        const int ln = nu >= 0 ? nu : lo;
        const int w = nu >= 0 ? 1 : 2;
        dcut += w * ((int)(c != ln) - (int)(a != lo));
        in_c += w * (int)(c == ln);
        out_a += w * (int)(a == lo);
        // differently-labelled neighbour counts: arc (u,v) seen from u; arc (v,u) from v when u stays
        // (a moving u updates v's count from its own row)
        const int du = (int)(ln != c) - (int)(lo != a);
        if (du) atomicAdd(&b.ndiff[u], du);
        if (nu < 0) dv += (int)(c != lo) - (int)(a != lo);
        const int hu = g.z;
        if (hu >= 0) {
            int32_t *row = b.hh + (size_t)hu * DMOLP_MAX_K;
            if ((unsigned)a < (unsigned)eff) atomicAdd(&row[a], -1);
            if ((unsigned)c < (unsigned)eff) atomicAdd(&row[c], 1);
        } else if (keep) {
            // u's 16-bit counts, two per word: a count leaves label a (it is >= 1: it counts v) and
            // enters label c (it stays <= deg(u) <= kLargeDeg), so no carry or borrow crosses a half
            uint32_t *wd = reinterpret_cast<uint32_t *>(b.vcnt + (size_t)u * 32);
            const bool ia = (unsigned)a < (unsigned)eff, ic = (unsigned)c < (unsigned)eff;
            const uint32_t da = 1u << ((a & 1) * 16), dcn = 1u << ((c & 1) * 16);
            if (ia && ic && (a >> 1) == (c >> 1)) {
                atomicAdd(&wd[a >> 1], dcn - da);
            } else {
                if (ia) atomicSub(&wd[a >> 1], da);
                if (ic) atomicAdd(&wd[c >> 1], dcn);
            }
        }
    };
    auto gather = [&](int u) { return make_int3(b.label[u], b.newlab[u], b.hidx[u]); };
    // a mover's row walked by the whole warp (all lanes call it)
    auto warp_mover = [&](int vj, int aj, int cj, int64_t sj, int64_t ej) {
        long long in_c = 0, out_a = 0;
        int dv = 0;
        warp_row_wide(b.col, sj, ej, lane, gather, [&](int u, int3 g) { arc(u, g, aj, cj, in_c, out_a, dv); },
                      [] { return false; });
        for (int o = 16; o > 0; o >>= 1) {
            in_c += __shfl_xor_sync(DMOLP_FULL_MASK, in_c, o);
            out_a += __shfl_xor_sync(DMOLP_FULL_MASK, out_a, o);
            dv += __shfl_xor_sync(DMOLP_FULL_MASK, dv, o);
        }
        if (lane == 0) {
            if (dv) atomicAdd(&b.ndiff[vj], dv);
            rd += (unsigned long long)(ej - sj);
            atomicAdd(&sacc[aj], (unsigned long long)(-1ll));
            atomicAdd(&sacc[cj], 1ull);
            if (in_c) atomicAdd(&sacc[k + cj], (unsigned long long)in_c);
            if (out_a) atomicAdd(&sacc[k + aj], (unsigned long long)(-out_a));
        }
    };
    if (n < nw * kUpdLaneMin) {
        // few movers: one per warp at a time, its row spread over the lanes
        for (int i = gw; i < n; i += nw) {
            const int v = b.mov[i];
            warp_mover(v, b.label[v], b.newlab[v], b.off[v], b.off[v + 1]);
        }
    } else {
        // many movers: 32 per warp and step; a row of at most kUpdLaneRow arcs is walked by its lane alone
        // (four arcs in flight), longer rows by the whole warp one after another
        for (int i0 = gw * 32; i0 < n; i0 += nw * 32) {
            const int i = i0 + lane;
            const bool valid = i < n;
            int v = 0, a = 0, c = 0;
            int64_t s = 0, e = 0;
            if (valid) {
                v = b.mov[i];
                a = b.label[v];
                c = b.newlab[v];
                s = b.off[v];
                e = b.off[v + 1];
            }
            const bool mine = valid && e - s <= kUpdLaneRow;
            if (mine) {
                long long in_c = 0, out_a = 0;
                int dv = 0;
                for (int64_t j0 = s; j0 < e; j0 += 4) {
                    int u[4];
                    int3 g[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) u[q] = j0 + q < e ? __ldg(b.col + j0 + q) : -1;
#pragma unroll
                    for (int q = 0; q < 4; ++q) g[q] = u[q] >= 0 ? gather(u[q]) : make_int3(0, -1, -1);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (u[q] >= 0) arc(u[q], g[q], a, c, in_c, out_a, dv);
                }
                if (dv) atomicAdd(&b.ndiff[v], dv);
                rd += (unsigned long long)(e - s);
                atomicAdd(&sacc[a], (unsigned long long)(-1ll));
                atomicAdd(&sacc[c], 1ull);
                if (in_c) atomicAdd(&sacc[k + c], (unsigned long long)in_c);
                if (out_a) atomicAdd(&sacc[k + a], (unsigned long long)(-out_a));
            }
            for (unsigned m = __ballot_sync(DMOLP_FULL_MASK, valid && !mine); m; m &= m - 1) {
                const int jl = __ffs(m) - 1;
                warp_mover(__shfl_sync(DMOLP_FULL_MASK, v, jl), __shfl_sync(DMOLP_FULL_MASK, a, jl),
                           __shfl_sync(DMOLP_FULL_MASK, c, jl), __shfl_sync(DMOLP_FULL_MASK, s, jl),
                           __shfl_sync(DMOLP_FULL_MASK, e, jl));
            }
        }
    }
    block_atomic_add((unsigned long long)dcut, &b.cnt->cut_arcs);  // the sum is taken mod 2^64: negative deltas add
    block_atomic_add(rd, &b.rec[t - 1].arcs_upd);
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        if (sacc[p]) atomicAdd(&b.vc[p], sacc[p]);
        if (sacc[k + p]) atomicAdd(&b.intra[p], sacc[k + p]);
    }
}

// Movers take their labels.
__global__ void k_apply(Buffers b) {
    if (b.ctrl->stopped) return;
    const int n = b.cnt->nchanged;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int v = b.mov[i];
        const int nl = b.newlab[v];
        b.label[v] = nl;
        b.newlab[v] = -1;
        const int r = b.hrank[v];
        if (r >= 0) b.hotlab[r] = (unsigned)nl < 255u ? (uint8_t)nl : (uint8_t)255;
    }
}

// ------------------------------------------------------------------------------------ stats
// The fused edge-cut / balance pass over all vertices: label counts (all vertices, coalesced), and per
// degree class the same-label and cut arcs.  Block ranges: [0,gv) vertex counts, then the three classes.
struct StatsArgs {
    int k, nv, gv, g0, g1, nb0, nb1, nb2;
    int use_hot;   // rows through colh and the block's copy of the hot labels (k <= 255)
    int keep_eff;  // > 0: write vcnt, the counts of labels < keep_eff (<= 32), of every non-hub vertex
    int hub_eff;   // > 0: write hh, every hub's counts of labels < hub_eff (the run start on symmetric graphs)
};

constexpr int kStatsLaneRow = 64;  // k_stats: rows of at most this many arcs are walked by one lane

__global__ void __launch_bounds__(256, 4) k_stats(Buffers b, StatsArgs a, const int *stopped, const int *skip) {
    if ((stopped && *stopped) || (skip && *skip)) return;
    extern __shared__ unsigned long long sacc[];  // [2k]: vertex counts, intra arcs; then the hot labels
    const int k = a.k;
    unsigned long long *svc = sacc, *sin = sacc + k;
    for (int p = threadIdx.x; p < 2 * k; p += blockDim.x) sacc[p] = 0;
    const uint8_t *s_hot = nullptr;
    const int32_t *col = b.col;
    if (a.use_hot) {  // block-uniform
        uint8_t *sh = reinterpret_cast<uint8_t *>(sacc + 2 * k);
        load_hot(b, sh);
        s_hot = sh;
        col = b.colh;
    }
    // kept counts of the rows a lane walks alone: byte counters (word w of thread t at s_kc[w * 256 + t])
    uint32_t *s_kc = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(sacc + 2 * k) + (a.use_hot ? kHotMax : 0));
    if (a.keep_eff)
        for (int i = threadIdx.x; i < 8 * kBlock; i += blockDim.x) s_kc[i] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned long long cut = 0;
    bool bad = false;
    // logical block ranges [vertex counts | thread class | warp class | hub rows], dispatched hub rows first
    // so that the longest rows start in the first wave, then the warp class, the thread class, the counts
    int bx;
    {
        const int r = blockIdx.x, g2 = (int)gridDim.x - a.gv - a.g0 - a.g1;
        if (r < g2) bx = a.gv + a.g0 + a.g1 + r;
        else if (r < g2 + a.g1) bx = a.gv + a.g0 + (r - g2);
        else if (r < g2 + a.g1 + a.g0) bx = a.gv + (r - g2 - a.g1);
        else bx = r - g2 - a.g1 - a.g0;
    }
    if (bx < a.gv) {  // whole warps iterate: the lanes sharing a label add once
        for (int v0 = bx * blockDim.x + (threadIdx.x & ~31); v0 < a.nv; v0 += a.gv * blockDim.x) {
            const int v = v0 + lane;
            const int lv = v < a.nv ? b.label[v] : -1;
            const bool ok = (unsigned)lv < (unsigned)k;
            bad |= v < a.nv && !ok;
            const unsigned m = __match_any_sync(DMOLP_FULL_MASK, ok ? lv : -1);
            if (ok && lane == __ffs(m) - 1) atomicAdd(&svc[lv], (unsigned long long)__popc(m));
        }
    } else if (bx < a.gv + a.g0 + a.g1) {
        // thread class: a lane per row; warp class: rows of at most kStatsLaneRow arcs a lane each too, longer
        // rows by the whole warp (one after another)
        const bool cls0 = bx < a.gv + a.g0;
        // one lane's row: eight ids, then their eight labels, in flight; byte counters for the kept counts
        auto lane_row = [&](int v, int64_t s, int deg, int lv) {
            unsigned int same = 0, diff = 0;
            for (int j = 0; j < deg; j += 8) {
                int u[8], l[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) u[q] = j + q < deg ? __ldg(col + s + j + q) : kNoArc;
#pragma unroll
                for (int q = 0; q < 8; ++q) l[q] = u[q] != kNoArc ? nbr_label(b.label, s_hot, u[q]) : lv;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (u[q] != kNoArc) {
                        bad |= (unsigned)l[q] >= (unsigned)k;
                        same += (l[q] == lv);
                        diff += (l[q] != lv);
                        if ((unsigned)l[q] < (unsigned)a.keep_eff)
                            s_kc[(l[q] >> 2) * kBlock + threadIdx.x] += 1u << ((l[q] & 3) * 8);
                    }
            }
            cut += diff;
            b.ndiff[v] = (int)diff;
            if (same && (unsigned)lv < (unsigned)k) atomicAdd(&sin[lv], (unsigned long long)same);
            if (a.keep_eff) {  // the byte counters (deg <= kStatsLaneRow) widened to 32 u16, cleared for the next row
                uint32_t w[16];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const uint32_t x = s_kc[q * kBlock + threadIdx.x];
                    s_kc[q * kBlock + threadIdx.x] = 0u;
                    w[2 * q] = (x & 0xFFu) | ((x & 0xFF00u) << 8);
                    w[2 * q + 1] = ((x >> 16) & 0xFFu) | ((x >> 8) & 0xFF0000u);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(b.vcnt + (size_t)v * 32);
#pragma unroll
                for (int q = 0; q < 4; ++q) dst[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
            }
        };
        if (cls0) {
            for (int i = (bx - a.gv) * blockDim.x + threadIdx.x; i < a.nb0; i += a.g0 * blockDim.x) {
                const int v = b.bucket[0][i];
                const int64_t s = b.off[v];
                lane_row(v, s, (int)(b.off[v + 1] - s), b.label[v]);
            }
        } else {
            const int wpb = blockDim.x >> 5;
            const int gw = (bx - a.gv - a.g0) * wpb + wib, nw = a.g1 * wpb;
            for (int i0 = gw * 32; i0 < a.nb1; i0 += nw * 32) {
                const int i = i0 + lane;
                const bool valid = i < a.nb1;
                int v = 0, lv = 0;
                int64_t s = 0, e = 0;
                if (valid) {
                    v = b.bucket[1][i];
                    lv = b.label[v];
                    s = b.off[v];
                    e = b.off[v + 1];
                }
                const bool mine = valid && e - s <= kStatsLaneRow;
                if (mine) lane_row(v, s, (int)(e - s), lv);
                for (unsigned m = __ballot_sync(DMOLP_FULL_MASK, valid && !mine); m; m &= m - 1) {
                    const int jl = __ffs(m) - 1;
                    const int vj = __shfl_sync(DMOLP_FULL_MASK, v, jl), lvj = __shfl_sync(DMOLP_FULL_MASK, lv, jl);
                    const int64_t sj = __shfl_sync(DMOLP_FULL_MASK, s, jl), ej = __shfl_sync(DMOLP_FULL_MASK, e, jl);
                    unsigned int same = 0, diff = 0;
                    // kept counts: lane c counts label c.  Per slot of a step, five votes on the bits of the
                    // lanes' labels select the lanes holding label c (bit-sliced compare), no shared atomics:
                    // neighbours mostly share a label, which would serialise atomics on one counter.
                    int mycnt = 0;
                    warp_row_wide_all(col, sj, ej, lane, 0, [&](int u) { return nbr_label(b.label, s_hot, u); },
                                      [&](int u, int lu) {
                        if (u != kNoArc) {
                            bad |= (unsigned)lu >= (unsigned)k;
                            same += (lu == lvj);
                            diff += (lu != lvj);
                        }
                        if (a.keep_eff) {  // kernel-uniform
                            unsigned sel = __ballot_sync(DMOLP_FULL_MASK, u != kNoArc && (unsigned)lu < (unsigned)a.keep_eff);
                            if (sel) {  // warp-uniform
#pragma unroll
                                for (int bit = 0; bit < 5; ++bit) {
                                    const unsigned bb = __ballot_sync(DMOLP_FULL_MASK, (lu >> bit) & 1);
                                    sel &= ((lane >> bit) & 1) ? bb : ~bb;
                                }
                                mycnt += __popc(sel);
                            }
                        }
                    });
                    if (a.keep_eff)  // lane c writes the count of label c (deg <= kLargeDeg fits 16 bits)
                        b.vcnt[(size_t)vj * 32 + lane] = (uint16_t)mycnt;
                    for (int o = 16; o > 0; o >>= 1) {
                        same += __shfl_xor_sync(DMOLP_FULL_MASK, same, o);
                        diff += __shfl_xor_sync(DMOLP_FULL_MASK, diff, o);
                    }
                    if (lane == 0) {
                        cut += diff;
                        b.ndiff[vj] = (int)diff;
                        if (same && (unsigned)lvj < (unsigned)k) atomicAdd(&sin[lvj], (unsigned long long)same);
                    }
                }
            }
        }
    } else {
        __shared__ unsigned int s_diff[8];
        __shared__ int s_hcw[kWarpsPerBlock][32];  // hub label counts per warp (hub_eff <= 32)
        int *s_hc = reinterpret_cast<int *>(s_kc);  // [hub_eff] block counts (hub_eff > 32; keep_eff is 0 then)
        const int heff = a.hub_eff;
        const int gb = bx - a.gv - a.g0 - a.g1, nbk = (int)gridDim.x - a.gv - a.g0 - a.g1;
        for (int i = gb; i < a.nb2; i += nbk) {
            const int v = b.bucket[2][i];
            const int lv = b.label[v];
            const int64_t s = b.off[v], e = b.off[v + 1];
            unsigned int same = 0, diff = 0;
            int mycnt = 0;  // hub_eff <= 32: lane c counts label c (bit-sliced votes per slot)
            if (heff > 32) {
                for (int c = threadIdx.x; c < heff; c += blockDim.x) s_hc[c] = 0;
                __syncthreads();
            }
            for (int64_t j0 = s; j0 < e; j0 += 4 * blockDim.x) {  // four ids per thread, then their labels
                int u[4], l[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int64_t j = j0 + q * blockDim.x + threadIdx.x;
                    u[q] = j < e ? __ldcs(col + j) : kNoArc;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) l[q] = u[q] != kNoArc ? nbr_label(b.label, s_hot, u[q]) : lv;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (u[q] != kNoArc) {
                        bad |= (unsigned)l[q] >= (unsigned)k;
                        same += (l[q] == lv);
                        diff += (l[q] != lv);
                    }
                if (heff > 32) {  // kernel-uniform
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (u[q] != kNoArc && (unsigned)l[q] < (unsigned)heff) atomicAdd(&s_hc[l[q]], 1);
                } else if (heff > 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        unsigned sel = __ballot_sync(DMOLP_FULL_MASK, u[q] != kNoArc && (unsigned)l[q] < (unsigned)heff);
                        if (sel) {  // warp-uniform
#pragma unroll
                            for (int bit = 0; bit < 5; ++bit) {
                                const unsigned bb = __ballot_sync(DMOLP_FULL_MASK, (l[q] >> bit) & 1);
                                sel &= ((lane >> bit) & 1) ? bb : ~bb;
                            }
                            mycnt += __popc(sel);
                        }
                    }
                }
            }
            if (heff > 0) {  // the hub's row of label counts, written whole (labels < hub_eff)
                int32_t *row = b.hh + (size_t)b.hidx[v] * DMOLP_MAX_K;
                if (heff <= 32) s_hcw[wib][lane] = mycnt;
                __syncthreads();
                if (heff <= 32) {
                    if ((int)threadIdx.x < heff) {
                        int t = 0;
                        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_hcw[w][threadIdx.x];
                        row[threadIdx.x] = t;
                    }
                } else {
                    for (int c = threadIdx.x; c < heff; c += blockDim.x) row[c] = s_hc[c];
                }
                __syncthreads();
            }
            cut += diff;
            for (int o = 16; o > 0; o >>= 1) {
                same += __shfl_xor_sync(DMOLP_FULL_MASK, same, o);
                diff += __shfl_xor_sync(DMOLP_FULL_MASK, diff, o);
            }
            if (lane == 0 && same && (unsigned)lv < (unsigned)k) atomicAdd(&sin[lv], (unsigned long long)same);
            if (lane == 0) s_diff[wib] = diff;
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned int t = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_diff[w];
                b.ndiff[v] = (int)t;
            }
            __syncthreads();
        }
    }
    if (__any_sync(DMOLP_FULL_MASK, bad) && lane == 0) b.ctrl->error = 1;
    block_atomic_add(cut, &b.cnt->cut_arcs);
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        if (svc[p]) atomicAdd(&b.vc[p], svc[p]);
        if (sin[p]) atomicAdd(&b.intra[p], sin[p]);
    }
}

// ------------------------------------------------------------------------------------ hot set
// degh[min(deg, 65535)] for every vertex with arcs; degrees below kHotHistLow in a block histogram first.
constexpr int kHotHistLow = 4096;
__global__ void k_hot_hist(Buffers b, int nv) {
    __shared__ unsigned int sh[kHotHistLow];
    for (int i = threadIdx.x; i < kHotHistLow; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        const int64_t d = b.off[v + 1] - b.off[v];
        if (d <= 0) continue;
        if (d < kHotHistLow) atomicAdd(&sh[d], 1u);
        else atomicAdd(&b.degh[d < 65535 ? d : 65535], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kHotHistLow; i += blockDim.x)
        if (sh[i]) atomicAdd(&b.degh[i], sh[i]);
}

// Vertices of degree >= dstar get ranks (b.flag counts them; the order of ranks is immaterial).
__global__ void k_hot_assign(Buffers b, int nv, int dstar) {
    for (int v0 = blockIdx.x * blockDim.x; v0 < nv; v0 += gridDim.x * blockDim.x) {
        const int v = v0 + threadIdx.x;
        const bool hot = v < nv && b.off[v + 1] - b.off[v] >= dstar;
        const int r = warp_append(b.flag, hot);
        if (hot) {
            b.hrank[v] = r;
            b.hotid[r] = v;
        }
    }
}

// colh = col with hot neighbours written as -(rank + 2).
__global__ void k_hot_encode(Buffers b, long long narcs) {
    const long long n4 = narcs >> 2;
    const int4 *c4 = reinterpret_cast<const int4 *>(b.col);
    int4 *h4 = reinterpret_cast<int4 *>(b.colh);
    auto enc = [&](int u) {
        const int r = b.hrank[u];
        return r >= 0 ? -(r + 2) : u;
    };
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
        const int4 x = __ldcs(c4 + i);
        h4[i] = make_int4(enc(x.x), enc(x.y), enc(x.z), enc(x.w));
    }
    for (long long j = (n4 << 2) + blockIdx.x * (long long)blockDim.x + threadIdx.x; j < narcs;
         j += (long long)gridDim.x * blockDim.x)
        b.colh[j] = enc(b.col[j]);
}

// Hot labels from the resident labels, clamped to 255.
__global__ void k_hot_refresh(Buffers b, int nhot) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nhot; r += gridDim.x * blockDim.x) {
        const int l = b.label[b.hotid[r]];
        b.hotlab[r] = (unsigned)l < 255u ? (uint8_t)l : (uint8_t)255;
    }
}

// ------------------------------------------------------------------------------------ end
// End of iteration t (one block; the scalar part on thread 0): the iteration record, the stopping rules of
// run_phase2 (phase2.cpp:309-415), the next iteration's candidate mode.
__device__ void lp_end(const Buffers &b, int k, int t, long long narcs, int mode, int symmetric) {
    LpControl *ctl = b.ctrl;
    LpCounters *cn = b.cnt;
    long long *ch = b.cnthist + (size_t)(t - 1) * 2 * DMOLP_MAX_K;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        ch[p] = sll(b.vc[p]);
        ch[DMOLP_MAX_K + p] = sll(b.intra[p]) / 2;
    }
    if (threadIdx.x != 0) return;
    LpRecordDev &r = b.rec[t - 1];
    r.window = cn->nwin[t & 1];
    r.candidates = t == 1 ? -1 : cn->ncand;
    r.changes = cn->nchanged;
    r.boundary = cn->nbnd;
    bool stats = true;
    if (r.window == 0) {
        stats = false;
        if (mode == DMOLP_LP_MODE_REF) ctl->stop_now = 1;
    } else if (r.changes == 0 && mode == DMOLP_LP_MODE_REF) {
        stats = false;
        ctl->stop_now = 2;
    }
    if (stats) {
        const unsigned long long arcs = cn->cut_arcs;
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
            if (mode == DMOLP_LP_MODE_REF && ctl->conv >= 10) ctl->stop_now = 3;
        }
    }
    r.edge_cut = ctl->prev_cut;
    ctl->iters_run = t;
    // the next iteration pulls unless pushing would walk fewer than 1/16 of all arcs (pulling finds the
    // same candidates only when every arc has its reverse); hub rows are not walked by the push.  Pulling
    // mostly stops at a row's first arcs, so it wins until the window is small (measured on R-MAT 22).
    ctl->pull = symmetric && (r.te_sel - r.te_hubsel) * 16ull > (unsigned long long)narcs;
    if (ctl->stop_now) {
        ctl->stopped = 1;
        ctl->stop_reason = ctl->stop_now;
    }
}

// Between iterations, one block: the end of iteration t_end (when > 0), then, unless that stopped the
// loop, the start of iteration t_begin (when > 0).
__global__ void k_lp_turn(Buffers b, int k, int t_end, int t_begin, long long narcs, int mode, int symmetric) {
    __shared__ int s_stopped;
    __shared__ double s_re[DMOLP_MAX_K], s_tp[DMOLP_MAX_K];
    if (threadIdx.x == 0) s_stopped = b.ctrl->stopped;
    __syncthreads();
    if (s_stopped) return;
    if (t_end > 0) {
        lp_end(b, k, t_end, narcs, mode, symmetric);
        __syncthreads();
        if (threadIdx.x == 0) s_stopped = b.ctrl->stopped;
        __syncthreads();
        if (s_stopped) return;
    }
    if (t_begin > 0) lp_begin(b, k, t_begin, narcs, s_re, s_tp);
}

// Asymmetric graphs: decide whether the full statistics pass runs (the reference skips it on an empty
// window and, with its stopping rules, on zero changes) and clear its accumulators.
__global__ void k_lp_mid(Buffers b, int k, int t, int mode) {
    LpControl *ctl = b.ctrl;
    if (ctl->stopped) return;
    __shared__ int s_skip;
    if (threadIdx.x == 0) {
        const int win = b.cnt->nwin[t & 1], ch = b.cnt->nchanged;
        const int skip = (win == 0) || (ch == 0 && mode == DMOLP_LP_MODE_REF);
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

__global__ void k_lp_init_end(Buffers b, int mode) {
    LpControl *ctl = b.ctrl;
    const unsigned long long arcs = b.cnt->cut_arcs;
    ctl->mode = mode;
    ctl->conv = 0;
    ctl->iters_run = 0;
    ctl->stop_reason = 0;
    ctl->stop_now = 0;
    ctl->skip_stats = 0;
    ctl->pull = 0;
    ctl->prev_cut = (long long)(arcs >> 1);
    if ((arcs & 1ull) || ctl->error) {
        ctl->error = 1;
        ctl->stopped = 1;
        ctl->stop_reason = 4;
    } else {
        ctl->stopped = 0;
    }
}

__global__ void k_reset_stats(Buffers b, int k, int clear_error) {
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        b.vc[p] = 0;
        b.intra[p] = 0;
    }
    if (threadIdx.x == 0) {
        b.cnt->cut_arcs = 0;
        if (clear_error) b.ctrl->error = 0;
    }
}

// ---- stand-alone pieces (dmolp_window_select / dmolp_lp_apply) ----
__global__ void k_ws_begin(Buffers b, int k, int t, int nprev) {
    for (int p = threadIdx.x; p < k; p += blockDim.x) b.npart[p] = 0;
    if (threadIdx.x == 0) {
        LpCounters *cn = b.cnt;
        cn->ncand = cn->nbnd = cn->nchanged = cn->nchunk = 0;
        cn->ndec[0] = cn->ndec[1] = cn->ndec[2] = 0;
        cn->nwin[(t - 1) & 1] = nprev;
        cn->nwin[t & 1] = 0;
        b.ctrl->stopped = 0;
        b.ctrl->pull = 0;
        LpRecordDev &r = b.rec[t - 1];
        r.te_prev = r.te_cand = r.te_sel = r.te_stats = 0;
        r.arcs_bnd = r.arcs_dec = r.arcs_upd = 0;
        r.win_sum = 0;
    }
}

// An explicit window (n vertices in b.cand) sorted into decision classes.
__global__ void k_classify(Buffers b, int n, int eff) {
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        int cls = -1, v = 0;
        if (i < n) {
            v = b.cand[i];
            const int deg = (int)(b.off[v + 1] - b.off[v]);
            const int own = b.label[v];
            cls = dec_class(deg, own, eff);
        }
        for (int c = 0; c < 3; ++c) {
            const int s2 = warp_append(&b.cnt->ndec[c], cls == c);
            if (cls == c) b.dec[c][s2] = v;
        }
    }
}

__global__ void k_zero_small(Buffers b) {
    LpCounters *cn = b.cnt;
    cn->ndec[0] = cn->ndec[1] = cn->ndec[2] = 0;
    cn->nhubq = 0;
    cn->dgrab[0] = cn->dgrab[1] = cn->dgrab[2] = 0;
    cn->nchanged = 0;
    b.ctrl->stopped = 0;
}

// Movers of dmolp_lp_apply as (vertex, label) pairs into bv/bnew.
__global__ void k_collect_moves(Buffers b) {
    const int n = b.cnt->nchanged;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int v = b.mov[i];
        b.bv[i] = v;
        b.bnew[i] = b.newlab[v];
    }
}

// Symmetry of the uploaded graph (rows strictly increasing).  Each arc (u,v), u != v, is looked up from its
// larger endpoint only -- (degree, id) of u above v's: u must be in v's (shorter) row, by binary search.  The
// other arcs are only counted.  With no duplicates the found reverses are distinct arcs, so the graph is
// symmetric iff every lookup succeeds and both counts agree (flag[0] = missing, cnt[0..1] = the counts).
template <int U>
__device__ __forceinline__ void sym_arcs(const Buffers &b, int u, int64_t du, const int *v, bool &missing,
                                         unsigned long long &big, unsigned long long &small) {
    // U arcs (u, v[q]) at once (v[q] < 0: no arc): their rows' bounds loaded together, then lower-bound
    // searches for u advanced in lockstep, so U independent loads are in flight per step
    int64_t lo[U], hi[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
        lo[q] = v[q] >= 0 ? b.off[v[q]] : 0;
        hi[q] = v[q] >= 0 ? b.off[v[q] + 1] : 0;
    }
    bool srch[U];
    int64_t e[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
        const int64_t dv = hi[q] - lo[q];
        srch[q] = false;
        e[q] = hi[q];
        if (v[q] >= 0 && v[q] != u) {
            if (du > dv || (du == dv && u > v[q])) {
                ++big;
                srch[q] = true;
            } else {
                ++small;
            }
        }
        if (!srch[q]) lo[q] = hi[q];
    }
    for (;;) {
        bool any = false;
        int x[U];
#pragma unroll
        for (int q = 0; q < U; ++q) x[q] = lo[q] < hi[q] ? __ldg(b.col + ((lo[q] + hi[q]) >> 1)) : 0;
#pragma unroll
        for (int q = 0; q < U; ++q) {
            if (lo[q] < hi[q]) {
                const int64_t mid = (lo[q] + hi[q]) >> 1;
                if (x[q] < u) lo[q] = mid + 1;
                else hi[q] = mid;
                any |= lo[q] < hi[q];
            }
        }
        if (!any) break;
    }
#pragma unroll
    for (int q = 0; q < U; ++q)
        if (srch[q] && (lo[q] >= e[q] || __ldg(b.col + lo[q]) != u)) missing = true;
}

// Every arc of u's row [s, e) in groups of U; lanes of a group (thread, warp or block) take the arcs
// j = s + first, s + first + step, ...
template <int U>
__device__ __forceinline__ void sym_row(const Buffers &b, int u, int64_t s, int64_t e, int64_t first, int64_t step,
                                        bool &missing, unsigned long long &big, unsigned long long &small) {
    for (int64_t j0 = s + first; j0 < e; j0 += U * step) {
        int v[U];
#pragma unroll
        for (int q = 0; q < U; ++q) {
            const int64_t j = j0 + q * step;
            v[q] = j < e ? __ldg(b.col + j) : -1;
        }
        sym_arcs<U>(b, u, e - s, v, missing, big, small);
    }
}

__global__ void __launch_bounds__(256) k_symcheck(Buffers b, int g0, int g1, int nb0, int nb1, int nb2,
                                                  unsigned long long *cnt) {
    const int lane = threadIdx.x & 31;
    bool missing = false;
    unsigned long long big = 0, small = 0;
    if ((int)blockIdx.x < g0) {  // thread per vertex
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb0; i += g0 * blockDim.x) {
            const int u = b.bucket[0][i];
            sym_row<4>(b, u, b.off[u], b.off[u + 1], 0, 1, missing, big, small);
        }
    } else if ((int)blockIdx.x < g0 + g1) {  // warp per vertex
        const int wpb = blockDim.x >> 5;
        const int gw = ((int)blockIdx.x - g0) * wpb + (threadIdx.x >> 5), nw = g1 * wpb;
        for (int i = gw; i < nb1; i += nw) {
            const int u = b.bucket[1][i];
            sym_row<2>(b, u, b.off[u], b.off[u + 1], lane, 32, missing, big, small);
        }
    } else {  // block per vertex
        const int gb = (int)blockIdx.x - g0 - g1, nbk = (int)gridDim.x - g0 - g1;
        for (int i = gb; i < nb2; i += nbk) {
            const int u = b.bucket[2][i];
            sym_row<4>(b, u, b.off[u], b.off[u + 1], threadIdx.x, blockDim.x, missing, big, small);
        }
    }
    big = warp_sum_u64(big);
    small = warp_sum_u64(small);
    if (lane == 0) {
        if (big) atomicAdd(&cnt[0], big);
        if (small) atomicAdd(&cnt[1], small);
    }
    if (__any_sync(DMOLP_FULL_MASK, missing) && lane == 0) *b.flag = 1;
}

// Multiset symmetry test in one streaming pass.  For every arc (u, v), u != v, of the pair p = (min, max):
//   S += s * F(p)   (mod 2^64),  s = +1 when u < v, -1 when u > v,  F(p) = mix(p ^ key),
// mix the SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
// 2014).  Every pair contributes (arcs u->v minus arcs v->u) times F(p), so a graph whose every arc has its
// reverse with the same multiplicity gives S = 0 exactly; any other graph gives a nonzero difference vector,
// and with the key drawn at random per context the sum vanishes with probability about 2^-64 (2^-(64 - t)
// when every multiplicity difference is a multiple of 2^t).  Self-loops are their own reverse and are skipped.
__device__ __forceinline__ unsigned long long sym_mix(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ void sym_hash_arc(unsigned u, unsigned v, unsigned long long key, unsigned long long &sum) {
    if (u == v) return;
    const unsigned long long p = u < v ? ((unsigned long long)u << 32 | v) : ((unsigned long long)v << 32 | u);
    const unsigned long long f = sym_mix(p ^ key);
    sum += u < v ? f : 0ull - f;
}

__global__ void __launch_bounds__(256) k_symhash(Buffers b, int g0, int g1, int nb0, int nb1, int nb2,
                                                 unsigned long long key, unsigned long long *sum) {
    const int lane = threadIdx.x & 31;
    unsigned long long acc = 0;
    // logical blocks [thread class | warp class | block class], dispatched block class (hub rows) first
    const int g2 = (int)gridDim.x - g0 - g1, r = blockIdx.x;
    const int bx = r < g2 ? g0 + g1 + r : r - g2;
    if (bx < g0) {  // thread per vertex (rows of at most 16 arcs)
        for (int i = bx * blockDim.x + threadIdx.x; i < nb0; i += g0 * blockDim.x) {
            const int u = b.bucket[0][i];
            const int64_t s = b.off[u], e = b.off[u + 1];
#pragma unroll 4
            for (int64_t j = s; j < e; ++j) sym_hash_arc((unsigned)u, (unsigned)__ldcs(b.col + j), key, acc);
        }
    } else if (bx < g0 + g1) {  // warp per vertex
        const int wpb = blockDim.x >> 5;
        const int gw = (bx - g0) * wpb + (threadIdx.x >> 5), nw = g1 * wpb;
        for (int i = gw; i < nb1; i += nw) {
            const int u = b.bucket[1][i];
            const int64_t s = b.off[u], e = b.off[u + 1];
#pragma unroll 4
            for (int64_t j = s + lane; j < e; j += 32) sym_hash_arc((unsigned)u, (unsigned)__ldcs(b.col + j), key, acc);
        }
    } else {  // block per vertex
        const int gb = bx - g0 - g1, nbk = g2;
        for (int i = gb; i < nb2; i += nbk) {
            const int u = b.bucket[2][i];
            const int64_t s = b.off[u], e = b.off[u + 1];
#pragma unroll 4
            for (int64_t j = s + threadIdx.x; j < e; j += blockDim.x)
                sym_hash_arc((unsigned)u, (unsigned)__ldcs(b.col + j), key, acc);
        }
    }
    block_atomic_add(acc, sum);
}

__global__ void k_degrees(const int64_t *__restrict__ off, int64_t nv, int32_t *__restrict__ deg) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x)
        deg[v] = (int32_t)(off[v + 1] - off[v]);
}

__global__ void k_fill_int(int32_t *p, int64_t n, int32_t v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

int grid_for(dmolp_ctx *c) { return c->num_sms * kGridPerSm; }

int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

constexpr int kBndHistMaxK = 32;  // k_bnd builds the selection's first histogram up to this many labels

// hist_for_select: k_bnd adds the first-digit histogram of its records to histogram buffer 0 of the
// radix selection that follows (k <= kBndHistMaxK); deg_sel: k_bnd counts its records per degree superbin
// for the degree-bin selection instead.
BndArgs bnd_args(dmolp_ctx *c, int t, int all, int hubwin, int k, bool hist_for_select, bool deg_sel = false) {
    BndArgs a;
    a.t = t;
    a.all = all;
    a.hubwin = hubwin;
    a.dsup = deg_sel ? c->b.dsup : nullptr;
    a.hist = !deg_sel && hist_for_select && k <= kBndHistMaxK ? c->b.hist : nullptr;
    a.hshift = select_first_shift(c->dbits + c->ibits);
    a.ibits = c->ibits;
    a.maxdeg = (int)c->maxdeg;
    a.nb0 = c->nb[0];
    a.nb1 = c->nb[1];
    a.nb2 = c->nb[2];
    const int cap = c->num_sms * 8;
    a.g0 = clampi((c->nb[0] + 255) / 256, 1, cap);
    a.g1 = clampi((c->nb[1] + 7) / 8, 1, cap);
    return a;
}

size_t bnd_smem(int k, const BndArgs &a) {
    return (size_t)k * sizeof(int) +
           (a.dsup ? (size_t)k * kDsBins * sizeof(int) : (a.hist ? (size_t)k * kRadix * sizeof(int) : 0));
}

int bnd_grid(dmolp_ctx *c, const BndArgs &a) { return a.g0 + a.g1 + clampi(c->nb[2], 1, c->num_sms * 2); }

int dec_wstride(int eff) { return eff <= 32 ? 1024 : (eff > (kDecSmallK / 4) * 32 ? eff : (kDecSmallK / 4) * 32); }

size_t dec_smem(int eff, bool use_hot) {
    return (size_t)kWarpsPerBlock * dec_wstride(eff) * sizeof(int) + (use_hot ? (size_t)kHotMax : 0);
}

DecArgs dec_args(int t, int eff, bool hub_ready, bool use_hot, bool kept) {
    DecArgs a;
    a.kept = kept ? 1 : 0;
    a.t = t;
    a.eff = eff;
    a.wstride = dec_wstride(eff);
    a.hub_ready = hub_ready ? 1 : 0;
    a.use_hot = use_hot ? 1 : 0;
    return a;
}

// Persistent grid of k_decide: as many blocks as stay resident (the warps take their work from counters).
int dec_grid(dmolp_ctx *c, int eff) {
    static int per_sm[2] = {0, 0};
    int &n = per_sm[eff <= 32 ? 0 : 1];
    if (n == 0) {
        int r = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_decide, kBlock,
                                                          dec_smem(eff <= 32 ? 32 : DMOLP_MAX_K, true)) != cudaSuccess ||
            r < 1)
            r = kGridPerSm;
        n = r;
    }
    return c->num_sms * n;
}

// use_hot: the hot labels are current; applies when the graph has a hot set and k <= 255 (exact bytes).
StatsArgs stats_args(dmolp_ctx *c, int k, bool use_hot, int keep_eff = 0, int hub_eff = 0) {
    StatsArgs a;
    a.k = k;
    a.keep_eff = keep_eff;
    a.hub_eff = c->nb[2] > 0 ? hub_eff : 0;
    a.use_hot = use_hot && c->nhot > 0 && k <= 255;
    a.nv = (int)c->nv;
    const int cap = c->num_sms * 8;
    a.gv = clampi((int)((c->nv + 255) / 256), 1, c->num_sms * 2);
    a.g0 = clampi((c->nb[0] + 255) / 256, 1, cap);
    a.g1 = clampi((c->nb[1] + 7) / 8, 1, cap);
    a.nb0 = c->nb[0];
    a.nb1 = c->nb[1];
    a.nb2 = c->nb[2];
    return a;
}

int stats_grid(dmolp_ctx *c, const StatsArgs &a) { return a.gv + a.g0 + a.g1 + clampi(c->nb[2], 1, c->num_sms * 2); }

size_t stats_smem(const StatsArgs &a) {
    const size_t kc = a.keep_eff ? 8 * kBlock * sizeof(int) : 0, hc = a.hub_eff > 32 ? (size_t)a.hub_eff * sizeof(int) : 0;
    return 2 * (size_t)a.k * sizeof(unsigned long long) + (a.use_hot ? (size_t)kHotMax : 0) + (kc > hc ? kc : hc);
}

// The LP decisions of the selected window: hub row chunks queued, the classes counted / decided, hub
// argmaxes last; when the hub counts are kept current, k_decide alone (hub argmaxes first).  use_hot: the
// hot labels are current (used when the graph has a hot set and eff <= 32).
void launch_decide(dmolp_ctx *c, int t, int eff, bool recount_hubs, bool use_hot, bool kept) {
    Buffers &b = c->b;
    const bool hubs = c->nb[2] > 0;
    if (hubs && recount_hubs) {
        k_hub_prep<<<c->num_sms * 2, kBlock, 0, c->stream>>>(b, eff);
        c->launches++;
    }
    const bool hot = use_hot && c->nhot > 0 && eff <= 32;
    k_decide<<<dec_grid(c, eff), kBlock, dec_smem(eff, hot && !kept), c->stream>>>(
        b, dec_args(t, eff, !recount_hubs, hot && !kept, kept));
    c->launches++;
    if (hubs && recount_hubs) {
        k_hub_final<<<c->num_sms * 2, kBlock, 0, c->stream>>>(b, eff, t);
        c->launches++;
    }
}

// Optional timing of one kernel launch (dmolp_set_profiling): an event pair around it on the same stream.
// While a graph is being captured the records become event-record nodes of the graph, which owns them.
struct ProfScope {
    dmolp_ctx *c;
    cudaEvent_t e1 = nullptr;
    ProfScope(dmolp_ctx *c_, int kind, int t) : c(c_) {
        if (!c->profiling) return;
        cudaEvent_t e0;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        dmolp_ctx::ProfEvents &pe = c->capturing ? c->capture_prof : c->prof_pending;
        pe.ev.push_back(e0);
        pe.ev.push_back(e1);
        pe.kind.push_back(kind);
        pe.iter.push_back(t);
        if (!c->capturing) c->prof_owned.push_back(1);
        record(e0);
    }
    void record(cudaEvent_t e) {
        if (c->capturing) cudaEventRecordWithFlags(e, c->stream, cudaEventRecordExternal);
        else cudaEventRecord(e, c->stream);
    }
    ~ProfScope() {
        if (e1) record(e1);
    }
};

}  // namespace

void lp_check_symmetric(dmolp_ctx *c, unsigned long long *counts) {
    const int cap = c->num_sms * 8;
    const int g0 = clampi((c->nb[0] + 255) / 256, 1, cap), g1 = clampi((c->nb[1] + 7) / 8, 1, cap);
    const int g2 = clampi(c->nb[2], 1, c->num_sms * 2);
    k_symcheck<<<g0 + g1 + g2, kBlock, 0, c->stream>>>(c->b, g0, g1, c->nb[0], c->nb[1], c->nb[2], counts);
    c->launches++;
}

void lp_symmetry_hash(dmolp_ctx *c, unsigned long long *sum, unsigned long long key) {
    const int cap = c->num_sms * 8;
    const int g0 = clampi((c->nb[0] + 255) / 256, 1, cap), g1 = clampi((c->nb[1] + 7) / 8, 1, cap);
    const int g2 = clampi(c->nb[2], 1, c->num_sms * 2);
    k_symhash<<<g0 + g1 + g2, kBlock, 0, c->stream>>>(c->b, g0, g1, c->nb[0], c->nb[1], c->nb[2], key, sum);
    c->launches++;
}

void lp_degrees(dmolp_ctx *c, const int64_t *off, int64_t nv, int32_t *deg) {
    if (nv <= 0) return;
    k_degrees<<<grid_for(c), kBlock, 0, c->stream>>>(off, nv, deg);
    c->launches++;
}

void lp_fill(dmolp_ctx *c, int32_t *p, int64_t n, int32_t v) {
    k_fill_int<<<grid_for(c), kBlock, 0, c->stream>>>(p, n, v);
    c->launches++;
}

void lp_reset_stats(dmolp_ctx *c, int k, const int *stopped) {
    k_reset_stats<<<1, 256, 0, c->stream>>>(c->b, k, stopped == nullptr);
    c->launches++;
}

void lp_stats(dmolp_ctx *c, int k, const int *stopped, const int *skip, bool use_hot, int keep_eff, int hub_eff) {
    const StatsArgs a = stats_args(c, k, use_hot, keep_eff, hub_eff);
    k_stats<<<stats_grid(c, a), kBlock, stats_smem(a), c->stream>>>(c->b, a, stopped, skip);
    c->launches++;
}

void lp_hot_hist(dmolp_ctx *c) {
    cudaMemsetAsync(c->b.degh, 0, 65536 * sizeof(unsigned int), c->stream);
    k_hot_hist<<<grid_for(c), kBlock, 0, c->stream>>>(c->b, (int)c->nv);
    c->launches++;
}

void lp_hot_build(dmolp_ctx *c, int dstar) {
    k_hot_assign<<<grid_for(c), kBlock, 0, c->stream>>>(c->b, (int)c->nv, dstar);
    k_hot_encode<<<grid_for(c), kBlock, 0, c->stream>>>(c->b, c->narcs);
    c->launches += 2;
}

void lp_hot_refresh(dmolp_ctx *c) {
    if (c->nhot == 0) return;
    k_hot_refresh<<<clampi((c->nhot + 255) / 256, 1, grid_for(c)), kBlock, 0, c->stream>>>(c->b, c->nhot);
    c->launches++;
}

void lp_hub_index(dmolp_ctx *c) {
    lp_fill(c, c->b.hidx, c->nv + 1, -1);
    if (c->nb[2] > 0) {
        k_hub_index<<<clampi((c->nb[2] + 255) / 256, 1, grid_for(c)), kBlock, 0, c->stream>>>(c->b, c->nb[2]);
        c->launches++;
    }
}

void lp_init_end(dmolp_ctx *c, int mode) {
    k_lp_init_end<<<1, 1, 0, c->stream>>>(c->b, mode);
    c->launches++;
}

// The window of iteration t as the selection emits it (see SplitArgs).
SplitArgs split_args(const dmolp_ctx *c, const Buffers &b, int t, int eff) {
    SplitArgs sp;
    sp.RE = b.RE;
    sp.ibits = c->ibits;
    sp.maxdeg = (int)c->maxdeg;
    sp.sstamp = b.sstamp;
    sp.win = b.win[t & 1];
    sp.nwin = &b.cnt->nwin[t & 1];
    for (int c = 0; c < 3; ++c) sp.dec[c] = b.dec[c];
    sp.ndec = b.cnt->ndec;
    sp.te = &b.rec[t - 1].te_sel;
    sp.wsum = &b.rec[t - 1].win_sum;
    sp.t = t;
    sp.eff = eff;
    sp.npart = b.npart;
    sp.ratio = b.ratiotab + t;
    return sp;
}

void lp_iteration(dmolp_ctx *c, const LpLaunch &L, int t, bool first, bool last) {
    Buffers &b = c->b;
    const int grid = grid_for(c);
    const int *stopped = &b.ctrl->stopped;
    bool hist_ready = false;
    const int sym = c->symmetric ? 1 : 0;
    if (first) {  // otherwise the previous iteration's closing k_lp_turn began this one
        k_lp_turn<<<1, 256, 0, c->stream>>>(b, L.k, 0, t, (long long)c->narcs, L.mode, sym);
        c->launches += 1;
    }
    if (t > 1) {
        // the previous window by decision class; hubs through hubwin
        ProfScope ps(c, 2, t);
        k_mark_win<<<grid, kBlock, 0, c->stream>>>(b, t, grid / 2);
        c->launches += 1;
        if (c->nb[2] > 0) {
            k_hubwin_queue<<<clampi((c->nb[2] + 255) / 256, 1, grid), kBlock, 0, c->stream>>>(b, t, c->nb[2]);
            k_hubwin_apply<<<grid, kBlock, 0, c->stream>>>(b, t);
            c->launches += 2;
        }
    }
    const bool deg_sel = L.k <= kDegSelMaxK;  // the degree-bin selection (else the radix selection)
    {
        ProfScope ps(c, 0, t);
        // hubwin is cleared only for graphs with hubs
        const BndArgs a = bnd_args(c, t, t == 1, c->nb[2] > 0, L.k, true, deg_sel);
        k_bnd<<<bnd_grid(c, a), kBlock, bnd_smem(L.k, a), c->stream>>>(b, a, L.k);
        hist_ready = a.hist != nullptr;
    }
    c->launches += 1;
    {
        ProfScope ps(c, 4, t);
        const SplitArgs sp = split_args(c, b, t, L.eff);
        if (!(deg_sel && select_window_deg(c, L.k, sp, stopped)))
            select_smallest(c, b.bown, b.bkey, &b.cnt->npos, L.k, c->dbits + c->ibits, b.bsel, stopped, &sp, hist_ready);
    }
    {
        ProfScope ps(c, 1, t);
        launch_decide(c, t, L.eff, !c->symmetric, true, c->counts_kept);
    }
    if (c->symmetric) {
        {
            ProfScope ps(c, 3, t);
            k_update<<<grid, kBlock, 2 * L.k * sizeof(unsigned long long), c->stream>>>(b, L.k, L.eff, t,
                                                                                         c->counts_kept ? 1 : 0);
        }
        k_apply<<<grid, kBlock, 0, c->stream>>>(b);
        c->launches += 2;
    } else {
        k_apply<<<grid, kBlock, 0, c->stream>>>(b);
        k_lp_mid<<<1, 256, 0, c->stream>>>(b, L.k, t, L.mode);
        const StatsArgs a = stats_args(c, L.k, true);
        k_stats<<<stats_grid(c, a), kBlock, stats_smem(a), c->stream>>>(b, a, stopped, &b.ctrl->skip_stats);
        c->launches += 3;
    }
    k_lp_turn<<<1, 256, 0, c->stream>>>(b, L.k, t, last ? 0 : t + 1, (long long)c->narcs, L.mode, sym);
    c->launches += 1;
}

// dmolp_window_select: previous window in win[(t-1)&1] (nprev entries), RE in b.RE, stamps cleared.
void lp_window_from_list(dmolp_ctx *c, int k, int t, const double *RE_dev, int nprev) {
    (void)RE_dev;
    Buffers &b = c->b;
    const int grid = grid_for(c);
    k_ws_begin<<<1, 256, 0, c->stream>>>(b, k, t, nprev);
    k_mark<<<grid, kBlock, 0, c->stream>>>(b, t);
    k_mark_chunks<<<grid, kBlock, 0, c->stream>>>(b, t);
    const bool deg_sel = k <= kDegSelMaxK;
    const BndArgs a = bnd_args(c, t, 0, 0, k, true, deg_sel);
    k_bnd<<<bnd_grid(c, a), kBlock, bnd_smem(k, a), c->stream>>>(b, a, k);
    c->launches += 4;
    const SplitArgs sp = split_args(c, b, t, DMOLP_MAX_K);
    if (!(deg_sel && select_window_deg(c, k, sp, nullptr)))
        select_smallest(c, b.bown, b.bkey, &b.cnt->npos, k, c->dbits + c->ibits, b.bsel, nullptr, &sp, a.hist != nullptr);
}

// dmolp_lp_apply: window in b.cand (n entries), penalties in b.tpen; movers reported in bv/bnew.
void lp_apply_list(dmolp_ctx *c, int k, int eff, int n) {
    (void)k;
    Buffers &b = c->b;
    const int grid = grid_for(c);
    k_zero_small<<<1, 1, 0, c->stream>>>(b);
    k_classify<<<grid, kBlock, 0, c->stream>>>(b, n, eff);
    launch_decide(c, 1, eff, true, false, false);
    k_collect_moves<<<grid, kBlock, 0, c->stream>>>(b);
    k_apply<<<grid, kBlock, 0, c->stream>>>(b);
    c->launches += 4;
}

}  // namespace dmolp
