// Batched phase 1: the BFS / hub-seeded initial partition of every graph of a batch in one persistent launch.
//
// A CTA takes the next graph from the queue (largest first) and runs phase 1 on it exactly as the
// single-graph path does (dmolp_phase1; src/phase1/seed.cpp:138-242, partition.cpp:323-604):
//   seeds       the first seed, then repeatedly the first unused hub (in hub order) of maximum degree that
//               lies outside the radius-2 balls of the seeds so far; stops when no hub is left
//   completion  where fewer than k seeds were found: unused hubs by degree (first in hub order on ties),
//               then other vertices by degree (lowest id)
//   growth      rounds: per part the theta frontier vertices with the smallest (degree, id) expand (an
//               in-CTA MSD radix select, segmented by part), unlabelled neighbours are claimed with
//               atomicMin over part ids (lowest part wins), claimed vertices join their part's frontier and
//               unselected ones carry over; with every frontier empty, all unlabelled vertices go to the
//               smallest part (lowest index on ties)
// The hub lists and first seeds come from the host (the reference's order-dependent sort, computed per
// graph in the single-graph code's own function).  Degrees are CSR row lengths: a batch holds graphs with
// sorted, duplicate-free rows, whose line token counts equal them.
#include <climits>

#include "batch.cuh"

namespace dmolp {
namespace batch {
namespace {

constexpr int kP1Threads = 512;
constexpr int kDigitBits = 6;
constexpr int kDigits = 1 << kDigitBits;

struct P1Smem {
    long long psize[kBatchMaxK];
    int npart[kBatchMaxK], need[kBatchMaxK], below[kBatchMaxK], keep[kBatchMaxK];
    int hist[kBatchMaxK * kDigits];
    int seeds[kBatchMaxK];
    unsigned long long best[kP1Threads / 32];
    int nseeds, nfront, nnext, nclaim, nsel, nact[2], open, inst, labelled;
    unsigned long long te;
};

__device__ __forceinline__ int push(int *ctr, bool pred) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(DMOLP_FULL_MASK, pred);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(ctr, __popc(m));
    base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
    return base + __popc(m & ((1u << lane) - 1));
}

// Block-wide maximum of a 64-bit key (every thread passes its own; the result in every thread).
__device__ __forceinline__ unsigned long long block_max(unsigned long long x, P1Smem &sm) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(DMOLP_FULL_MASK, x, o);
        x = y > x ? y : x;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm.best[w] = x;
    __syncthreads();
    unsigned long long r = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = sm.best[i] > r ? sm.best[i] : r;
    __syncthreads();
    return r;
}

__device__ __forceinline__ int deg_of(const P1Args &a, int v) { return (int)(a.off[v + 1] - a.off[v]); }

// Radius-2 ball of seed s: level 1 its row, level 2 the rows of its neighbours (except s itself).
__device__ void mark_ball(const P1Args &a, int s, P1Smem &sm) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t rs = a.off[s], re = a.off[s + 1];
    if (threadIdx.x == 0) {
        a.cov[s] = 1;
        atomicAdd(&sm.te, (unsigned long long)(re - rs));
    }
    for (int64_t j = rs + threadIdx.x; j < re; j += blockDim.x) a.cov[a.col[j]] = 1;
    unsigned long long te = 0;
    for (int64_t i = rs + w; i < re; i += nw) {
        const int u = a.col[i];
        if (u == s) continue;
        const int64_t us = a.off[u], ue = a.off[u + 1];
        if (lane == 0) te += (unsigned long long)(ue - us);
        for (int64_t j = us + lane; j < ue; j += 32) a.cov[a.col[j]] = 1;
    }
    if (lane == 0 && te) atomicAdd(&sm.te, te);
}

__device__ void run_p1(const P1Args &a, int ii, P1Smem &sm) {
    const Inst I = a.inst[ii];
    const int k = I.k, nv = I.nv, vb = (int)I.vbase;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t hs = a.hstart[ii], nh = a.hstart[ii + 1] - hs;
    int32_t *const front[2] = {a.l_front0 + vb, a.l_front1 + vb};
    int32_t *const claimed = a.l_claim + vb;
    int32_t *const act[2] = {a.l_act0 + vb, a.l_act1 + vb};
    if (threadIdx.x == 0) {
        sm.te = 0;
        sm.nseeds = 0;
    }
    for (int p = threadIdx.x; p < kBatchMaxK; p += blockDim.x) {
        sm.psize[p] = 0;
        sm.seeds[p] = -1;
    }
    for (int v = vb + (int)threadIdx.x; v < vb + nv; v += blockDim.x) {
        a.label[v] = -1;
        a.claim[v] = INT_MAX;
        a.cov[v] = 0;
        a.seedm[v] = 0;
        a.sel[v] = 0;
    }
    for (int64_t i = threadIdx.x; i < nh; i += blockDim.x) a.hub_used[hs + i] = 0;
    __syncthreads();
    int nfound = 0, rounds = 0;
    if (nv > 0) {
        // ---- seeds (seed.cpp:192-242) ----
        if (threadIdx.x == 0) {
            const int f = vb + a.first[ii];
            sm.seeds[0] = f;
            sm.nseeds = 1;
            a.seedm[f] = 1;
            if (a.first_hub[ii] >= 0) a.hub_used[hs + a.first_hub[ii]] = 1;
        }
        __syncthreads();
        if (nh > 0 && k > 1) {
            int balls = 0;
            for (int p = 1; p < k; ++p) {
                for (; balls < sm.nseeds; ++balls) mark_ball(a, sm.seeds[balls], sm);
                __syncthreads();
                unsigned long long key = 0;
                for (int64_t i = threadIdx.x; i < nh; i += blockDim.x) {
                    const int h = vb + a.hubs[hs + i];
                    if (a.hub_used[hs + i] || a.cov[h]) continue;
                    const unsigned long long c =
                        ((unsigned long long)(unsigned)deg_of(a, h) << 32) | (0xffffffffull - (unsigned long long)i);
                    key = c > key ? c : key;
                }
                const unsigned long long best = block_max(key, sm);
                if (best == 0) break;
                if (threadIdx.x == 0) {
                    const int64_t idx = (int64_t)(0xffffffffull - (best & 0xffffffffull));
                    const int h = vb + a.hubs[hs + idx];
                    sm.seeds[sm.nseeds++] = h;
                    a.hub_used[hs + idx] = 1;
                    a.seedm[h] = 1;
                }
                __syncthreads();
            }
        }
        nfound = sm.nseeds;
        // ---- seed completion (fewer than k seeds) ----
        while (sm.nseeds < k) {
            unsigned long long key = 0;
            for (int64_t i = threadIdx.x; i < nh; i += blockDim.x) {
                if (a.hub_used[hs + i]) continue;
                const int h = vb + a.hubs[hs + i];
                const unsigned long long c =
                    ((unsigned long long)(unsigned)deg_of(a, h) << 32) | (0xffffffffull - (unsigned long long)i);
                key = c > key ? c : key;
            }
            unsigned long long best = block_max(key, sm);
            int pick = -1;
            if (best) {
                const int64_t idx = (int64_t)(0xffffffffull - (best & 0xffffffffull));
                pick = vb + a.hubs[hs + idx];
                if (threadIdx.x == 0) a.hub_used[hs + idx] = 1;
            } else {
                key = 0;
                for (int v = threadIdx.x; v < nv; v += blockDim.x) {
                    if (a.seedm[vb + v]) continue;
                    const unsigned long long c =
                        ((unsigned long long)(unsigned)deg_of(a, vb + v) << 32) | (0xffffffffull - (unsigned)v);
                    key = c > key ? c : key;
                }
                best = block_max(key, sm);
                if (best == 0) break;  // every vertex is a seed
                pick = vb + (int)(0xffffffffull - (best & 0xffffffffull));
            }
            if (threadIdx.x == 0) {
                sm.seeds[sm.nseeds++] = pick;
                a.seedm[pick] = 1;
            }
            __syncthreads();
        }
        // ---- growth (partition.cpp:335-604) ----
        if (threadIdx.x == 0) {
            int n = 0;
            for (int p = 0; p < k && p < sm.nseeds; ++p) {
                const int s = sm.seeds[p];
                a.label[s] = p;
                front[0][n++] = s;
                sm.psize[p] += 1;
            }
            sm.nfront = n;
            sm.labelled = n;
        }
        __syncthreads();
        const int ib = I.ibits;
        int npass = (I.dbits + ib + kDigitBits - 1) / kDigitBits;
        if (npass < 1) npass = 1;
        const int top = npass * kDigitBits;
        int cur = 0;
        for (;;) {
            if (sm.labelled >= nv) break;
            if (sm.nfront == 0) {  // every frontier empty: all unlabelled vertices join the smallest part
                int bestp = 0;
                for (int p = 1; p < k; ++p)
                    if (sm.psize[p] < sm.psize[bestp]) bestp = p;
                __syncthreads();
                for (int i0 = (int)(threadIdx.x & ~31u); i0 < nv; i0 += blockDim.x) {
                    const int v = vb + i0 + lane;
                    const bool un = i0 + lane < nv && a.label[v] < 0;
                    if (un) a.label[v] = bestp;
                    const int slot = push(&sm.nfront, un);
                    if (un) front[cur][slot] = v;
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    sm.psize[bestp] += sm.nfront;
                    sm.labelled += sm.nfront;
                }
                __syncthreads();
            }
            // frontier records per part; need = min(count, theta)
            for (int p = threadIdx.x; p < kBatchMaxK; p += blockDim.x) sm.npart[p] = 0;
            for (int i = threadIdx.x; i < k * kDigits; i += blockDim.x) sm.hist[i] = 0;
            if (threadIdx.x == 0) {
                sm.nclaim = 0;
                sm.nsel = 0;
            }
            __syncthreads();
            const int nf = sm.nfront;
            for (int i = threadIdx.x; i < nf; i += blockDim.x) atomicAdd(&sm.npart[a.label[front[cur][i]]], 1);
            __syncthreads();
            for (int p = threadIdx.x; p < k; p += blockDim.x) sm.need[p] = sm.npart[p] < a.theta ? sm.npart[p] : a.theta;
            __syncthreads();
            // select need[p] smallest (degree, local id) per part; selected vertices get sel = 1
            int nlist = nf;
            const int32_t *list = front[cur];
            for (int pass = 0; pass < npass; ++pass) {
                const int shift = top - kDigitBits * (pass + 1);
                for (int i0 = (int)(threadIdx.x & ~31u); i0 < nlist; i0 += blockDim.x) {
                    const int i = i0 + lane;
                    int bin = -(lane + 1);
                    if (i < nlist) {
                        const int v = list[i];
                        const int p = a.label[v];
                        if (sm.need[p] > 0) {
                            const uint64_t key = ((uint64_t)deg_of(a, v) << ib) | (uint64_t)(v - vb);
                            bin = p * kDigits + (int)((key >> shift) & (kDigits - 1));
                        }
                    }
                    const unsigned m = __match_any_sync(DMOLP_FULL_MASK, bin);
                    if (bin >= 0 && lane == __ffs(m) - 1) atomicAdd(&sm.hist[bin], __popc(m));
                }
                if (threadIdx.x == 0) {
                    sm.open = 0;
                    sm.nact[pass & 1] = 0;
                }
                __syncthreads();
                for (int p = wib; p < k; p += kP1Threads / 32) {
                    int *h = sm.hist + p * kDigits;
                    const int c0 = h[2 * lane], c1 = h[2 * lane + 1];
                    h[2 * lane] = 0;
                    h[2 * lane + 1] = 0;
                    const int sum = c0 + c1;
                    int incl = sum;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
                        if (lane >= o) incl += y;
                    }
                    const int total = __shfl_sync(DMOLP_FULL_MASK, incl, 31);
                    const int nd = sm.need[p];
                    __syncwarp();
                    if (nd <= 0) {
                        if (lane == 0) {
                            sm.below[p] = 0;
                            sm.keep[p] = -1;
                        }
                    } else if (nd >= total) {
                        if (lane == 0) {
                            sm.below[p] = kDigits;
                            sm.keep[p] = -1;
                            sm.need[p] = 0;
                        }
                    } else {
                        const int ex0 = incl - sum, in0 = ex0 + c0, in1 = in0 + c1;
                        int d = -1, r = 0, cnt = 0;
                        if (ex0 < nd && nd <= in0) {
                            d = 2 * lane;
                            r = nd - ex0;
                            cnt = c0;
                        } else if (in0 < nd && nd <= in1) {
                            d = 2 * lane + 1;
                            r = nd - in0;
                            cnt = c1;
                        }
                        if (d >= 0) {
                            if (r == cnt) {
                                sm.below[p] = d + 1;
                                sm.keep[p] = -1;
                                sm.need[p] = 0;
                            } else {
                                sm.below[p] = d;
                                sm.keep[p] = d;
                                sm.need[p] = r;
                                atomicAdd(&sm.open, 1);
                            }
                        }
                    }
                }
                __syncthreads();
                int32_t *const nxt = act[pass & 1];
                for (int i0 = (int)(threadIdx.x & ~31u); i0 < nlist; i0 += blockDim.x) {
                    const int i = i0 + lane;
                    bool keepv = false;
                    int v = 0;
                    if (i < nlist) {
                        v = list[i];
                        const int p = a.label[v];
                        const uint64_t key = ((uint64_t)deg_of(a, v) << ib) | (uint64_t)(v - vb);
                        const int d = (int)((key >> shift) & (kDigits - 1));
                        if (d < sm.below[p]) a.sel[v] = 1;
                        else keepv = d == sm.keep[p];
                    }
                    const int slot = push(&sm.nact[pass & 1], keepv);
                    if (keepv) nxt[slot] = v;
                }
                __syncthreads();
                if (sm.open == 0) break;
                list = nxt;
                nlist = sm.nact[pass & 1];
                __syncthreads();
            }
            // claims: warp per selected frontier vertex, atomicMin over part ids (partition.cpp:455-476)
            unsigned long long te = 0;
            for (int i = wib; i < nf; i += kP1Threads / 32) {
                const int u = front[cur][i];
                if (!a.sel[u]) continue;  // warp-uniform
                const int p = a.label[u];
                const int64_t s = a.off[u], e = a.off[u + 1];
                if (lane == 0) te += (unsigned long long)(e - s);
                for (int64_t j0 = s; j0 < e; j0 += 32) {
                    const int64_t j = j0 + lane;
                    bool first = false;
                    int v = 0;
                    if (j < e) {
                        v = a.col[j];
                        if (a.label[v] < 0) first = atomicMin(&a.claim[v], p) == INT_MAX;
                    }
                    const int slot = push(&sm.nclaim, first);
                    if (first) claimed[slot] = v;
                }
            }
            te = warp_sum_u64(te);
            if (lane == 0 && te) atomicAdd(&sm.te, te);
            if (threadIdx.x == 0) sm.nnext = 0;
            __syncthreads();
            // commit: claimed vertices take their part and form the next frontier with the unselected ones
            int32_t *const nxtf = front[cur ^ 1];
            const int nc = sm.nclaim;
            for (int i0 = (int)(threadIdx.x & ~31u); i0 < nc; i0 += blockDim.x) {
                const int i = i0 + lane;
                int v = 0;
                if (i < nc) {
                    v = claimed[i];
                    const int p = a.claim[v];
                    a.label[v] = p;
                    a.claim[v] = INT_MAX;
                    atomicAdd((unsigned long long *)&sm.psize[p], 1ull);
                }
                const int slot = push(&sm.nnext, i < nc);
                if (i < nc) nxtf[slot] = v;
            }
            for (int i0 = (int)(threadIdx.x & ~31u); i0 < nf; i0 += blockDim.x) {
                const int i = i0 + lane;
                bool carry = false;
                int v = 0;
                if (i < nf) {
                    v = front[cur][i];
                    carry = !a.sel[v];
                    a.sel[v] = 0;
                }
                const int slot = push(&sm.nnext, carry);
                if (carry) nxtf[slot] = v;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                sm.nfront = sm.nnext;
                sm.labelled += nc;
            }
            cur ^= 1;
            ++rounds;
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        P1Out o;
        o.nseeds_found = nfound;
        o.rounds = rounds;
        o.te = sm.te;
        a.out[ii] = o;
    }
    for (int p = threadIdx.x; p < kBatchMaxK; p += blockDim.x) a.seeds_out[(size_t)ii * kBatchMaxK + p] = p < k ? sm.seeds[p] : -1;
    __syncthreads();
}

__global__ void __launch_bounds__(kP1Threads) k_batch_p1(P1Args a) {
    __shared__ P1Smem sm;
    for (;;) {
        if (threadIdx.x == 0) sm.inst = atomicAdd(a.next, 1);
        __syncthreads();
        const int q = sm.inst;
        if (q >= a.ninst) break;
        if (a.only && !a.only[a.order[q]]) {  // this graph keeps its labels
            __syncthreads();                   // every thread has read sm.inst before it is rewritten
            continue;
        }
        run_p1(a, a.order[q], sm);
    }
}

}  // namespace

void launch_p1(const P1Args &a, int grid, cudaStream_t s) {
    cudaMemsetAsync(a.next, 0, sizeof(int), s);
    k_batch_p1<<<grid, kP1Threads, 0, s>>>(a);
}

}  // namespace batch
}  // namespace dmolp
