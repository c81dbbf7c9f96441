// Phase 1 on the resident CSR: seed coverage and the theta-limited multi-source BFS growth.
//
//   ball      the radius-2 ball of a new seed (compute_bfs with MAX_LEVELS = 3, src/phase1/seed.cpp:20-101)
//             is OR-ed into a coverage byte map: level 1 = the seed's row, level 2 = the rows of level 1
//   hub scan  first unused, uncovered hub of maximum raw degree in hub order (seed.cpp:154-170): one
//             64-bit atomicMax over (degree, ~hub_index)
//   round     (partition.cpp:371-603) per part, the theta frontier vertices with the smallest
//             (raw degree, id) -- segmented radix select -- expand; an unlabelled neighbour is claimed by
//             atomicMin over part ids, which is the reference's "lowest part wins" (its parts are visited in
//             ascending order with a shared visited set, partition.cpp:455-476); claimed vertices join
//             their part's frontier, unselected frontier vertices carry over.
#include <climits>

#include "kernels.cuh"

namespace dmolp {
namespace {

// phase-1 counters (b.p1cnt): 0 = front size (cur), 1 = front size (next), 2 = claimed count,
// 3 = labelled total, 4 = records
__global__ void k_p1_level1(Buffers b, int seed) {
    const int64_t s = b.off[seed], e = b.off[seed + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.covered[seed] = 1;
        atomicAdd(b.p1te, (unsigned long long)(e - s));
    }
    for (int64_t j = s + blockIdx.x * blockDim.x + threadIdx.x; j < e; j += (int64_t)gridDim.x * blockDim.x)
        b.covered[b.col[j]] = 1;
}

// Warp per level-1 vertex (the seed's neighbours, excluding the seed itself on a self-loop).
__global__ void k_p1_level2(Buffers b, int seed) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t s = b.off[seed], e = b.off[seed + 1];
    unsigned long long te = 0;
    for (int64_t i = s + gw; i < e; i += nw) {
        const int u = b.col[i];
        if (u == seed) continue;
        const int64_t us = b.off[u], ue = b.off[u + 1];
        if (lane == 0) te += (unsigned long long)(ue - us);
        for (int64_t j = us + lane; j < ue; j += 32) b.covered[ld_stream(b.col + j)] = 1;
    }
    te = warp_sum_u64(te);
    if (lane == 0 && te) atomicAdd(b.p1te, te);
}

__global__ void k_p1_hub_argmax(Buffers b, int64_t nhubs) {
    unsigned long long best = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nhubs; i += (int64_t)gridDim.x * blockDim.x) {
        if (b.hub_used[i]) continue;
        const int h = b.hubs[i];
        if (b.covered[h]) continue;
        const unsigned long long key = ((unsigned long long)(unsigned)b.rawdeg[h] << 32) |
                                       (unsigned long long)(0xffffffffu - (unsigned)i);
        best = best > key ? best : key;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long ob = __shfl_xor_sync(DMOLP_FULL_MASK, best, o);
        best = best > ob ? best : ob;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(b.best, best);
}

__global__ void k_p1_init(Buffers b, int nv) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        b.label[v] = -1;
        b.claim[v] = INT_MAX;
    }
}

// seeds_dev[p] (p < nseeds, -1 = no seed): label the seed and start its frontier.
__global__ void k_p1_seeds(Buffers b, const int32_t *seeds, int nseeds) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int n = 0, lab = 0;
        for (int p = 0; p < nseeds; ++p) {
            const int s = seeds[p];
            if (s < 0) continue;
            b.label[s] = p;
            b.win[0][n++] = s;
            ++lab;
            b.psize[p] += 1;
        }
        b.p1cnt[0] = n;
        b.p1cnt[3] = lab;
    }
}

// All frontiers empty (partition.cpp:376-394): every unlabelled vertex joins `best` and its frontier.
__global__ void k_p1_fallback(Buffers b, int nv, int best, int cur) {
    int32_t *front = b.win[cur];
    for (int v0 = blockIdx.x * blockDim.x; v0 < nv; v0 += gridDim.x * blockDim.x) {
        const int v = v0 + threadIdx.x;
        const bool un = v < nv && b.label[v] < 0;
        if (un) b.label[v] = best;
        const int slot = warp_append(&b.p1cnt[0], un);
        if (un) front[slot] = v;
        const int c = __popc(__ballot_sync(DMOLP_FULL_MASK, un));
        if ((threadIdx.x & 31) == 0 && c) {
            atomicAdd(&b.p1cnt[3], c);
            atomicAdd((unsigned long long *)&b.psize[best], (unsigned long long)c);
        }
    }
}

// Selection records of the current frontier: segment = part, key = (raw degree, id).  The records per part
// are counted in shared memory first (k parts), then added with one global atomic per part and block.
__global__ void k_p1_records(Buffers b, int cur, int ibits, int k) {
    extern __shared__ int s_np[];  // [k]
    for (int p = threadIdx.x; p < k; p += blockDim.x) s_np[p] = 0;
    __syncthreads();
    const int n = b.p1cnt[0];
    const int32_t *front = b.win[cur];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int v = front[i];
        const int p = b.label[v];
        b.bown[i] = p;
        b.bkey[i] = ((uint64_t)(unsigned)b.rawdeg[v] << ibits) | (uint64_t)v;
        b.bsel[i] = 0;
        atomicAdd(&s_np[p], 1);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x)
        if (s_np[p]) atomicAdd(&b.npart[p], s_np[p]);
    if (blockIdx.x == 0 && threadIdx.x == 0) b.p1cnt[4] = n;
}

__global__ void k_p1_need(Buffers b, int k, int theta) {
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        const int n = b.npart[p];
        b.need[p] = n < theta ? n : theta;
        b.npart[p] = 0;  // consumed; ready for the next round
    }
}

// Claims of the arcs [s, e) of a selected frontier vertex of part p, one warp: unlabelled neighbours take
// atomicMin(part); the one thread that turns a claim from INT_MAX appends the vertex to the claimed list.
__device__ __forceinline__ void claim_arcs(const Buffers &b, int p, int64_t s, int64_t e) {
    const int lane = threadIdx.x & 31;
    for (int64_t j0 = s; j0 < e; j0 += 32) {
        const int64_t j = j0 + lane;
        bool first = false;
        int v = 0;
        if (j < e) {
            v = ld_stream(b.col + j);
            if (b.label[v] < 0) first = atomicMin(&b.claim[v], p) == INT_MAX;
        }
        const int slot = warp_append(&b.p1cnt[2], first);
        if (first) b.cand[slot] = v;
    }
}

// Warp per selected frontier vertex: its first kChunk arcs; the rest of a longer row (the seeds are hubs) is
// queued in kChunk pieces for k_p1_claim_chunks, so that no warp walks a whole hub row alone.  Claims are
// atomicMin, so the order in which pieces run does not matter.
__global__ void k_p1_claim(Buffers b, int cur) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int n = b.p1cnt[0];
    const int32_t *front = b.win[cur];
    unsigned long long te = 0;
    for (int i = gw; i < n; i += nw) {
        if (!b.bsel[i]) continue;
        const int u = front[i];
        const int p = b.bown[i];
        const int64_t s = b.off[u], e = b.off[u + 1];
        if (lane == 0) {
            te += (unsigned long long)(e - s);
            for (int64_t c = s + kChunk; c < e; c += kChunk) {
                const int q = atomicAdd(&b.p1cnt[5], 1);
                b.chunkq[q] = make_int2(i, (int)(c - s));
            }
        }
        claim_arcs(b, p, s, e - s > kChunk ? s + kChunk : e);
    }
    te = warp_sum_u64(te);
    if (lane == 0 && te) atomicAdd(b.p1te, te);
}

// Warp per queued piece of a long frontier row.
__global__ void k_p1_claim_chunks(Buffers b, int cur) {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int n = b.p1cnt[5];
    const int32_t *front = b.win[cur];
    for (int q = gw; q < n; q += nw) {
        const int2 c = b.chunkq[q];
        const int u = front[c.x];
        const int64_t rs = b.off[u], re = b.off[u + 1];
        const int64_t s = rs + c.y;
        claim_arcs(b, b.bown[c.x], s, re - s > kChunk ? s + kChunk : re);
    }
}

// Claimed vertices take their part and join the next frontier; unselected frontier vertices carry over.
__global__ void k_p1_commit(Buffers b, int cur) {
    const int nclaim = b.p1cnt[2], nfront = b.p1cnt[0];
    int32_t *next = b.win[cur ^ 1];
    const int32_t *front = b.win[cur];
    for (int i0 = blockIdx.x * blockDim.x; i0 < nclaim; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        int v = 0, p = 0;
        const bool ok = i < nclaim;
        if (ok) {
            v = b.cand[i];
            p = b.claim[v];
            b.label[v] = p;
            b.claim[v] = INT_MAX;
            atomicAdd((unsigned long long *)&b.psize[p], 1ull);
        }
        const int slot = warp_append(&b.p1cnt[1], ok);
        if (ok) next[slot] = v;
        const int c = __popc(__ballot_sync(DMOLP_FULL_MASK, ok));
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(&b.p1cnt[3], c);
    }
    for (int i0 = blockIdx.x * blockDim.x; i0 < nfront; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        const bool carry = i < nfront && !b.bsel[i];
        const int slot = warp_append(&b.p1cnt[1], carry);
        if (carry) next[slot] = front[i];
    }
}

// Next round: the next frontier becomes current.
__global__ void k_p1_advance(Buffers b) {
    b.p1cnt[0] = b.p1cnt[1];
    b.p1cnt[1] = 0;
    b.p1cnt[2] = 0;
    b.p1cnt[5] = 0;
}

int grid_for(dmolp_ctx *c) { return c->num_sms * 4; }

}  // namespace

void p1_mark_ball(dmolp_ctx *c, int seed) {
    k_p1_level1<<<c->num_sms, 256, 0, c->stream>>>(c->b, seed);
    k_p1_level2<<<grid_for(c), kBlock, 0, c->stream>>>(c->b, seed);
    c->launches += 2;
}

void p1_hub_argmax(dmolp_ctx *c, int64_t nhubs) {
    cudaMemsetAsync(c->b.best, 0, sizeof(unsigned long long), c->stream);
    k_p1_hub_argmax<<<grid_for(c), kBlock, 0, c->stream>>>(c->b, nhubs);
    c->launches += 1;
}

void p1_init_labels(dmolp_ctx *c) {
    k_p1_init<<<grid_for(c), kBlock, 0, c->stream>>>(c->b, (int)c->nv);
    c->launches += 1;
}

void p1_set_seeds(dmolp_ctx *c, const int32_t *seeds_dev, int nseeds) {
    k_p1_seeds<<<1, 32, 0, c->stream>>>(c->b, seeds_dev, nseeds);
    c->launches += 1;
}

void p1_fallback(dmolp_ctx *c, int best_part, int cur) {
    // the current frontier is empty (checked by the caller), so appending starts at 0 in win[cur]
    k_p1_fallback<<<grid_for(c), kBlock, 0, c->stream>>>(c->b, (int)c->nv, best_part, cur);
    c->launches += 1;
}

// One expansion round on frontier buffer `cur` (the frontier lives in win[cur], its size in p1cnt[0]).
void p1_round(dmolp_ctx *c, int k, int theta, int cur) {
    const int grid = grid_for(c);
    k_p1_records<<<grid, kBlock, (size_t)k * sizeof(int), c->stream>>>(c->b, cur, c->ibits, k);
    k_p1_need<<<1, 256, 0, c->stream>>>(c->b, k, theta);
    c->launches += 2;
    select_smallest(c, c->b.bown, c->b.bkey, &c->b.p1cnt[4], k, c->rbits + c->ibits, c->b.bsel, nullptr);
    k_p1_claim<<<grid, kBlock, 0, c->stream>>>(c->b, cur);
    k_p1_claim_chunks<<<grid, kBlock, 0, c->stream>>>(c->b, cur);
    k_p1_commit<<<grid, kBlock, 0, c->stream>>>(c->b, cur);
    k_p1_advance<<<1, 1, 0, c->stream>>>(c->b);
    c->launches += 4;
}

}  // namespace dmolp
