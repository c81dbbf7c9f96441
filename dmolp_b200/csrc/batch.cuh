// Batched LP: device-side instance table and kernel arguments (batch_kernels.cu), used by batch_cabi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/dmolp_b200.h"
#include "common.cuh"

namespace dmolp {

// The reference's hub list of a graph from its per-vertex degrees (src/phase1/init.cpp:139-177), as the
// single-graph path computes it (dmolp_cabi.cu).
std::vector<int> hubs_of(const std::vector<int32_t> &degree);

namespace batch {

constexpr int kBatchMaxK = DMOLP_BATCH_MAX_K;
constexpr int kStampStride = 512;  // > the longest run (kMaxIter iterations)

struct Inst {
    int64_t vbase;   // first vertex of the instance in the union graph
    int64_t narcs;   // arcs of the instance
    int32_t nv, k;
    int32_t maxdeg, ibits, dbits, symmetric;
};

struct Out {
    long long edge_cut, te, arcs, visits;
    int iterations, stop_reason, status, changes;
};

struct Args {
    const int64_t *off;
    const int32_t *col;
    int32_t *label, *newlab, *cstamp;
    int32_t *ndiff;  // neighbours with another label, exact at every iteration start
    int32_t *l_cand, *l_bnd, *l_act, *l_win0, *l_win1;  // per-instance slices at vbase
    const Inst *inst;
    const int32_t *order;
    int ninst;
    int *next, *stamp_base;
    Out *out;
    long long *counts;  // [ninst][2 * kBatchMaxK]: vertex counts, intra-part edges
    const double *logtab, *ratiotab;
    int mode, iters, cap;
};

// What the other device modules (the learned proposal) need of a resident batch.
struct View {
    const int64_t *off;
    const int32_t *col;
    int32_t *label;
    const Inst *inst;
    const int32_t *order;
    int ninst;
    int64_t nv, narcs;
    cudaStream_t stream;
    int num_sms, device;
};
bool view(dmolp_batch *b, View *v);  // false when nothing is uploaded

// Batched phase 1 (batch_p1.cu).
struct P1Out {
    int nseeds_found, rounds;
    unsigned long long te;
};

struct P1Args {
    const int64_t *off;
    const int32_t *col;
    int32_t *label;
    const Inst *inst;
    const int32_t *order;
    int ninst;
    int *next;
    const int32_t *hubs;       // per graph, local ids in the reference's hub order
    const int64_t *hstart;     // [ninst + 1]
    const int32_t *first;      // [ninst] first seed (local id)
    const int32_t *first_hub;  // [ninst] its index in the graph's hub list, or -1
    uint8_t *hub_used, *cov, *seedm, *sel;
    int32_t *claim;
    int32_t *l_front0, *l_front1, *l_claim, *l_act0, *l_act1;  // per-graph slices at vbase
    int32_t *seeds_out;                                        // [ninst][kBatchMaxK]
    P1Out *out;
    const uint8_t *only;  // [ninst] or null: run only the graphs flagged 1
    int theta;
};

void launch_p1(const P1Args &a, int grid, cudaStream_t s);

int occupancy(int nt, int td);
bool launch(const Args &a, int nt, int td, int grid, cudaStream_t s);
void prepare(const int64_t *off, int32_t *col, Inst *inst, int ninst, int *next, int *err, int grid, cudaStream_t s);

}  // namespace batch
}  // namespace dmolp
