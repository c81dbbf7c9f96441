/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.  CPU restatement of the DMOLP partitioning path at one rank,
 * used by tests/ (as the checker) and by bench.py's cpu_baseline leg.  The product never links it.
 */
#ifndef DMOLP_ORACLE_H
#define DMOLP_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t initial_edge_cut;
    double initial_vertex_balance;
    double initial_edge_balance;
    int32_t num_seeds;
    int32_t first_seed;
    int32_t first_seed_degree;
    int32_t rounds;
    int64_t num_hubs;
    uint64_t te;
} oracle_phase1_result;

typedef struct {
    int32_t iteration;
    int32_t window;
    int32_t candidates;
    int32_t changes;
    int64_t edge_cut;
    uint64_t window_hash;
    uint64_t labels_hash;
    uint64_t te_prev, te_cand, te_sel, te_stats;
    uint64_t window_sum; /* sum of SplitMix64(id) over the window, mod 2^64 */
} oracle_iter_record;

typedef struct {
    int64_t edge_cut;
    double vertex_balance;
    double edge_balance;
    int32_t iterations_run;
    int32_t stop_reason; /* 0 = iteration limit, 1 = empty window, 2 = no changes, 3 = converged */
    uint64_t te_total;
    int64_t total_vertices;
    int64_t total_edges;
} oracle_phase2_result;

/* Parse the reference's adjacency text (src/phase1/init.cpp:25-100) into the CSR the reference builds
 * (src/phase1/partition.cpp:182-262: rows sorted, de-duplicated, self-loops kept) plus the raw per-line
 * token count used as the vertex degree in phase 1.  Two calls: sizes first (off/col/rawdeg NULL). */
int oracle_load_adjtext(const char *path, int64_t *nv, int64_t *narcs, int64_t *off, int32_t *col, int32_t *rawdeg);

int oracle_degree_order(int64_t n, int32_t *ids, int32_t *degrees);
int oracle_find_hubs(int64_t nv, const int32_t *rawdeg, int32_t *hubs_out, int64_t *nhubs);

int oracle_phase1(int64_t nv, const int64_t *off, const int32_t *col, const int32_t *rawdeg, int k, int theta,
                  int32_t *labels_out, int32_t *seeds_out, int64_t *vertex_counts, int64_t *edge_counts,
                  oracle_phase1_result *res);

/* mode: 0 = the reference's loop with its three stopping rules (max 500 iterations);
 *       1 = exactly `iters` iterations.
 * cap:  0 = the reference kernel's label cap min(k,32); 1 = no cap (every label < k is scored).
 * records (may be NULL) receives one entry per iteration; counts_out (may be NULL) receives
 * 2*k int64 per iteration (vertex counts, then intra-part edge counts). */
int oracle_phase2(int64_t nv, const int64_t *off, const int32_t *col, int k, int32_t *labels, int mode, int iters,
                  int cap, oracle_iter_record *records, int64_t *counts_out, double *penalty_out,
                  oracle_phase2_result *res);

/* One LP decision for a single vertex given its neighbour labels (the kernel's per-vertex rule). */
int32_t oracle_lp_decide(int32_t own, const int32_t *nbr_labels, int64_t deg, const double *penalty, int k, int cap);

const char *oracle_last_error(void);
uint64_t oracle_fnv1a(const void *data, size_t n);
uint64_t oracle_set_sum(const int32_t *v, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
