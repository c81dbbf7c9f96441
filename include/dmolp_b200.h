/*
 * dmolp_b200.h -- C-ABI of the B200-native DMOLP partitioning path (libdmolp_b200.so).
 *
 * One context owns one CUDA device, one stream and a graph resident in HBM (int64 offsets, int32
 * neighbour ids, int32 labels).  Every entry point returns a status code (DMOLP_OK == 0) and never aborts;
 * dmolp_last_error() describes the last failure on the calling thread.  All pointers are HOST pointers
 * unless the name says _device.  Calls on one context must come from one host thread at a time.
 *
 * The reference (DMOLP, C++/MPI/CUDA) has no C-ABI; each entry point below names the reference interface
 * it replaces (paths relative to the reference tree).  The reference's C++ signatures themselves
 * (run_phase1, run_phase2 and the lower-level functions of include/phase1 and include/phase2) are provided on
 * top of this ABI by libdmolp_dropin.so.
 */
#ifndef DMOLP_B200_H
#define DMOLP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define DMOLP_OK 0
#define DMOLP_ERR_ARG 1            /* bad argument (size, k, theta, null pointer) */
#define DMOLP_ERR_CUDA 2           /* a CUDA runtime call failed */
#define DMOLP_ERR_NOMEM 3          /* device or host allocation failed */
#define DMOLP_ERR_STATE 4          /* call out of order (e.g. no graph uploaded) */
#define DMOLP_ERR_BAD_LABELS 5     /* a label outside [0,k) or an odd cut-arc count: where the reference
                                      calls MPI_Abort (src/phase2/phase2.cpp:239-250) */
#define DMOLP_ERR_NO_GPU 6         /* no CUDA device */

/* ---- modes ---- */
#define DMOLP_LP_MODE_REF 0        /* the reference's loop: at most 500 iterations, stops on an empty
                                      window, on zero changes, or after 10 consecutive iterations whose
                                      edge-cut change is below 3 % (src/phase2/phase2.cpp:263-416) */
#define DMOLP_LP_MODE_FIXED 1      /* exactly `iterations` iterations, no early stop */
#define DMOLP_LP_CAP_REF 0         /* score labels < min(k,32), as boundaryLPKernel_unified does
                                      (src/phase2/gpu_lp_boundary.cu:360) */
#define DMOLP_LP_CAP_FULL 1        /* score every label < k (extension; its own oracle) */

#define DMOLP_MAX_K 1024

typedef struct dmolp_ctx dmolp_ctx;

typedef struct {
    int64_t initial_edge_cut;      /* Phase1Metrics::initial_edge_cut  (include/graph_types.h:277) */
    double initial_vertex_balance; /* Phase1Metrics::initial_vertex_balance */
    double initial_edge_balance;   /* Phase1Metrics::initial_edge_balance */
    int32_t num_seeds_found;       /* seeds found by the reference rule (the rest by seed completion) */
    int32_t rounds;                /* expansion rounds */
    int64_t num_hubs;
    uint64_t traversed_edges;      /* arcs read by ball marking + expansion */
    double gpu_ms;                 /* device time of the phase (CUDA events) */
    double hubs_ms;                /* host: hub sort and first seed (wall clock) */
    double seeds_ms;               /* seed search and completion (wall clock) */
    double expand_ms;              /* expansion rounds and initial metrics (wall clock) */
} dmolp_phase1_info;

typedef struct {
    int32_t mode;                  /* DMOLP_LP_MODE_* */
    int32_t iterations;            /* DMOLP_LP_MODE_FIXED: iterations to run */
    int32_t cap;                   /* DMOLP_LP_CAP_* */
    int32_t flags;                 /* reserved, 0 */
} dmolp_lp_config;

typedef struct {
    int64_t edge_cut;              /* PartitioningMetrics::edge_cut (include/graph_types.h:313) */
    double vertex_balance;
    double edge_balance;
    int32_t iterations_run;
    int32_t stop_reason;           /* 0 limit, 1 empty window, 2 no changes, 3 converged */
    uint64_t traversed_edges;      /* sum over iterations of the four traversed-edge terms */
    int64_t total_vertices;
    int64_t total_edges;
    double gpu_ms;                 /* device time of the LP loop (CUDA events) */
} dmolp_lp_result;

typedef struct {                   /* one per LP iteration */
    int32_t iteration;
    int32_t window;                /* selected boundary vertices */
    int32_t candidates;
    int32_t changes;
    int32_t boundary;              /* boundary candidates (before the per-label selection) */
    int32_t reserved;
    int64_t edge_cut;
    uint64_t te_prev, te_cand, te_sel, te_stats;  /* traversed-edge terms of the reference's loop */
    uint64_t arcs_read;            /* arcs this implementation actually read in the iteration */
    uint64_t window_sum;           /* order-independent checksum of the selected window: the sum, mod 2^64,
                                      of the SplitMix64 finaliser of each vertex id */
} dmolp_lp_record;

const char *dmolp_last_error(void);

/* The calling thread's current CUDA device (0 when none is set). */
int dmolp_current_device(void);

/* The architecture of this library's device code as the CUDA runtime loaded it on `device`
 * (cudaFuncAttributes::binaryVersion of one of its kernels: 100 for sm_100a).  No counterpart in the
 * reference. */
int dmolp_device_code_version(int device, int *version);

/* Create a context on CUDA device `device`.  Replaces the device set-up of allocateGPU
 * (src/main.cpp:25-121), which picks local_rank % device_count. */
int dmolp_create(int device, dmolp_ctx **out);
int dmolp_destroy(dmolp_ctx *ctx);

/* Copy a CSR graph to the device and keep it resident.  offsets[nv+1] (int64), indices[narcs] (int32,
 * 0 <= id < nv), raw_degree[nv] (the per-line token count phase 1 sorts by; NULL = CSR degree).  The
 * arrays are validated first (a rejected upload keeps the previous graph); indices in pinned host memory
 * are copied while the validation runs.
 * Replaces the per-iteration subgraph allocation and copies of runBoundaryLPOnGPU_SubgraphUnified
 * (src/phase2/gpu_lp_boundary.cu:456-471) and the Graph built by build_local_graph_and_ghosts
 * (src/phase1/partition.cpp:182). */
int dmolp_graph_upload(dmolp_ctx *ctx, int64_t nv, int64_t narcs, const int64_t *offsets, const int32_t *indices,
                       const int32_t *raw_degree);

/* The reference's adjacency text parsed ON THE DEVICE into the resident graph: first line = header
 * (ignored, as the reference's vertex count comes from the lines), line v+1 = neighbour ids of vertex v.
 * Same result as dmolp_adjtext_load + dmolp_graph_upload: fast_atoi tokenisation (a token starts at the
 * first byte of a non-empty line and at every digit after a non-digit; its value is its digit run, empty =
 * 0), a NUL ends its line's parse, an unterminated last line is dropped, raw degree = tokens on the line,
 * CSR row = sorted, de-duplicated tokens with self-loops kept; an id >= V is an error (DMOLP_ERR_ARG, and
 * the previous graph stays).  Replaces load_graph (src/phase1/init.cpp:25-100) and the CSR construction of
 * build_local_graph_and_ghosts (src/phase1/partition.cpp:227-262).
 * dmolp_graph_upload_adjtext takes the text in host memory (len bytes); dmolp_graph_load_adjtext reads a
 * file through a pinned staging ring, copying each piece to the device while the next is read.
 * info (may be NULL) receives sizes and times. */
typedef struct {
    int64_t num_vertices;
    int64_t num_arcs;               /* after de-duplication */
    int64_t num_tokens;             /* sum of raw degrees */
    int64_t rows_sorted_on_device;  /* rows that were not strictly increasing in the text */
    double read_ms;                 /* file read + host-to-device copy (wall clock), or the copy alone */
    double parse_ms;                /* parse + CSR build on the device (CUDA events, first to last kernel) */
    double total_ms;                /* the whole call (wall clock), state set-up included */
    int64_t kernels;                /* kernels launched by the parse */
    double count_ms;                /* device time of the text count pass (one kernel) */
    double emit_ms;                 /* device time of the token emit pass (one kernel) */
    double setup_ms;                /* resident-state allocation and initialisation (wall clock) */
} dmolp_ingest_info;
int dmolp_graph_upload_adjtext(dmolp_ctx *ctx, const char *text, int64_t len, dmolp_ingest_info *info);
int dmolp_graph_load_adjtext(dmolp_ctx *ctx, const char *path, dmolp_ingest_info *info);
/* The same parse of text already in device memory (d_text: len bytes on the context's device, e.g. read
 * there by the caller's own I/O path); the text is copied into the parse buffer and left unchanged. */
int dmolp_graph_upload_adjtext_device(dmolp_ctx *ctx, const char *d_text, int64_t len, dmolp_ingest_info *info);

/* Sizes of the resident graph, and a copy of it to host arrays offsets[nv+1], indices[narcs],
 * raw_degree[nv] (any may be NULL).  The reference's run_phase1 hands its Graph back to the caller
 * (src/phase1/phase1.cpp:22-160); this is how a device-parsed graph gets there. */
int dmolp_graph_size(dmolp_ctx *ctx, int64_t *nv, int64_t *narcs);
int dmolp_graph_get(dmolp_ctx *ctx, int64_t *offsets, int32_t *indices, int32_t *raw_degree);

/* Phase 1: hubs, first seed, seeds, theta-limited multi-source BFS growth, initial metrics.  Leaves the
 * labels on the device.  seeds_out[k], vertex_counts[k], edge_counts[k] may be NULL.
 * Replaces find_hub_nodes / find_first_seed (src/phase1/init.cpp:139-187), find_seeds
 * (src/phase1/seed.cpp:192), partition_expansion (src/phase1/partition.cpp:323) and the metrics of
 * run_phase1 (src/phase1/phase1.cpp:83-153). */
int dmolp_phase1(dmolp_ctx *ctx, int k, int theta, int32_t *seeds_out, int64_t *vertex_counts,
                 int64_t *edge_counts, dmolp_phase1_info *info);

/* The two halves of phase 1, for callers that supply their own hubs / seeds.
 * dmolp_find_seeds: up to k seeds by the reference rule -- the first seed, then repeatedly the first unused
 * hub (in the given order) of maximum raw degree outside the radius-2 balls of the seeds so far; stops
 * early when none is left, as find_seeds does (src/phase1/seed.cpp:192-242).  seeds_out needs k entries.
 * dmolp_expand_partitions: theta-limited multi-source BFS growth from seeds[0..nseeds) (part p grows from
 * seeds[p]; parts >= nseeds start empty), labels left on the device (src/phase1/partition.cpp:323-604). */
int dmolp_find_seeds(dmolp_ctx *ctx, int k, int32_t first_seed, const int32_t *hubs, int64_t nhubs, int32_t *seeds_out,
                     int32_t *nseeds);
int dmolp_expand_partitions(dmolp_ctx *ctx, int k, int theta, const int32_t *seeds, int32_t nseeds, int32_t *rounds);

/* Phase 2: boundary label propagation with balance penalties on the resident labels.
 * records[max_records] (may be NULL) receives one entry per iteration.
 * Replaces run_phase2 (src/phase2/phase2.cpp:256-449). */
int dmolp_lp_run(dmolp_ctx *ctx, int k, const dmolp_lp_config *cfg, dmolp_lp_result *res, dmolp_lp_record *records,
                 int max_records);

/* The fused edge-cut / balance reduction on the resident labels: cut = arcs with different labels / 2,
 * vertex_counts[p], edge_counts[p] = intra-part arcs / 2.  Replaces computeEdgeCut and
 * computePartitionStats (src/phase2/phase2.cpp:55-117, 214-253). */
int dmolp_metrics(dmolp_ctx *ctx, int k, int64_t *edge_cut, int64_t *vertex_counts, int64_t *edge_counts);

/* Resident labels <-> host (int32[nv]). */
int dmolp_labels_get(dmolp_ctx *ctx, int32_t *labels);
int dmolp_labels_set(dmolp_ctx *ctx, const int32_t *labels);

/* One boundary-window selection on the resident graph and labels, from an explicit previous window.
 * RE[k] as calculatePenalties returns it; iteration is 1-based.  out[] needs room for nv entries; the
 * selected set is returned in ascending id order.  Replaces expandBoundaryNodes
 * (src/phase2/gpu_lp_boundary.cu:185-305). */
int dmolp_window_select(dmolp_ctx *ctx, int k, int iteration, const double *RE, const int32_t *prev, int64_t nprev,
                        int32_t *out, int64_t *nout);

/* One synchronous LP update of `window` with the given penalties; labels of moved vertices are changed
 * on the device and reported (changed_nodes/changed_labels need room for nwindow entries).  Replaces
 * runBoundaryLPOnGPU_Streaming / _SubgraphUnified and boundaryLPKernel_unified
 * (src/phase2/gpu_lp_boundary.cu:327-565). */
int dmolp_lp_apply(dmolp_ctx *ctx, int k, int cap, const double *penalty, const int32_t *window, int64_t nwindow,
                   int32_t *changed_nodes, int32_t *changed_labels, int64_t *nchanged);

/* Per-iteration history of the last dmolp_lp_run: penalties[iters*k] (the penalty vector each iteration
 * used) and counts[iters*2k] (vertex counts then intra-part edge counts after each iteration).  No
 * reference counterpart: calculatePenalties' vectors and computePartitionStats' counts are internal there
 * (src/phase2/phase2.cpp:297, 393); exposed for bitwise parity checks. */
int dmolp_lp_history(dmolp_ctx *ctx, int k, int iters, double *penalties, int64_t *counts);

/* Device pointers of the resident arrays (for callers that keep data on the GPU). */
int dmolp_device_labels(dmolp_ctx *ctx, int32_t **labels_device);

/* The CUDA stream every kernel of this context runs on (a cudaStream_t), e.g. to record timing events on it. */
void *dmolp_stream(dmolp_ctx *ctx);

/* Keep a device-side copy of the current labels / copy it back (device to device, on the context's stream).
 * No reference counterpart: lets a caller rerun phase 2 from the same start without a host round trip. */
int dmolp_labels_save(dmolp_ctx *ctx);
int dmolp_labels_restore(dmolp_ctx *ctx);

/* Optional per-kernel timing: when enabled, dmolp_lp_run brackets its fused scan and statistics kernels with
 * CUDA events and accumulates their device time and algorithmic bytes (read with dmolp_kernel_profile).
 * kernel: 0 = boundary test, 1 = LP decisions, 2 = window marking, 3 = incremental cut/balance update,
 * 4 = per-label window selection (all radix-select launches of an iteration).
 * No reference counterpart. */
int dmolp_set_profiling(dmolp_ctx *ctx, int enable);
int dmolp_kernel_profile(dmolp_ctx *ctx, int kernel, double *total_ms, int64_t *launches, double *bytes);

/* How long a grid barrier of the cooperative window selections waits before it gives up: `polls` reads of
 * its generation word (0 = the default, 2^22, about a second).  Its blocks are co-resident (cooperative
 * launch), so the default is never reached; a barrier that gives up stops the loop and every block leaves the
 * kernel, and the call returns DMOLP_ERR_CUDA naming the barrier, with the context ready for the next call.
 * No reference counterpart (the reference's kernel has no barrier).  Mainly for testing that path. */
int dmolp_set_wait_limit(dmolp_ctx *ctx, uint32_t polls);

/* How the LP loop tests whether the resident graph is symmetric (every arc's reverse present, with the same
 * multiplicity), which lets it update cut and balance from the movers alone.  exact = 0 (default): one
 * streaming pass forms a keyed 64-bit multiset sum, zero for every symmetric graph; an asymmetric graph
 * passes with probability about 2^-64 (key drawn per context).  exact = 1: every reverse arc is looked up
 * by binary search (a few ms per 10^8 arcs).  Either way the test runs once per uploaded graph, when the loop
 * first needs it.  No reference counterpart (the reference always recounts). */
int dmolp_set_symmetry_test(dmolp_ctx *ctx, int exact);
/* The test's answer for the resident graph (runs it now if the loop has not yet): 1 = symmetric with rows
 * strictly increasing (incremental statistics apply), else 0. */
int dmolp_graph_symmetric(dmolp_ctx *ctx, int *symmetric);

/* ---- phase-1 hubs on the host (no device work) ----
 * dmolp_find_hubs_pairs: find_hub_nodes (src/phase1/init.cpp:139-177) on n (id, degree) pairs given in the
 * reference's degree-map order: the pairs sorted by degree in exactly the order std::sort leaves them (ties
 * included), the Lorenz-curve tangent's x-intercept, and the hubs past it in descending sort order; hubs
 * needs room for n entries.  dmolp_degree_order returns that sorted order itself (ids[], degrees[] rewritten
 * in place).  Both run on all host threads and give std::sort's permutation (checked against it). */
int dmolp_find_hubs_pairs(int64_t n, const int32_t *ids, const int32_t *degrees, int32_t *hubs, int64_t *nhubs);
int dmolp_degree_order(int64_t n, int32_t *ids, int32_t *degrees);
/* find_hub_nodes and find_first_seed (src/phase1/init.cpp:139-187; init.hpp:10-11) on the raw degrees one
 * rank gathers (raw_degree[v] for v < nv; the degree map iterates v = nv-1 down to 0): the hubs as
 * dmolp_find_hubs_pairs gives them (hubs needs room for nv entries) and the first seed with its degree, by
 * the reference's loop and its tie test, which compares a vertex id with the best degree ((-1, -1) when
 * there is no vertex of degree >= 0).  The host step of dmolp_phase1. */
int dmolp_find_hubs(int64_t nv, const int32_t *raw_degree, int32_t *hubs, int64_t *nhubs, int32_t *first_seed,
                    int32_t *first_seed_degree);

/* ---- host-side graph loading (no device work) ----
 * Parse the reference's adjacency text: first line V, line i+1 = neighbour ids of vertex i.  Produces the
 * CSR the reference builds (rows sorted and de-duplicated, self-loops kept) and the raw per-line token
 * count.  Replaces load_graph (src/phase1/init.cpp:25-100) and the CSR construction of
 * build_local_graph_and_ghosts (src/phase1/partition.cpp:227-262). */
typedef struct dmolp_host_graph dmolp_host_graph;
int dmolp_adjtext_load(const char *path, dmolp_host_graph **out);
const char *dmolp_adjtext_error(void);
int64_t dmolp_host_graph_nv(const dmolp_host_graph *g);
int64_t dmolp_host_graph_narcs(const dmolp_host_graph *g);
const int64_t *dmolp_host_graph_offsets(const dmolp_host_graph *g);
const int32_t *dmolp_host_graph_indices(const dmolp_host_graph *g);
const int32_t *dmolp_host_graph_raw_degree(const dmolp_host_graph *g);
void dmolp_host_graph_free(dmolp_host_graph *g);

/* The fused edge-cut / balance reduction without any device allocation.  No counterpart in the reference.
 * For callers that cannot let a library allocate device memory -- e.g. a process whose GPU memory belongs to
 * another allocator (a framework's caching pool, or a server that reserves all memory at start-up) -- this
 * entry point needs no context: the caller passes its CSR and labels as DEVICE pointers (offsets[nv+1],
 * indices[], labels[nv] on `device`, ids in [0,nv)) and a stream (NULL = the legacy default stream) and gets
 * the results in HOST memory, as dmolp_metrics returns them.  Its only scratch is a file-scope device array
 * of 2*DMOLP_NOALLOC_MAX_K+2 64-bit counters (16 KiB), held by every GPU that loads the library until exit;
 * k above DMOLP_NOALLOC_MAX_K is rejected with DMOLP_ERR_ARG.  Every call shares that array and clears the
 * part it uses first; calls that overlap on the GPU race.  The first call on a device looks up the array's
 * address with that device current; make it before any stream capture.  That address is kept for the life of
 * the process, so a cudaDeviceReset after the first call on a device is not supported.  The calling thread's
 * current device is the same after the call as before.  A neighbour id outside [0,nv) or a decreasing pair of
 * offsets is skipped by the kernel and reported as DMOLP_ERR_ARG (offsets[nv] cannot be range-checked: the
 * call takes no arc count); a label outside [0,k) or an odd cut-arc count is DMOLP_ERR_BAD_LABELS.
 * Errors: dmolp_last_error(). */
#define DMOLP_NOALLOC_MAX_K 1024
int dmolp_metrics_noalloc(int device, int64_t nv, const int64_t *offsets_device, const int32_t *indices_device,
                          const int32_t *labels_device, int k, void *stream, int64_t *edge_cut, int64_t *vertex_counts,
                          int64_t *edge_counts);

/* Number of kernel launches this context has issued (all entry points). */
int64_t dmolp_kernel_launches(const dmolp_ctx *ctx);

/* ---------------------------------------------------------------------------------------------------------
 * Batched phase 2: many independent graphs, each with its own part count, partitioned by one persistent
 * kernel launch replayed from a captured CUDA graph.  No counterpart in the reference, which partitions one
 * graph per run; every instance follows run_phase2 (src/phase2/phase2.cpp:256-449) exactly as dmolp_lp_run
 * does and ends with the same labels, cut and counts as a single-graph run on the same graph and labels.
 * ------------------------------------------------------------------------------------------------------- */
#define DMOLP_BATCH_MAX_K 64

typedef struct dmolp_batch dmolp_batch;

typedef struct {                   /* the launch shape; the autotuner picks it */
    int32_t block_threads;         /* threads per CTA: 256, 512 or 1024 */
    int32_t thread_row_max;        /* rows of at most this many arcs are walked by one thread: 8 or 16 */
    int32_t blocks_per_sm;         /* resident CTAs per SM (0 = as many as fit) */
    int32_t reserved;
} dmolp_batch_tuning;

typedef struct {                   /* one per instance */
    int64_t edge_cut;
    uint64_t traversed_edges;      /* the same four terms as dmolp_lp_result */
    uint64_t arcs_read;            /* arcs this implementation read */
    uint64_t vertex_visits;        /* vertex rows this implementation opened (offsets + own label) */
    double vertex_balance, edge_balance;
    int32_t iterations_run;
    int32_t stop_reason;
    int32_t status;                /* DMOLP_OK, or DMOLP_ERR_BAD_LABELS for labels outside [0,k) */
    int32_t changes;               /* moves over all iterations */
} dmolp_batch_result;

int dmolp_batch_create(int device, dmolp_batch **out);
int dmolp_batch_destroy(dmolp_batch *b);

/* The batch as one union CSR: instance i owns vertices [vstart[i], vstart[i+1]) and their rows of
 * offsets[] (int64, nv+1 entries, offsets[0] = 0); indices[] hold ids LOCAL to the instance (0-based).
 * parts[i] = k of instance i in [1, DMOLP_BATCH_MAX_K].  nv < 2^31.  Resets the labels to 0. */
int dmolp_batch_upload(dmolp_batch *b, int32_t ninst, const int64_t *vstart, const int64_t *offsets,
                       const int32_t *indices, const int32_t *parts);
/* Labels of all instances, int32[nv] in union order, values in [0, parts[i]). */
int dmolp_batch_labels_set(dmolp_batch *b, const int32_t *labels);
int dmolp_batch_labels_get(dmolp_batch *b, int32_t *labels);
int dmolp_batch_labels_save(dmolp_batch *b);     /* device-side copy of the labels ... */
int dmolp_batch_labels_restore(dmolp_batch *b);  /* ... put back (the autotuner overwrites the copy) */
int dmolp_batch_device_labels(dmolp_batch *b, int32_t **labels);  /* device pointer to the labels */
void *dmolp_batch_stream(dmolp_batch *b);              /* the batch's cudaStream_t */

/* Phase 2 on every instance (cfg as for dmolp_lp_run).  tune NULL: the autotuned shape if
 * dmolp_batch_autotune ran, else a default.  results[ninst] (may be NULL); gpu_ms (may be NULL) = device time
 * of the launch.  An instance with labels outside [0,k) is left unchanged, its status says so, and the call
 * returns DMOLP_ERR_BAD_LABELS after all others ran. */
int dmolp_batch_lp_run(dmolp_batch *b, const dmolp_lp_config *cfg, const dmolp_batch_tuning *tune,
                       dmolp_batch_result *results, double *gpu_ms);
/* Times every launch shape on the uploaded batch and its current labels (restored after each trial) and
 * keeps the fastest for later runs.  best / best_ms may be NULL. */
int dmolp_batch_autotune(dmolp_batch *b, const dmolp_lp_config *cfg, dmolp_batch_tuning *best, double *best_ms);
/* ---------------------------------------------------------------------------------------------------------
 * Learned initial partition (no counterpart in the reference, whose phase 1 is BFS / hub seeding): a 3-layer
 * mean-aggregation message-passing network, Z = [H | mean over neighbours of H] @ W + b per layer, widths
 * 16 -> 64 -> 64 -> 16, BF16 weights and activations with FP32 accumulation on the tensor cores.  Inputs per
 * vertex: degree / mean degree, log(1 + degree), 8 random-walk features (log landing probabilities of lazy
 * walks from 8 farthest-point anchors, standardised per graph) and k / 64.  The 16-wide output embedding is
 * turned into k balanced labels per graph by recursive coordinate bisection.  Trained with an
 * edge-contrastive loss on final partitions of the plain method.  Works on a dmolp_batch; a graph the
 * proposal cannot serve (fewer vertices than parts, a non-finite embedding, an empty part) is flagged so the
 * caller seeds it with phase 1 instead.
 * ------------------------------------------------------------------------------------------------------- */
typedef struct dmolp_mpnn dmolp_mpnn;

int64_t dmolp_mpnn_num_params(void);           /* length of the flat FP32 parameter vector */
int dmolp_mpnn_create(int device, dmolp_mpnn **out);  /* fixed-seed Glorot hidden layers, zero output layer */
int dmolp_mpnn_destroy(dmolp_mpnn *m);
/* Polls of a GEMM's MMA completion barrier before the GEMM gives up (0 = the default, 2^24 non-blocking
 * checks, a fraction of a second; far above any real MMA).  A GEMM that gives up waits (bounded) for the MMA in flight, frees its tensor memory and sets an
 * error flag: the call returns DMOLP_ERR_CUDA and the network stays usable.  Mainly for testing that path. */
int dmolp_mpnn_set_wait_limit(dmolp_mpnn *m, uint32_t polls);
/* Parameters, flat FP32: per layer W [K x N] row-major then b [N]; K = 32, 128, 128; N = 64, 64, 16.
 * Setting them resets the optimiser state. */
int dmolp_mpnn_set_params(dmolp_mpnn *m, const float *params);
int dmolp_mpnn_get_params(dmolp_mpnn *m, float *params);
/* Input features of the batch's graphs, computed on the device; features[nv*16] (may be NULL) receives
 * them before the BF16 rounding.  dmolp_mpnn_set_features installs features given by the caller instead. */
int dmolp_mpnn_features(dmolp_mpnn *m, dmolp_batch *b, float *features);
int dmolp_mpnn_set_features(dmolp_mpnn *m, dmolp_batch *b, const float *features);
/* Forward pass on the current features; embedding[nv*16] (may be NULL). */
int dmolp_mpnn_forward(dmolp_mpnn *m, dmolp_batch *b, float *embedding);
/* Training needs the activations of every layer: call this before the features of a training batch. */
int dmolp_mpnn_prepare_training(dmolp_mpnn *m, dmolp_batch *b);
/* Backward of the last forward pass for an upstream gradient d_embedding[nv*16]; grads[num_params] out. */
int dmolp_mpnn_backward(dmolp_mpnn *m, dmolp_batch *b, const float *d_embedding, float *grads);
/* One Adam step (lr; beta 0.9 / 0.999) on the edge-contrastive loss against target labels target[nv]:
 * mean over arcs (v,u) of |p_v - p_u|^2 when the targets agree, max(0, 1 - |p_v - p_u|^2) otherwise, p the
 * proposal coordinates. */
int dmolp_mpnn_train_step(dmolp_mpnn *m, dmolp_batch *b, const int32_t *target, float lr, double *loss);
/* Labels from the current features and an embedding (NULL = the last forward pass) into the batch's
 * labels; status[ninst] (may be NULL): 0 = proposal used, 1 = not usable (the graph keeps labels 0 and needs
 * phase-1 seeding). */
int dmolp_mpnn_decode(dmolp_mpnn *m, dmolp_batch *b, const float *embedding, int32_t *status);
/* The learned gate: per graph, the mean of output column 8 over its vertices after the last forward pass;
 * >= 0 means the proposal is expected to end at an edge cut no higher than phase-1 seeding's. */
int dmolp_mpnn_gate(dmolp_mpnn *m, dmolp_batch *b, double *scores);
/* One Adam step on the gate alone: binary cross-entropy of sigmoid(score) against target[ninst] (1 = the
 * proposal beat phase 1 on this graph, from runs of the plain method). */
int dmolp_mpnn_train_gate(dmolp_mpnn *m, dmolp_batch *b, const float *target, float lr, double *loss);
/* Features + forward + decode + gate.  status: 0 = proposal used, 1 = not usable, 2 = the gate prefers
 * phase-1 seeding; for 1 and 2 the caller seeds the graph with phase 1. */
int dmolp_batch_propose(dmolp_batch *b, dmolp_mpnn *m, int32_t *status);

/* Phase 1 on every instance (as dmolp_phase1 with this theta, labels into the batch), one persistent
 * launch; only[ninst] (may be NULL) restricts it to the instances flagged 1, the others keep their labels.  Degrees are the CSR row lengths (the graphs of a batch have sorted, duplicate-free rows).  The
 * reference's order-dependent hub lists and first seeds are computed on the host once per upload.
 * seeds[ninst * DMOLP_BATCH_MAX_K] (may be NULL): each graph's seeds (ids inside the graph, -1 unused);
 * results[ninst] (may be NULL); gpu_ms (may be NULL) = device time of the launch. */
typedef struct {
    int32_t num_seeds_found;       /* seeds found by the reference rule (the rest by seed completion) */
    int32_t rounds;                /* expansion rounds */
    uint64_t traversed_edges;      /* arcs read by ball marking + expansion */
} dmolp_batch_p1_result;
int dmolp_batch_phase1(dmolp_batch *b, int theta, const uint8_t *only, int32_t *seeds, dmolp_batch_p1_result *results,
                       double *gpu_ms);

/* Per-part vertex counts and intra-part edge counts of instance i after the last run (k entries each). */
int dmolp_batch_counts(dmolp_batch *b, int32_t inst, int64_t *vertex_counts, int64_t *edge_counts);

#ifdef __cplusplus
}
#endif
#endif
