// Device-resident state of one dmolp context (layout in HBM) and the small control blocks the
// iteration kernels share.  Everything is allocated once per graph upload; the LP loop allocates nothing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "ingest.cuh"

namespace dmolp {

// Degree classes of the bucketed kernels: thread per vertex, warp per vertex, block per vertex.
constexpr int kSmallDeg = 16;    // deg <= 16: one thread walks the row
constexpr int kDecSmall = 32;    // LP decisions: rows of at most 32 arcs are counted by one thread ...
constexpr int kDecSmallK = 64;   // ... when at most 64 labels are scored (byte counters in shared memory)
constexpr int kLargeDeg = 4096;  // deg > 4096: one block walks the row
constexpr int kChunk = 4096;     // row chunk of the window-marking kernel
constexpr int kHotMax = 16384;   // LP gathers: labels of up to this many highest-degree vertices per block
constexpr int kHubChunk = 2048;  // row chunk of the decisions of deg > kLargeDeg vertices

// Polls of a grid-barrier generation word before the barrier gives up (about a second on B200).
constexpr unsigned int kDefaultWaitPolls = 1u << 22;

// Per-iteration counters of the LP loop (reset by the first kernel of each iteration).
struct LpCounters {
    int ncand;        // candidates this iteration (t >= 2)
    int nbnd;         // boundary candidates (selection records)
    int nwin[2];      // window (selected set) sizes, double-buffered by iteration parity
    int nactive[2];   // radix-select active lists
    int nchanged;     // selected vertices whose label changed (movers)
    int ndec[3];      // selected vertices per decision class
    int ndec_prev[3]; // the previous iteration's ndec (its window by class, for the marking)
    int nchunk;       // queued row chunks of the marking kernel
    int nhubq;        // queued row chunks of the hub decisions
    int npos;         // selection record slots: one per vertex with arcs (fixed per graph)
    unsigned long long cut_arcs;   // arcs whose endpoint labels differ (kept current incrementally)
    int dgrab[3];     // decisions: work items taken so far per class (thread groups, warp groups, hub chunks)
    int nhubw;        // queued row chunks of hubs that entered or left the window
};

// Loop control shared by the iteration kernels.
struct LpControl {
    int stopped;        // set at the end of the iteration that met a stopping rule; later kernels return
    int stop_now;       // stopping rule met in the current iteration (1 empty, 2 no change, 3 converged)
    int skip_stats;     // current iteration runs no statistics pass
    int conv;           // consecutive iterations with relative cut change < 3 %
    long long prev_cut; // last computed edge cut
    int iters_run;
    int stop_reason;
    int error;          // 1 = odd cut-arc count or invalid label (the reference aborts)
    int mode;           // DMOLP_LP_MODE_*
    int pull;           // next iteration finds candidates by pulling (rows scanned for a window member)
    int sel_open[2];    // radix select: segments still needing records after a pass (by pass parity)
    unsigned int bar_count, bar_gen;  // grid barrier of the cooperative selection kernel
    int wait_timeout;   // a grid barrier gave up waiting (1 + the barrier's index in the kernel)
    int sel_tail;       // radix select: records appended to the list that block 0 finishes alone
};

// One LP iteration record as kept on the device.
struct LpRecordDev {
    int iteration, window, candidates, changes;
    int boundary, pad;
    long long edge_cut;
    unsigned long long te_prev, te_cand, te_sel, te_stats;
    // arcs the kernels actually read: boundary test (early exit), decisions, incremental update
    unsigned long long arcs_bnd, arcs_dec, arcs_upd;
    unsigned long long arcs_mark;  // arcs read by the window marking (window rows, rows of hubs that changed)
    unsigned long long te_hubsel;  // arcs of the selected hubs (part of te_sel)
    unsigned long long win_sum;    // sum of window_mix(v) over the selected window (order-independent checksum)
};

struct Buffers {
    // graph
    int64_t *off = nullptr;    // [nv+1]
    int32_t *col = nullptr;    // [narcs]
    int32_t *rawdeg = nullptr; // [nv]
    int32_t *label = nullptr;  // [nv]
    int32_t *ball = nullptr;   // vertex ids with arcs, by degree class then ascending id; position = record slot
    int32_t *bucket[3] = {nullptr, nullptr, nullptr};  // the three classes inside ball
    // LP scratch
    int32_t *stamp = nullptr;  // [nv] iteration stamp of candidate marking (push)
    int32_t *sstamp = nullptr; // [nv] iteration stamp of the selected window (pull)
    int32_t *ndiff = nullptr;  // [nv] neighbours with another label (the boundary test is ndiff > 0)
    int32_t *cand = nullptr;   // [nv] phase-1 claimed list / stand-alone window list
    int32_t *win[2] = {nullptr, nullptr};  // [nv] each: selected window of the iteration (by parity)
    int32_t *bv = nullptr, *bnew = nullptr;  // [nv] mover pairs of dmolp_lp_apply; phase-1 records
    int32_t *bown = nullptr;   // [nv] record slot: own label of a boundary vertex, -1 otherwise
    uint64_t *bkey = nullptr;  // [nv] record slot: selection key
    uint8_t *bsel = nullptr;   // [nv] record slot: selected
    int32_t *dec[3] = {nullptr, nullptr, nullptr};  // [nv] each: selected vertices per decision class
    int32_t *newlab = nullptr; // [nv] new label of a mover in the current iteration, else -1
    int32_t *mov = nullptr;    // [nv] movers of the current iteration
    int2 *chunkq = nullptr;    // [chunk_cap] (vertex, first arc) of queued row chunks
    int2 *hubq = nullptr;      // [hubq_cap] (hub index, first arc) of queued hub-decision chunks
    int32_t *hh = nullptr;     // [nb[2] * MAX_K] per-hub label counts, row = hub index: recounted for the
                               // selected hubs each iteration, or (symmetric graphs) counted once per LP run
                               // and kept current from the movers' arcs
    int32_t *hidx = nullptr;   // [nv] hub index (position in bucket[2]) of a vertex with deg > kLargeDeg, else -1
    int32_t *hubwin = nullptr; // [nv] hubs of the previous window whose rows hold the vertex
    int32_t *hub_in = nullptr; // [nb[2]] hub is counted in hubwin (was in the window hubwin describes)
    int2 *hubwq = nullptr;     // [hubq_cap] (hub index, first arc) of rows entering or leaving hubwin
    // hot set: the (at most kHotMax) vertices of highest degree, whose labels the label-gathering kernels
    // read from a per-block shared copy
    int32_t *colh = nullptr;   // [narcs] col with a hot neighbour u written as -(hrank[u] + 2)
    int32_t *hrank = nullptr;  // [nv] rank of a hot vertex, else -1
    int32_t *hotid = nullptr;  // [kHotMax] vertex of each rank
    uint8_t *hotlab = nullptr; // [kHotMax] label of each hot vertex, clamped to 255 (kept current by k_apply)
    unsigned int *degh = nullptr;  // [65536] degree histogram (hot-set threshold)
    // kept label counts (symmetric graphs, eff <= 32): vcnt[v * 32 + c] = neighbours of v with label c, for
    // every vertex with at most kLargeDeg arcs (hubs: hh); built by the run's first statistics pass and
    // kept current by k_update
    uint16_t *vcnt = nullptr;      // [nv * 32]
    int32_t *active[2] = {nullptr, nullptr};  // [nv] radix-select active lists
    // per-part arrays (DMOLP_MAX_K); vc / intra hold signed values in two's complement
    unsigned int *hist = nullptr;        // [kSelHistBuffers * MAX_K * 256] radix-select histograms
    // degree-bin window selection (k <= kDegSelMaxK): superbin counts of the boundary records per label
    // (written by the boundary test), fine-bin counts of the partial superbins (by iteration parity), and
    // each selection block's fine-bin counts
    unsigned int *dsup = nullptr;        // [kDegSelMaxK * kDsBins]
    unsigned int *dfine[2] = {nullptr, nullptr};  // [kDegSelMaxK * kDsFine] each
    unsigned int *dcntb = nullptr;       // [num_sms * kDegSelMaxK * kDsFine]
    int *dtcnt = nullptr;                // [2 * kDegSelMaxK] tail records per label (by iteration parity)
    uint64_t *dlkey = nullptr;           // [nv] keys of the selection warps' lists (labels in active[0])
    uint64_t *dtkey = nullptr;           // [nv] keys of the selection's tail segments
    int32_t *need = nullptr;             // [MAX_K]
    int32_t *sel_below = nullptr;        // [MAX_K]
    int32_t *keep_digit = nullptr;       // [MAX_K]
    int32_t *npart = nullptr;            // [MAX_K] records per segment
    unsigned long long *vc = nullptr;    // [MAX_K] vertex counts
    unsigned long long *intra = nullptr; // [MAX_K] intra-part arcs
    long long *psize = nullptr;          // [MAX_K] phase-1 part sizes
    double *tpen = nullptr;              // [MAX_K] 1 + penalty
    double *RE = nullptr;                // [MAX_K]
    double *penhist = nullptr;           // [kMaxIter * MAX_K]
    long long *cnthist = nullptr;        // [kMaxIter * 2 * MAX_K]
    double *logtab = nullptr;            // [kMaxIter + 1] log(t)
    double *ratiotab = nullptr;          // [kMaxIter + 1] exp(-t/5)
    LpCounters *cnt = nullptr;
    LpControl *ctrl = nullptr;
    LpRecordDev *rec = nullptr;          // [kMaxIter]
    // phase 1 scratch
    uint8_t *covered = nullptr;          // [nv]
    int32_t *hubs = nullptr;             // [nv]
    uint8_t *hub_used = nullptr;         // [nv]
    int32_t *claim = nullptr;            // [nv] (aliases stamp)
    unsigned long long *best = nullptr;  // [1] packed hub argmax
    int *p1cnt = nullptr;                // [8] phase-1 counters
    unsigned long long *p1te = nullptr;  // [1]
    int *flag = nullptr;                 // [1] scratch flag (symmetry check)
    unsigned long long *symcnt = nullptr;  // [2] arc counts / multiset sums of the symmetry test
};

}  // namespace dmolp

struct dmolp_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    int64_t nv = 0, narcs = 0;
    int64_t maxdeg = 0, maxraw = 0;
    int ibits = 1, dbits = 1, rbits = 1;  // bits for ids, CSR degree, raw degree
    int nb[3] = {0, 0, 0};                // vertices per degree class
    int64_t chunk_cap = 0, hubq_cap = 0;
    bool symmetric = false;               // every arc (u,v) has its reverse: incremental statistics apply
    bool symmetry_known = false;          // `symmetric` has been tested for the resident graph
    bool rows_sorted = false;             // every row strictly increasing (precondition of the test)
    bool symmetry_exact = false;          // test by reverse-arc searches instead of the multiset sums
    unsigned long long sym_key = 0;       // key of the multiset symmetry sum, drawn per context
    bool has_graph = false;
    bool hot_ready = false;               // colh / hrank / hotid built for the resident graph
    bool counts_kept = false;             // the current LP run decides from vcnt / hh (no label gathers)
    unsigned int wait_polls = dmolp::kDefaultWaitPolls;  // polls of a grid barrier before it gives up
    int nhot = 0;                         // hot vertices
    int lp_runs = 0;                      // dmolp_lp_run calls on the resident graph
    std::vector<int32_t> h_rawdeg;        // host copy for the hub sort
    bool h_rawdeg_valid = false;          // h_rawdeg mirrors the resident raw degrees
    dmolp::Buffers b;
    std::vector<void *> allocations;
    long long launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int32_t *saved_labels = nullptr;  // dmolp_labels_save
    // optional kernel timing (dmolp_set_profiling): event pairs around timed kernels
    struct ProfEvents {
        std::vector<cudaEvent_t> ev;  // pairs, in launch order
        std::vector<int> kind, iter;  // kernel id and LP iteration per pair
    };
    // captured LP iteration graphs, keyed by (k, eff, mode, first iteration, iteration count, profiling);
    // a profiling graph owns the events recorded by its event-record nodes
    struct GraphEntry {
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
        ProfEvents prof;
    };
    std::map<std::tuple<int, int, int, int, int, int>, GraphEntry> graphs;
    bool use_graphs = true;
    bool capturing = false;
    ProfEvents capture_prof;               // events created while capturing a profiling graph
    bool profiling = false;
    ProfEvents prof_pending;               // pairs to read after the run
    std::vector<char> prof_owned;          // per pending pair: destroy after reading (direct launches)
    double prof_ms[5] = {0, 0, 0, 0, 0};
    long long prof_launches[5] = {0, 0, 0, 0, 0};
    double prof_bytes[5] = {0, 0, 0, 0, 0};
    cudaError_t launch_error = cudaSuccess;  // first failed launch that returns no status to its caller
    void *arena = nullptr;                 // every resident buffer of the graph (layout in graph_alloc)
    size_t arena_cap = 0;
    dmolp::ingest::Pool scratch;           // device scratch of the text parse, reused across loads
    // pinned staging ring of dmolp_graph_load_adjtext (allocated on first use)
    char *pin[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t pin_ev[4] = {nullptr, nullptr, nullptr, nullptr};
};

constexpr int kPinSlots = 4;
constexpr int64_t kPinSlot = 32ll << 20;  // bytes per staging slot
