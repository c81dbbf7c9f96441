// Host-side launchers of the DMOLP kernels (one translation unit per kernel family).
#pragma once

#include <utility>
#include <vector>

#include "device_state.cuh"

namespace dmolp {

// ---- host (hubsort.cpp) ----
// find_hub_nodes on (vertex, degree) pairs in the reference's map order, std::sort's tie order kept.
std::vector<int> hubs_from_pairs(std::vector<std::pair<int, int>> sd);
// The same on the raw degrees of one rank (pairs in map order, vertex V-1 down to 0, built on all threads).
std::vector<int> hubs_from_degrees(const int32_t *degree, int64_t nv);
// find_first_seed's (vertex, degree) over that order, its id-vs-degree tie test included.
std::pair<int, int> first_seed_of(const int32_t *degree, int64_t nv);

// ---- segmented radix select (select_kernels.cu) ----
// Records i < *n_dev carry a segment seg[i] in [0,nseg) (or -1: an empty slot, ignored) and a 64-bit key
// whose top bit is below `keybits`; keys are unique.  For every segment p, marks sel[i] = 1 on the need[p] records with the
// smallest keys (need[] is consumed).  sel[] must be zero on entry.  `stopped` (may be null) turns the
// launches into no-ops once it is non-zero.
// The LP window straight out of the selection: the key of a selected record slot holds its vertex and
// degree (key = (dk << ibits) | v, dk = maxdeg - deg when RE[label] > 1, else deg; label = its segment);
// v is stamped sstamp[v] = t, appended to win / nwin and to its decision-class list dec[c] / ndec[c], and
// its degree added to *te.  The segments' needs are min(n, ceil(*ratio * n)) for n = npart[seg] (the
// reference's ceil(e^(-t/5) n), gpu_lp_boundary.cu:244) instead of the need[] argument.
struct SplitArgs {
    const double *RE;
    const int32_t *npart;
    const double *ratio;
    int32_t *sstamp;
    int32_t *win;
    int *nwin;
    int32_t *dec[3];
    int *ndec;
    unsigned long long *te;
    unsigned long long *wsum;  // += window_mix(v) for every selected v
    int t, eff, ibits, maxdeg;
};
// first_hist_ready: the writer of the records has already added every record's first digit (bits
// [select_first_shift(keybits), +8) of its key) into histogram buffer 0 of c->b.hist, bin seg * 256 + digit.
void select_smallest(dmolp_ctx *c, const int32_t *seg, const uint64_t *key, const int *n_dev, int nseg, int keybits,
                     uint8_t *sel, const int *stopped, const SplitArgs *split = nullptr, bool first_hist_ready = false);
inline int select_first_shift(int keybits) { return ((keybits + kRadixBits - 1) / kRadixBits - 1) * kRadixBits; }
void select_prepare();  // kernel attributes; call once before any capture
// The LP window by degree bins (k_select_deg): the same window as select_smallest with `split`, for at most
// kDegSelMaxK labels, with the boundary test's superbin counts in b.dsup (BndArgs::dsup).  Returns false
// (nothing launched) for more labels.
bool select_window_deg(dmolp_ctx *c, int nseg, const SplitArgs &split, const int *stopped);
int select_binary_version();  // sm version of the loaded device code (major * 10 + minor), -1 on failure

// ---- LP loop (lp_kernels.cu) ----
struct LpLaunch {
    int k;
    int eff;       // labels scored: min(k,32) or k
    int mode;      // DMOLP_LP_MODE_*
};
void lp_check_symmetric(dmolp_ctx *c, unsigned long long *counts);  // *b.flag: a reverse is missing
void lp_symmetry_hash(dmolp_ctx *c, unsigned long long *sum, unsigned long long key);  // *sum += the multiset sum
void lp_fill(dmolp_ctx *c, int32_t *p, int64_t n, int32_t v);
void lp_degrees(dmolp_ctx *c, const int64_t *off, int64_t nv, int32_t *deg);  // deg[v] = off[v+1] - off[v]
void lp_reset_stats(dmolp_ctx *c, int k, const int *stopped);
// use_hot: the hot labels are current (lp_hot_refresh since the labels were last set outside the loop)
// keep_eff > 0: also write the kept label counts vcnt (labels < keep_eff <= 32) of every non-hub vertex
void lp_stats(dmolp_ctx *c, int k, const int *stopped, const int *skip, bool use_hot = false, int keep_eff = 0,
              int hub_eff = 0);  // hub_eff > 0: also every hub's label counts (hh), labels < hub_eff
void lp_hot_hist(dmolp_ctx *c);              // b.degh = histogram of min(degree, 65535), degree > 0
void lp_hot_build(dmolp_ctx *c, int dstar);  // vertices of degree >= dstar ranked; colh; b.flag = their number
void lp_hot_refresh(dmolp_ctx *c);           // hot labels from the resident labels
void lp_init_end(dmolp_ctx *c, int mode);
void lp_hub_index(dmolp_ctx *c);            // b.hidx from bucket[2] (once per graph)
// keeps it current; otherwise the selected hubs' rows are recounted.
void lp_iteration(dmolp_ctx *c, const LpLaunch &L, int t, bool first, bool last);
// one-off pieces used by dmolp_window_select / dmolp_lp_apply
void lp_window_from_list(dmolp_ctx *c, int k, int t, const double *RE_dev, int nprev);
void lp_apply_list(dmolp_ctx *c, int k, int eff, int n);

// ---- phase 1 (seed_kernels.cu) ----
void p1_mark_ball(dmolp_ctx *c, int seed);
void p1_hub_argmax(dmolp_ctx *c, int64_t nhubs);
void p1_init_labels(dmolp_ctx *c);
void p1_set_seeds(dmolp_ctx *c, const int32_t *seeds_dev, int nseeds);
void p1_fallback(dmolp_ctx *c, int best_part, int cur);
void p1_round(dmolp_ctx *c, int k, int theta, int cur);

}  // namespace dmolp
