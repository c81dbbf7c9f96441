// C-ABI of the batched phase 2 (include/dmolp_b200.h, dmolp_batch_*): upload of a batch of graphs as one
// union CSR, labels in and out, the captured persistent launch, and the launch-shape autotuner.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/dmolp_b200.h"
#include "batch.cuh"

namespace dmolp {
void set_last_error(const std::string &msg);  // dmolp_cabi.cu
}

using namespace dmolp;
using namespace dmolp::batch;

struct dmolp_batch {
    int device = 0, num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool has_graph = false;
    int ninst = 0;
    int64_t nv = 0, narcs = 0;
    std::vector<void *> allocations;
    Args a{};
    Inst *inst = nullptr;
    int32_t *order = nullptr, *saved = nullptr;
    int *err = nullptr;
    std::vector<Inst> h_inst;
    std::vector<Out> h_out;
    std::vector<long long> h_counts;
    bool tuned = false;
    dmolp_batch_tuning tuning{512, 16, 0, 0};
    std::map<std::tuple<int, int, int, int, int, int>, cudaGraphExec_t> graphs;
    // phase 1: per-vertex degrees on the host (for the hub lists), device work arrays, cached hub lists
    std::vector<int32_t> h_deg;
    std::vector<int64_t> h_vstart;
    bool have_hubs = false;
    P1Args p1{};
    uint8_t *p1_only = nullptr;
    std::vector<P1Out> h_p1;
};

namespace {

int fail(int code, const std::string &msg) {
    set_last_error(msg);
    return code;
}

#define BCUDA(call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(e_ == cudaErrorMemoryAllocation ? DMOLP_ERR_NOMEM : DMOLP_ERR_CUDA,           \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

template <typename T>
int balloc(dmolp_batch *b, T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DMOLP_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    b->allocations.push_back(q);
    *p = (T *)q;
    return DMOLP_OK;
}

void drop_graphs(dmolp_batch *b) {
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

void free_all(dmolp_batch *b) {
    drop_graphs(b);
    for (void *p : b->allocations) cudaFree(p);
    b->allocations.clear();
    b->a = Args();
    b->has_graph = false;
    b->tuned = false;
}

int bsync(dmolp_batch *b) {
    BCUDA(cudaStreamSynchronize(b->stream));
    BCUDA(cudaGetLastError());
    return DMOLP_OK;
}

#define BTRY(x)              \
    do {                     \
        int r_ = (x);        \
        if (r_) return r_;   \
    } while (0)

// Capture (once per shape and configuration) and launch the batch.
int run_graph(dmolp_batch *b, const dmolp_batch_tuning &t, const dmolp_lp_config &cfg) {
    const int occ = occupancy(t.block_threads, t.thread_row_max);
    if (occ <= 0) return fail(DMOLP_ERR_ARG, "unsupported launch shape");
    const int bps = t.blocks_per_sm <= 0 ? occ : std::min(t.blocks_per_sm, occ);
    const int grid = std::max(1, std::min(b->ninst, b->num_sms * bps));
    const auto key = std::make_tuple(t.block_threads, t.thread_row_max, grid, (int)cfg.mode, (int)cfg.iterations,
                                     (int)cfg.cap);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
        Args a = b->a;
        a.mode = cfg.mode;
        a.iters = cfg.iterations;
        a.cap = cfg.cap;
        cudaGraph_t g = nullptr;
        BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const bool ok = launch(a, t.block_threads, t.thread_row_max, grid, b->stream);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (!ok) {
            if (g) cudaGraphDestroy(g);
            return fail(DMOLP_ERR_ARG, "unsupported launch shape");
        }
        if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        cudaGraphExec_t ex = nullptr;
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        it = b->graphs.emplace(key, ex).first;
    }
    BCUDA(cudaGraphLaunch(it->second, b->stream));
    return DMOLP_OK;
}

int check_cfg(const dmolp_lp_config *cfg) {
    if (!cfg) return fail(DMOLP_ERR_ARG, "null config");
    if (cfg->mode != DMOLP_LP_MODE_REF && cfg->mode != DMOLP_LP_MODE_FIXED) return fail(DMOLP_ERR_ARG, "bad mode");
    if (cfg->mode == DMOLP_LP_MODE_FIXED && (cfg->iterations < 0 || cfg->iterations > kMaxIter))
        return fail(DMOLP_ERR_ARG, "iterations must be in [0, 500]");
    if (cfg->cap != DMOLP_LP_CAP_REF && cfg->cap != DMOLP_LP_CAP_FULL) return fail(DMOLP_ERR_ARG, "bad cap");
    return DMOLP_OK;
}

// The reference's balance = max over parts of count / expected (src/phase2/phase2.cpp:426-432).
void balance(const long long *vc, const long long *ec, int k, double *vb, double *eb) {
    long long tv = 0, te = 0;
    for (int p = 0; p < k; ++p) {
        tv += vc[p];
        te += ec[p];
    }
    const double ev = (double)tv / k;
    const double ee = te > 0 ? (double)te / k : 1.0;
    double mv = 0.0, me = 0.0;
    for (int p = 0; p < k; ++p) {
        mv = std::max(mv, ev > 0 ? (double)vc[p] / ev : 1.0);
        me = std::max(me, ee > 0 ? (double)ec[p] / ee : 1.0);
    }
    *vb = mv;
    *eb = me;
}

}  // namespace

namespace dmolp {
namespace batch {
bool view(dmolp_batch *b, View *v) {
    if (!b || !b->has_graph) return false;
    v->off = b->a.off;
    v->col = b->a.col;
    v->label = b->a.label;
    v->inst = b->inst;
    v->order = b->order;
    v->ninst = b->ninst;
    v->nv = b->nv;
    v->narcs = b->narcs;
    v->stream = b->stream;
    v->num_sms = b->num_sms;
    v->device = b->device;
    return true;
}
}  // namespace batch
}  // namespace dmolp

extern "C" {

int dmolp_batch_create(int device, dmolp_batch **out) {
    if (!out) return fail(DMOLP_ERR_ARG, "null output");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(DMOLP_ERR_NO_GPU, "no CUDA device");
    }
    if (device < 0 || device >= n) return fail(DMOLP_ERR_ARG, "device index out of range");
    BCUDA(cudaSetDevice(device));
    dmolp_batch *b = new dmolp_batch();
    b->device = device;
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
        delete b;
        return fail(DMOLP_ERR_CUDA, "stream / event creation failed");
    }
    *out = b;
    return DMOLP_OK;
}

int dmolp_batch_destroy(dmolp_batch *b) {
    if (!b) return DMOLP_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    free_all(b);
    cudaEventDestroy(b->ev0);
    cudaEventDestroy(b->ev1);
    cudaStreamDestroy(b->stream);
    delete b;
    return DMOLP_OK;
}

int dmolp_batch_upload(dmolp_batch *b, int32_t ninst, const int64_t *vstart, const int64_t *offsets,
                       const int32_t *indices, const int32_t *parts) {
    if (!b || ninst < 1 || !vstart || !offsets || !parts) return fail(DMOLP_ERR_ARG, "bad arguments");
    if (vstart[0] != 0) return fail(DMOLP_ERR_ARG, "vstart[0] must be 0");
    for (int i = 0; i < ninst; ++i) {
        if (vstart[i + 1] < vstart[i]) return fail(DMOLP_ERR_ARG, "vstart must be non-decreasing");
        if (parts[i] < 1 || parts[i] > DMOLP_BATCH_MAX_K)
            return fail(DMOLP_ERR_ARG, "parts[" + std::to_string(i) + "] outside [1, 64]");
    }
    const int64_t nv = vstart[ninst];
    if (nv >= (int64_t(1) << 31) - 1) return fail(DMOLP_ERR_ARG, "the batch must have fewer than 2^31 vertices");
    if (offsets[0] != 0) return fail(DMOLP_ERR_ARG, "offsets[0] must be 0");
    bool mono = true;
#pragma omp parallel for reduction(&& : mono)
    for (int64_t v = 0; v < nv; ++v) mono = mono && offsets[v + 1] >= offsets[v];
    if (!mono) return fail(DMOLP_ERR_ARG, "offsets must be non-decreasing");
    const int64_t narcs = offsets[nv];
    if (narcs > 0 && !indices) return fail(DMOLP_ERR_ARG, "null indices");
    BCUDA(cudaSetDevice(b->device));
    BCUDA(cudaStreamSynchronize(b->stream));
    free_all(b);
    Args &a = b->a;
    int32_t *label = nullptr, *newlab = nullptr, *cstamp = nullptr, *ndiff = nullptr, *lc = nullptr, *lb = nullptr, *la = nullptr,
            *w0 = nullptr, *w1 = nullptr, *col = nullptr, *order = nullptr, *saved = nullptr;
    int64_t *off = nullptr;
    Inst *inst = nullptr;
    Out *out = nullptr;
    long long *counts = nullptr;
    double *lt = nullptr, *rt = nullptr;
    int *ctr = nullptr;
    BTRY(balloc(b, &off, nv + 1));
    BTRY(balloc(b, &col, narcs));
    BTRY(balloc(b, &label, nv));
    BTRY(balloc(b, &newlab, nv));
    BTRY(balloc(b, &cstamp, nv));
    BTRY(balloc(b, &ndiff, nv));
    BTRY(balloc(b, &lc, nv));
    BTRY(balloc(b, &lb, nv));
    BTRY(balloc(b, &la, nv));
    BTRY(balloc(b, &w0, nv));
    BTRY(balloc(b, &w1, nv));
    BTRY(balloc(b, &saved, nv));
    BTRY(balloc(b, &inst, ninst));
    BTRY(balloc(b, &order, ninst));
    BTRY(balloc(b, &out, ninst));
    BTRY(balloc(b, &counts, (size_t)ninst * 2 * kBatchMaxK));
    BTRY(balloc(b, &lt, kMaxIter + 1));
    BTRY(balloc(b, &rt, kMaxIter + 1));
    BTRY(balloc(b, &ctr, 4));
    uint8_t *cov = nullptr, *seedm = nullptr, *selm = nullptr;
    int32_t *claim = nullptr, *seeds_out = nullptr;
    P1Out *p1out = nullptr;
    BTRY(balloc(b, &cov, nv));
    BTRY(balloc(b, &seedm, nv));
    BTRY(balloc(b, &selm, nv));
    BTRY(balloc(b, &claim, nv));
    BTRY(balloc(b, &seeds_out, (size_t)ninst * kBatchMaxK));
    BTRY(balloc(b, &p1out, ninst));
    std::vector<Inst> hi(ninst);
    for (int i = 0; i < ninst; ++i) {
        Inst &I = hi[i];
        I.vbase = vstart[i];
        I.nv = (int32_t)(vstart[i + 1] - vstart[i]);
        I.narcs = offsets[vstart[i + 1]] - offsets[vstart[i]];
        I.k = parts[i];
        I.maxdeg = I.ibits = I.dbits = I.symmetric = 0;
    }
    // largest instances first: the persistent CTAs take them in this order
    std::vector<int32_t> ord(ninst);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
        return hi[x].narcs + hi[x].nv > hi[y].narcs + hi[y].nv;
    });
    // log(t) and e^(-t/5) with the host's libm, as the reference computes them (phase2.cpp:199,
    // gpu_lp_boundary.cu:244)
    std::vector<double> hl(kMaxIter + 1, 0.0), hr(kMaxIter + 1, 1.0);
    for (int t = 1; t <= kMaxIter; ++t) {
        hl[t] = std::log((double)t);
        hr[t] = std::exp((-t) / (5.0));
    }
    cudaStream_t s = b->stream;
    BCUDA(cudaMemcpyAsync(off, offsets, (nv + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    if (narcs) BCUDA(cudaMemcpyAsync(col, indices, narcs * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    BCUDA(cudaMemcpyAsync(inst, hi.data(), ninst * sizeof(Inst), cudaMemcpyHostToDevice, s));
    BCUDA(cudaMemcpyAsync(order, ord.data(), ninst * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    BCUDA(cudaMemcpyAsync(lt, hl.data(), hl.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    BCUDA(cudaMemcpyAsync(rt, hr.data(), hr.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    BCUDA(cudaMemsetAsync(label, 0, nv * sizeof(int32_t), s));
    BCUDA(cudaMemsetAsync(newlab, 0xff, nv * sizeof(int32_t), s));
    BCUDA(cudaMemsetAsync(cstamp, 0, nv * sizeof(int32_t), s));
    BCUDA(cudaMemsetAsync(ndiff, 0, nv * sizeof(int32_t), s));
    BCUDA(cudaMemsetAsync(ctr, 0, 4 * sizeof(int), s));
    prepare(off, col, inst, ninst, ctr, ctr + 2, b->num_sms * 4, s);
    BTRY(bsync(b));
    int h_err = 0;
    BCUDA(cudaMemcpy(&h_err, ctr + 2, sizeof(int), cudaMemcpyDeviceToHost));
    if (h_err) {
        free_all(b);
        return fail(DMOLP_ERR_ARG, "instance " + std::to_string(h_err - 1) + ": neighbour id outside its graph");
    }
    BCUDA(cudaMemcpy(hi.data(), inst, ninst * sizeof(Inst), cudaMemcpyDeviceToHost));
    a.off = off;
    a.col = col;
    a.label = label;
    a.newlab = newlab;
    a.cstamp = cstamp;
    a.ndiff = ndiff;
    a.l_cand = lc;
    a.l_bnd = lb;
    a.l_act = la;
    a.l_win0 = w0;
    a.l_win1 = w1;
    a.inst = inst;
    a.order = order;
    a.ninst = ninst;
    a.next = ctr;
    a.stamp_base = ctr + 1;
    a.out = out;
    a.counts = counts;
    a.logtab = lt;
    a.ratiotab = rt;
    b->inst = inst;
    b->order = order;
    b->saved = saved;
    b->err = ctr + 2;
    b->h_inst = hi;
    b->h_out.assign(ninst, Out());
    b->h_counts.assign((size_t)ninst * 2 * kBatchMaxK, 0);
    b->ninst = ninst;
    b->nv = nv;
    b->narcs = narcs;
    // phase 1: host degrees (hub lists are computed on the first dmolp_batch_phase1 call)
    b->h_deg.resize(nv);
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < nv; ++v) b->h_deg[v] = (int32_t)(offsets[v + 1] - offsets[v]);
    b->h_vstart.assign(vstart, vstart + ninst + 1);
    b->have_hubs = false;
    b->p1_only = nullptr;
    P1Args &q = b->p1;
    q = P1Args();
    q.off = off;
    q.col = col;
    q.label = label;
    q.inst = inst;
    q.order = order;
    q.ninst = ninst;
    q.next = ctr + 3;
    q.cov = cov;
    q.seedm = seedm;
    q.sel = selm;
    q.claim = claim;
    q.l_front0 = w0;
    q.l_front1 = w1;
    q.l_claim = lb;
    q.l_act0 = lc;
    q.l_act1 = la;
    q.seeds_out = seeds_out;
    q.out = p1out;
    b->h_p1.assign(ninst, P1Out());
    b->has_graph = true;
    return DMOLP_OK;
}

int dmolp_batch_labels_set(dmolp_batch *b, const int32_t *labels) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    if (!labels) return fail(DMOLP_ERR_ARG, "null labels");
    BCUDA(cudaSetDevice(b->device));
    BCUDA(cudaMemcpyAsync(b->a.label, labels, b->nv * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream));
    return bsync(b);
}

int dmolp_batch_labels_get(dmolp_batch *b, int32_t *labels) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    if (!labels) return fail(DMOLP_ERR_ARG, "null labels");
    BCUDA(cudaSetDevice(b->device));
    BCUDA(cudaMemcpyAsync(labels, b->a.label, b->nv * sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream));
    return bsync(b);
}

int dmolp_batch_labels_save(dmolp_batch *b) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    BCUDA(cudaSetDevice(b->device));
    BCUDA(cudaMemcpyAsync(b->saved, b->a.label, b->nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, b->stream));
    return DMOLP_OK;
}

int dmolp_batch_labels_restore(dmolp_batch *b) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    BCUDA(cudaSetDevice(b->device));
    BCUDA(cudaMemcpyAsync(b->a.label, b->saved, b->nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, b->stream));
    return DMOLP_OK;
}

int dmolp_batch_device_labels(dmolp_batch *b, int32_t **labels) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    if (!labels) return fail(DMOLP_ERR_ARG, "null output");
    *labels = b->a.label;
    return DMOLP_OK;
}

void *dmolp_batch_stream(dmolp_batch *b) { return b ? (void *)b->stream : nullptr; }

int dmolp_batch_lp_run(dmolp_batch *b, const dmolp_lp_config *cfg, const dmolp_batch_tuning *tune,
                       dmolp_batch_result *results, double *gpu_ms) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    BTRY(check_cfg(cfg));
    BCUDA(cudaSetDevice(b->device));
    const dmolp_batch_tuning t = tune ? *tune : b->tuning;
    BCUDA(cudaEventRecord(b->ev0, b->stream));
    BTRY(run_graph(b, t, *cfg));
    BCUDA(cudaEventRecord(b->ev1, b->stream));
    const int n = b->ninst;
    BCUDA(cudaMemcpyAsync(b->h_out.data(), b->a.out, n * sizeof(Out), cudaMemcpyDeviceToHost, b->stream));
    if (results)
        BCUDA(cudaMemcpyAsync(b->h_counts.data(), b->a.counts, b->h_counts.size() * sizeof(long long),
                              cudaMemcpyDeviceToHost, b->stream));
    BTRY(bsync(b));
    if (gpu_ms) {
        float ms = 0;
        BCUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        *gpu_ms = ms;
    }
    int first_bad = -1;
    for (int i = 0; i < n; ++i) {
        const Out &o = b->h_out[i];
        if (o.status != DMOLP_OK && first_bad < 0) first_bad = i;
        if (!results) continue;
        dmolp_batch_result &r = results[i];
        r.edge_cut = o.edge_cut;
        r.traversed_edges = (uint64_t)o.te;
        r.arcs_read = (uint64_t)o.arcs;
        r.vertex_visits = (uint64_t)o.visits;
        r.iterations_run = o.iterations;
        r.stop_reason = o.stop_reason;
        r.status = o.status;
        r.changes = o.changes;
        const long long *c = b->h_counts.data() + (size_t)i * 2 * kBatchMaxK;
        balance(c, c + kBatchMaxK, b->h_inst[i].k, &r.vertex_balance, &r.edge_balance);
    }
    if (first_bad >= 0)
        return fail(DMOLP_ERR_BAD_LABELS,
                    "instance " + std::to_string(first_bad) + ": label outside [0,k) or odd cut-arc count");
    return DMOLP_OK;
}

int dmolp_batch_autotune(dmolp_batch *b, const dmolp_lp_config *cfg, dmolp_batch_tuning *best, double *best_ms) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    BTRY(check_cfg(cfg));
    BCUDA(cudaSetDevice(b->device));
    const size_t lb = b->nv * sizeof(int32_t);
    BCUDA(cudaMemcpyAsync(b->saved, b->a.label, lb, cudaMemcpyDeviceToDevice, b->stream));
    dmolp_batch_tuning bt{0, 0, 0, 0};
    double bms = 1e300;
    for (int nt : {256, 512, 1024})
        for (int td : {8, 16}) {
            const int occ = occupancy(nt, td);
            for (int bps = 1; bps <= occ; bps *= 2) {
                const dmolp_batch_tuning t{nt, td, bps, 0};
                double ms = 0;
                for (int rep = 0; rep < 2; ++rep) {  // first run captures and warms up
                    BCUDA(cudaMemcpyAsync(b->a.label, b->saved, lb, cudaMemcpyDeviceToDevice, b->stream));
                    const int r = dmolp_batch_lp_run(b, cfg, &t, nullptr, &ms);
                    if (r != DMOLP_OK && r != DMOLP_ERR_BAD_LABELS) return r;
                }
                if (ms < bms) {
                    bms = ms;
                    bt = t;
                }
            }
        }
    BCUDA(cudaMemcpyAsync(b->a.label, b->saved, lb, cudaMemcpyDeviceToDevice, b->stream));
    BTRY(bsync(b));
    b->tuning = bt;
    b->tuned = true;
    if (best) *best = bt;
    if (best_ms) *best_ms = bms;
    return DMOLP_OK;
}

int dmolp_batch_phase1(dmolp_batch *b, int theta, const uint8_t *only, int32_t *seeds, dmolp_batch_p1_result *results,
                       double *gpu_ms) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    if (theta < 1) return fail(DMOLP_ERR_ARG, "theta must be >= 1 (with theta = 0 the reference never ends)");
    BCUDA(cudaSetDevice(b->device));
    const int n = b->ninst;
    P1Args &q = b->p1;
    if (!b->have_hubs) {
        // hub lists and first seeds per graph, in the reference's order (init.cpp:139-187)
        std::vector<std::vector<int>> hubs(n);
        std::vector<int32_t> first(n, 0), first_hub(n, -1);
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 0; i < n; ++i) {
            const int64_t v0 = b->h_vstart[i], v1 = b->h_vstart[i + 1];
            std::vector<int32_t> deg(b->h_deg.begin() + v0, b->h_deg.begin() + v1);
            hubs[i] = hubs_of(deg);
            std::pair<int, int> f(-1, -1);
            for (int64_t v = v1 - v0 - 1; v >= 0; --v) {  // init.cpp:179-187, with its id-vs-degree tie test
                const int d = deg[v];
                if (d > f.second || (d == f.second && (int)v < f.second)) f = std::make_pair((int)v, d);
            }
            first[i] = f.first < 0 ? 0 : f.first;
            auto it = std::find(hubs[i].begin(), hubs[i].end(), f.first);
            first_hub[i] = it == hubs[i].end() ? -1 : (int32_t)(it - hubs[i].begin());
        }
        std::vector<int64_t> hstart(n + 1, 0);
        for (int i = 0; i < n; ++i) hstart[i + 1] = hstart[i] + (int64_t)hubs[i].size();
        std::vector<int32_t> flat(std::max<int64_t>(1, hstart[n]));
        for (int i = 0; i < n; ++i) std::copy(hubs[i].begin(), hubs[i].end(), flat.begin() + hstart[i]);
        int32_t *dh = nullptr, *df = nullptr, *dfh = nullptr;
        int64_t *dhs = nullptr;
        uint8_t *used = nullptr;
        BTRY(balloc(b, &dh, flat.size()));
        BTRY(balloc(b, &dhs, n + 1));
        BTRY(balloc(b, &df, n));
        BTRY(balloc(b, &dfh, n));
        BTRY(balloc(b, &used, flat.size()));
        BCUDA(cudaMemcpyAsync(dh, flat.data(), flat.size() * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream));
        BCUDA(cudaMemcpyAsync(dhs, hstart.data(), (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, b->stream));
        BCUDA(cudaMemcpyAsync(df, first.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream));
        BCUDA(cudaMemcpyAsync(dfh, first_hub.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream));
        BTRY(bsync(b));
        q.hubs = dh;
        q.hstart = dhs;
        q.first = df;
        q.first_hub = dfh;
        q.hub_used = used;
        b->have_hubs = true;
    }
    q.theta = theta;
    q.only = nullptr;
    if (only) {
        if (!b->p1_only) BTRY(balloc(b, &b->p1_only, n));
        BCUDA(cudaMemcpyAsync(b->p1_only, only, n, cudaMemcpyHostToDevice, b->stream));
        q.only = b->p1_only;
    }
    BCUDA(cudaMemsetAsync(q.out, 0, n * sizeof(P1Out), b->stream));
    BCUDA(cudaEventRecord(b->ev0, b->stream));
    launch_p1(q, std::max(1, std::min(n, b->num_sms * 2)), b->stream);
    BCUDA(cudaGetLastError());
    BCUDA(cudaEventRecord(b->ev1, b->stream));
    BCUDA(cudaMemcpyAsync(b->h_p1.data(), q.out, n * sizeof(P1Out), cudaMemcpyDeviceToHost, b->stream));
    if (seeds)
        BCUDA(cudaMemcpyAsync(seeds, q.seeds_out, (size_t)n * kBatchMaxK * sizeof(int32_t), cudaMemcpyDeviceToHost,
                              b->stream));
    BTRY(bsync(b));
    if (gpu_ms) {
        float ms = 0;
        BCUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        *gpu_ms = ms;
    }
    if (seeds)  // union ids -> ids inside each graph
        for (int i = 0; i < n; ++i)
            for (int p = 0; p < kBatchMaxK; ++p) {
                int32_t &s = seeds[(size_t)i * kBatchMaxK + p];
                if (s >= 0) s -= (int32_t)b->h_vstart[i];
            }
    if (results)
        for (int i = 0; i < n; ++i) {
            results[i].num_seeds_found = b->h_p1[i].nseeds_found;
            results[i].rounds = b->h_p1[i].rounds;
            results[i].traversed_edges = b->h_p1[i].te;
        }
    return DMOLP_OK;
}

int dmolp_batch_counts(dmolp_batch *b, int32_t inst, int64_t *vertex_counts, int64_t *edge_counts) {
    if (!b || !b->has_graph) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    if (inst < 0 || inst >= b->ninst) return fail(DMOLP_ERR_ARG, "instance index out of range");
    BCUDA(cudaSetDevice(b->device));
    std::vector<long long> c(2 * kBatchMaxK);
    BCUDA(cudaMemcpy(c.data(), b->a.counts + (size_t)inst * 2 * kBatchMaxK, c.size() * sizeof(long long),
                     cudaMemcpyDeviceToHost));
    const int k = b->h_inst[inst].k;
    for (int p = 0; p < k; ++p) {
        if (vertex_counts) vertex_counts[p] = c[p];
        if (edge_counts) edge_counts[p] = c[kBatchMaxK + p];
    }
    return DMOLP_OK;
}

}  // extern "C"
