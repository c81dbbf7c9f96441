// C-ABI entry points (include/dmolp_b200.h): context, resident graph, phase 1, phase 2, metrics.
//
// Host-side steps that decide ORDER-dependent results stay on the host, in the reference's exact form:
// the hub sort (an unstable std::sort over vertices V-1..0, src/phase1/init.cpp:139-177) and the first-seed
// scan (init.cpp:179-187).  Everything that touches the graph's arcs runs on the device.
#include <fcntl.h>
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/dmolp_b200.h"
#include "ingest.cuh"
#include "kernels.cuh"

using namespace dmolp;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define DMOLP_CUDA(call)                                                                              \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(e_ == cudaErrorMemoryAllocation ? DMOLP_ERR_NOMEM : DMOLP_ERR_CUDA,           \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

int bits_for(int64_t x) {
    int b = 1;
    while (b < 62 && (int64_t(1) << b) <= x) ++b;
    return b;
}

template <typename T>
int dalloc(dmolp_ctx *c, T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DMOLP_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    c->allocations.push_back(q);
    *p = (T *)q;
    return DMOLP_OK;
}

void drop_graphs(dmolp_ctx *c) {
    for (auto &kv : c->graphs) {
        cudaGraphExecDestroy(kv.second.exec);
        for (cudaEvent_t e : kv.second.prof.ev) cudaEventDestroy(e);
    }
    c->graphs.clear();
}

void free_all(dmolp_ctx *c) {
    drop_graphs(c);
    for (void *p : c->allocations) cudaFree(p);
    c->allocations.clear();
    c->saved_labels = nullptr;
    c->b = Buffers();
    c->has_graph = false;
}

int check_launch(dmolp_ctx *c) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    (void)c;
    return DMOLP_OK;
}

int sync(dmolp_ctx *c) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
    return check_launch(c);
}

// Clears the degree-bin selection's counts (superbin counts; fine-bin and tail counts of both parities).
int clear_select_bins(dmolp_ctx *c) {
    Buffers &b = c->b;
    DMOLP_CUDA(cudaMemsetAsync(b.dsup, 0, (size_t)kDegSelMaxK * kDsBins * sizeof(unsigned int), c->stream));
    for (int i = 0; i < 2; ++i)
        DMOLP_CUDA(cudaMemsetAsync(b.dfine[i], 0, (size_t)kDegSelMaxK * kDsFine * sizeof(unsigned int), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.dtcnt, 0, 2 * kDegSelMaxK * sizeof(int), c->stream));
    return DMOLP_OK;
}

// A grid barrier of a cooperative selection that gave up waiting (its blocks are co-resident, so only a
// wait limit far below the default makes this happen): report it, and clear the barrier state and the
// selections' counts for the next launch.
int check_waits(dmolp_ctx *c) {
    if (c->launch_error != cudaSuccess) {
        const cudaError_t e = c->launch_error;
        c->launch_error = cudaSuccess;
        cudaGetLastError();
        return fail(DMOLP_ERR_CUDA, std::string("window selection launch: ") + cudaGetErrorString(e));
    }
    int to = 0;
    DMOLP_CUDA(cudaMemcpyAsync(&to, &c->b.ctrl->wait_timeout, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    int st = sync(c);
    if (st) return st;
    if (!to) return DMOLP_OK;
    // bar_count, bar_gen, wait_timeout are adjacent
    DMOLP_CUDA(cudaMemsetAsync(&c->b.ctrl->bar_count, 0, 3 * sizeof(int), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(c->b.hist, 0, (size_t)kSelHistBuffers * DMOLP_MAX_K * kRadix * sizeof(unsigned int),
                               c->stream));
    int st2 = clear_select_bins(c);
    if (st2) return st2;
    sync(c);
    return fail(DMOLP_ERR_CUDA, "grid barrier " + std::to_string(to - 1) +
                                    " of a window selection gave up waiting (wait limit " +
                                    std::to_string(c->wait_polls) + " polls)");
}

// The reference's balance = max over parts of count / expected (src/phase2/phase2.cpp:426-432).
void balances(const std::vector<long long> &vc, const std::vector<long long> &ec, int k, double *vb, double *eb,
              int64_t *tv_out, int64_t *te_out) {
    long long tv = 0, te = 0;
    for (int p = 0; p < k; ++p) {
        tv += vc[p];
        te += ec[p];
    }
    const double ev = (double)tv / k;
    const double ee = te > 0 ? (double)te / k : 1.0;
    double mv = 0.0, me = 0.0;
    for (int p = 0; p < k; ++p) {
        const double rv = ev > 0 ? (double)vc[p] / ev : 1.0;
        const double re = ee > 0 ? (double)ec[p] / ee : 1.0;
        mv = std::max(mv, rv);
        me = std::max(me, re);
    }
    *vb = mv;
    *eb = me;
    if (tv_out) *tv_out = tv;
    if (te_out) *te_out = te;
}

// Fused cut/balance pass over the resident labels; fills host copies.  Returns the status.
int run_stats(dmolp_ctx *c, int k, unsigned long long *cut_arcs, std::vector<long long> &vc,
              std::vector<long long> &intra, int *bad) {
    lp_reset_stats(c, k, nullptr);
    lp_stats(c, k, nullptr, nullptr);
    std::vector<unsigned long long> hv(k), hi(k);
    LpCounters cn;
    LpControl ctl;
    DMOLP_CUDA(cudaMemcpyAsync(hv.data(), c->b.vc, k * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(hi.data(), c->b.intra, k * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(&cn, c->b.cnt, sizeof(cn), cudaMemcpyDeviceToHost, c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(&ctl, c->b.ctrl, sizeof(ctl), cudaMemcpyDeviceToHost, c->stream));
    int st = sync(c);
    if (st) return st;
    vc.assign(k, 0);
    intra.assign(k, 0);
    for (int p = 0; p < k; ++p) {
        vc[p] = (long long)hv[p];
        intra[p] = (long long)hi[p];
    }
    *cut_arcs = cn.cut_arcs;
    *bad = ctl.error;
    return DMOLP_OK;
}

// src/phase1/init.cpp:139-177 (see the comment at the top of this file): pairs in the order the reference's
// degree map iterates at one rank (V-1..0), sorted with std::sort's exact permutation on all host threads.
std::vector<int> find_hubs(const std::vector<int32_t> &raw) {
    return dmolp::hubs_from_degrees(raw.data(), (int64_t)raw.size());
}

// Capture (once) and launch the iterations [t0, t0+cnt) of an LP run as one CUDA graph.
int run_block_graph(dmolp_ctx *c, const LpLaunch &L, int t0, int cnt) {
    const auto key = std::make_tuple(L.k, L.eff, L.mode, t0, cnt, c->profiling ? 1 : 0);
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
        cudaGraph_t g = nullptr;
        dmolp_ctx::GraphEntry ge;
        const long long before = c->launches;
        DMOLP_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->capturing = true;
        c->capture_prof = dmolp_ctx::ProfEvents();
        for (int t = t0; t < t0 + cnt; ++t) lp_iteration(c, L, t, t == t0, t == t0 + cnt - 1);
        c->capturing = false;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        ge.kernels = c->launches - before;
        ge.prof = c->capture_prof;
        c->launches = before;
        if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ge.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        it = c->graphs.emplace(key, ge).first;
    }
    DMOLP_CUDA(cudaGraphLaunch(it->second.exec, c->stream));
    c->launches += it->second.kernels;
    const dmolp_ctx::ProfEvents &pe = it->second.prof;
    for (size_t i = 0; i < pe.kind.size(); ++i) {
        c->prof_pending.ev.push_back(pe.ev[2 * i]);
        c->prof_pending.ev.push_back(pe.ev[2 * i + 1]);
        c->prof_pending.kind.push_back(pe.kind[i]);
        c->prof_pending.iter.push_back(pe.iter[i]);
        c->prof_owned.push_back(0);
    }
    return DMOLP_OK;
}

}  // namespace

namespace dmolp {
void set_last_error(const std::string &msg) { g_err = msg; }
std::vector<int> hubs_of(const std::vector<int32_t> &degree) { return find_hubs(degree); }
}  // namespace dmolp

namespace {

// Places buffer `p` of n elements at the next 256-byte boundary of the arena (only sizes it when base is null).
template <typename T>
void place(char *base, size_t &off, T **p, size_t n) {
    off = (off + 255) & ~(size_t)255;
    if (base) *p = reinterpret_cast<T *>(base + off);
    off += std::max<size_t>(n, 1) * sizeof(T);
}

// Byte layout of every resident buffer of a graph inside one arena; returns the arena size.  With base null
// only the size is computed.
size_t layout(dmolp_ctx *c, char *base, int64_t nv, int64_t narcs, const size_t nball[3]) {
    Buffers &b = c->b;
    const size_t n = (size_t)nv + 1;
    size_t off = 0;
#define ALLOC(ptr, count) place(base, off, &(ptr), (count))
    ALLOC(b.off, n);
    ALLOC(b.col, (size_t)narcs);
    ALLOC(b.rawdeg, n);
    ALLOC(b.label, n);
    ALLOC(b.stamp, n);
    ALLOC(b.sstamp, n);
    ALLOC(b.ndiff, n);
    ALLOC(b.cand, n);
    ALLOC(b.win[0], n);
    ALLOC(b.win[1], n);
    ALLOC(b.bv, n);
    ALLOC(b.bown, n);
    ALLOC(b.bnew, n);
    ALLOC(b.bkey, n);
    ALLOC(b.bsel, n);
    ALLOC(b.active[0], n);
    ALLOC(b.active[1], n);
    ALLOC(b.hist, (size_t)kSelHistBuffers * DMOLP_MAX_K * kRadix);
    ALLOC(b.dsup, (size_t)kDegSelMaxK * kDsBins);
    ALLOC(b.dfine[0], (size_t)kDegSelMaxK * kDsFine);
    ALLOC(b.dfine[1], (size_t)kDegSelMaxK * kDsFine);
    ALLOC(b.dcntb, (size_t)c->num_sms * kDegSelMaxK * kDsFine);
    ALLOC(b.dtcnt, 2 * kDegSelMaxK);
    ALLOC(b.dlkey, n);
    ALLOC(b.dtkey, n);
    ALLOC(b.need, DMOLP_MAX_K);
    ALLOC(b.sel_below, DMOLP_MAX_K);
    ALLOC(b.keep_digit, DMOLP_MAX_K);
    ALLOC(b.npart, DMOLP_MAX_K);
    ALLOC(b.vc, DMOLP_MAX_K);
    ALLOC(b.intra, DMOLP_MAX_K);
    ALLOC(b.psize, DMOLP_MAX_K);
    ALLOC(b.tpen, DMOLP_MAX_K);
    ALLOC(b.RE, DMOLP_MAX_K);
    ALLOC(b.penhist, (size_t)kMaxIter * DMOLP_MAX_K);
    ALLOC(b.cnthist, (size_t)kMaxIter * 2 * DMOLP_MAX_K);
    ALLOC(b.logtab, kMaxIter + 1);
    ALLOC(b.ratiotab, kMaxIter + 1);
    ALLOC(b.cnt, 1);
    ALLOC(b.ctrl, 1);
    ALLOC(b.rec, kMaxIter);
    ALLOC(b.covered, n);
    ALLOC(b.hubs, n);
    ALLOC(b.hub_used, n);
    ALLOC(b.best, 1);
    ALLOC(b.p1cnt, 8);
    ALLOC(b.p1te, 1);
    ALLOC(b.flag, 1);
    ALLOC(b.symcnt, 2);
    ALLOC(b.ball, nball[0] + nball[1] + nball[2]);
    if (base) {
        b.bucket[0] = b.ball;
        b.bucket[1] = b.ball + nball[0];
        b.bucket[2] = b.bucket[1] + nball[1];
    }
    for (int i = 0; i < 3; ++i) ALLOC(b.dec[i], n);
    ALLOC(b.newlab, n);
    ALLOC(b.mov, n);
    ALLOC(b.chunkq, (size_t)c->chunk_cap);
    ALLOC(b.hubq, (size_t)c->hubq_cap);
    ALLOC(b.hh, nball[2] * (size_t)DMOLP_MAX_K);
    ALLOC(b.hidx, n);
    ALLOC(b.hubwin, n);
    ALLOC(b.hub_in, nball[2]);
    ALLOC(b.hubwq, (size_t)c->hubq_cap);
    ALLOC(b.colh, (size_t)narcs);
    ALLOC(b.hrank, n);
    ALLOC(b.hotid, kHotMax);
    ALLOC(b.hotlab, kHotMax);
    ALLOC(b.degh, 65536);
    ALLOC(b.vcnt, n * 32);
#undef ALLOC
    return off;
}

// Frees the previous graph's state and lays out every resident buffer for a graph of the given sizes in
// the context's arena: one allocation, kept for later graphs that fit (it grows to the largest graph
// uploaded on the context).  Repeated uploads then allocate nothing.
int graph_alloc(dmolp_ctx *c, int64_t nv, int64_t narcs, int64_t maxdeg, int64_t maxraw, const int64_t nbc[3]) {
    DMOLP_CUDA(cudaStreamSynchronize(c->stream));
    free_all(c);
    c->nv = nv;
    c->narcs = narcs;
    c->maxdeg = maxdeg;
    c->maxraw = maxraw;
    c->ibits = bits_for(nv > 0 ? nv - 1 : 0);
    c->dbits = bits_for(maxdeg);
    c->rbits = bits_for(maxraw);
    for (int i = 0; i < 3; ++i) c->nb[i] = (int)nbc[i];
    c->chunk_cap = narcs / kChunk + 2;
    c->hubq_cap = narcs / kHubChunk + nbc[2] + 2;
    const size_t nball[3] = {(size_t)nbc[0], (size_t)nbc[1], (size_t)nbc[2]};
    const size_t need = layout(c, nullptr, nv, narcs, nball);
    if (need > c->arena_cap) {
        if (c->arena) cudaFree(c->arena);
        c->arena = nullptr;
        c->arena_cap = 0;
        cudaError_t e = cudaMalloc(&c->arena, need);
        if (e != cudaSuccess) {
            cudaGetLastError();
            c->arena = nullptr;
            return fail(DMOLP_ERR_NOMEM, std::string("cudaMalloc (graph arena): ") + cudaGetErrorString(e));
        }
        c->arena_cap = need;
    }
    layout(c, (char *)c->arena, nv, narcs, nball);
    c->b.claim = c->b.stamp;  // phase 1 and the LP loop never run at the same time
    return DMOLP_OK;
}

// After off, col, rawdeg and the degree-class lists are on the device: clears the loop state, tests
// whether every arc has its reverse (when rows are strictly increasing) and loads the log / exp tables.
int graph_finish(dmolp_ctx *c, bool rows_sorted) {
    Buffers &b = c->b;
    const int64_t nv = c->nv;
    const size_t n = (size_t)nv + 1;
    DMOLP_CUDA(cudaMemsetAsync(b.label, 0, n * sizeof(int32_t), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.hist, 0, (size_t)kSelHistBuffers * DMOLP_MAX_K * kRadix * sizeof(unsigned int),
                               c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.ctrl, 0, sizeof(LpControl), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.cnt, 0, sizeof(LpCounters), c->stream));
    {
        const int st0 = clear_select_bins(c);
        if (st0) return st0;
    }
    const int npos = c->nb[0] + c->nb[1] + c->nb[2];
    DMOLP_CUDA(cudaMemcpyAsync(&b.cnt->npos, &npos, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.bown, 0xff, n * sizeof(int32_t), c->stream));  // all record slots empty
    lp_fill(c, b.newlab, (int64_t)n, -1);
    lp_fill(c, b.hrank, (int64_t)n, -1);  // no hot set until the first LP run builds it
    c->hot_ready = false;
    c->nhot = 0;
    c->lp_runs = 0;
    lp_hub_index(c);
    select_prepare();
    // whether every arc has its reverse is tested when the LP loop first needs it (ensure_symmetry)
    c->symmetric = false;
    c->symmetry_known = false;
    c->rows_sorted = rows_sorted;
    // log(t) and e^(-t/5) with the host's libm, as the reference computes them (phase2.cpp:199,
    // gpu_lp_boundary.cu:244)
    std::vector<double> lt(kMaxIter + 1, 0.0), rt(kMaxIter + 1, 1.0);
    for (int t = 1; t <= kMaxIter; ++t) {
        lt[t] = std::log((double)t);
        rt[t] = std::exp((-t) / (5.0));
    }
    DMOLP_CUDA(cudaMemcpyAsync(b.logtab, lt.data(), lt.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(b.ratiotab, rt.data(), rt.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    int s2 = sync(c);
    if (s2) return s2;
    c->has_graph = true;
    return DMOLP_OK;
}

// The hot set of the resident graph, built the first time the LP loop runs on it: the vertices of the
// highest degrees, at most kHotMax (all of degree >= d*, d* the smallest degree for which they fit).
int lp_hot_prepare(dmolp_ctx *c) {
    if (c->hot_ready) return DMOLP_OK;
    Buffers &b = c->b;
    std::vector<unsigned int> h(65536);
    lp_hot_hist(c);
    DMOLP_CUDA(cudaMemcpyAsync(h.data(), b.degh, h.size() * sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
    int s = sync(c);
    if (s) return s;
    long long acc = 0;
    int dstar = 0;
    for (int d = 65535; d >= 1; --d) {
        if (acc + h[d] > kHotMax) break;
        acc += h[d];
        dstar = d;
    }
    c->nhot = 0;
    if (acc > 0) {
        DMOLP_CUDA(cudaMemsetAsync(b.flag, 0, sizeof(int), c->stream));
        lp_hot_build(c, dstar);
        c->nhot = (int)acc;
    }
    c->hot_ready = true;
    return check_launch(c);
}

// Whether every arc has its reverse, tested on the device the first time the LP loop needs it (then the
// loop may update cut and balance from the movers alone); graphs whose rows are not strictly increasing
// always take the full statistics pass.  By default one streaming pass forms the keyed multiset sum (zero
// for every symmetric graph; zero for an asymmetric one with probability about 2^-64); with
// dmolp_set_symmetry_test(ctx, 1) every reverse arc is looked up instead.
int ensure_symmetry(dmolp_ctx *c) {
    if (c->symmetry_known) return DMOLP_OK;
    Buffers &b = c->b;
    c->symmetric = false;
    if (c->rows_sorted && c->nv > 0) {
        DMOLP_CUDA(cudaMemsetAsync(b.flag, 0, sizeof(int), c->stream));
        DMOLP_CUDA(cudaMemsetAsync(b.symcnt, 0, 2 * sizeof(unsigned long long), c->stream));
        if (c->symmetry_exact) lp_check_symmetric(c, b.symcnt);
        else lp_symmetry_hash(c, b.symcnt, c->sym_key);
        int missing = 1;
        unsigned long long hc[2] = {0, 1};
        DMOLP_CUDA(cudaMemcpyAsync(&missing, b.flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        DMOLP_CUDA(cudaMemcpyAsync(hc, b.symcnt, sizeof(hc), cudaMemcpyDeviceToHost, c->stream));
        int s1 = sync(c);
        if (s1) return s1;
        c->symmetric = c->symmetry_exact ? (missing == 0 && hc[0] == hc[1]) : hc[0] == 0;
    }
    c->symmetry_known = true;
    return DMOLP_OK;
}

// Device buffer (parse scratch) for `len` bytes of text, padded to whole parse tiles (padding zeroed).
int text_buffer(dmolp_ctx *c, int64_t len, uint8_t **out) {
    const int64_t cap = ingest::padded_bytes(len);
    std::string err;
    *out = (uint8_t *)c->scratch.get(ingest::kText, (size_t)cap, err);
    if (!*out) return fail(DMOLP_ERR_NOMEM, err);
    DMOLP_CUDA(cudaMemsetAsync(*out + len, 0, (size_t)(cap - len), c->stream));
    return DMOLP_OK;
}

int pinned_ring(dmolp_ctx *c) {
    for (int s = 0; s < kPinSlots; ++s) {
        if (!c->pin[s]) DMOLP_CUDA(cudaHostAlloc((void **)&c->pin[s], kPinSlot, cudaHostAllocDefault));
        if (!c->pin_ev[s]) DMOLP_CUDA(cudaEventCreateWithFlags(&c->pin_ev[s], cudaEventDisableTiming));
    }
    return DMOLP_OK;
}

// Parse the text on the device into the resident CSR.  A text the parse rejects leaves the previous graph
// in place; a CUDA failure after that leaves no graph.
int ingest_text(dmolp_ctx *c, uint8_t *d_txt, int64_t len, int64_t body0, int64_t body1, dmolp_ingest_info *info) {
    ingest::Parsed p;
    std::string err;
    DMOLP_CUDA(cudaEventRecord(c->ev0, c->stream));
    if (ingest::parse(c->stream, d_txt, len, body0, body1, c->scratch, p, err)) {
        ingest::release(p);
        cudaGetLastError();
        return fail(DMOLP_ERR_ARG, err);
    }
    const auto ta = std::chrono::steady_clock::now();
    int st = graph_alloc(c, p.nv, p.narcs, p.maxdeg, p.maxraw, p.nb);
    double setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta).count();
    if (!st) {
        Buffers &b = c->b;
        int32_t *const bucket[3] = {b.bucket[0], b.bucket[1], b.bucket[2]};
        if (ingest::build(c->stream, p, b.off, b.col, b.rawdeg, bucket, err)) st = fail(DMOLP_ERR_CUDA, err);
    }
    if (!st) {
        DMOLP_CUDA(cudaEventRecord(c->ev1, c->stream));
        c->h_rawdeg.clear();  // the host mirror of the raw degrees is fetched when phase 1 first needs it
        c->h_rawdeg_valid = false;
        st = sync(c);
    }
    c->launches += p.launches;
    if (info) {
        info->num_vertices = p.nv;
        info->num_arcs = p.narcs;
        info->num_tokens = p.ntok;
        info->rows_sorted_on_device = p.rows_sorted;
        info->parse_ms = 0.0;
        float ms = 0.f;
        if (!st && cudaEventElapsedTime(&ms, c->ev0, c->ev1) == cudaSuccess) info->parse_ms = ms;
        info->kernels = p.launches;
        info->count_ms = p.count_ms;
        info->emit_ms = p.emit_ms;
    }
    ingest::release(p);
    if (st) {
        free_all(c);
        return st;
    }
    const auto tf = std::chrono::steady_clock::now();
    st = graph_finish(c, true);
    setup_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tf).count();
    if (info) info->setup_ms = setup_ms;
    return st;
}

}  // namespace

extern "C" {

const char *dmolp_last_error(void) { return g_err.c_str(); }

int dmolp_device_code_version(int device, int *version) {
    if (!version) return fail(DMOLP_ERR_ARG, "null pointer");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(DMOLP_ERR_NO_GPU, "no CUDA device");
    }
    if (device < 0 || device >= n) return fail(DMOLP_ERR_ARG, "device index out of range");
    int cur = 0;
    cudaGetDevice(&cur);
    DMOLP_CUDA(cudaSetDevice(device));
    *version = dmolp::select_binary_version();
    cudaSetDevice(cur);
    if (*version < 0) return fail(DMOLP_ERR_CUDA, "cudaFuncGetAttributes failed");
    return DMOLP_OK;
}

int dmolp_current_device(void) {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return d;
}

int dmolp_create(int device, dmolp_ctx **out) {
    if (!out) return fail(DMOLP_ERR_ARG, "out is null");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(DMOLP_ERR_NO_GPU, "no CUDA device");
    }
    if (device < 0 || device >= n) return fail(DMOLP_ERR_ARG, "device index out of range");
    DMOLP_CUDA(cudaSetDevice(device));
    dmolp_ctx *c = new dmolp_ctx();
    c->device = device;
    {  // key of the multiset symmetry sum: unknown outside the process, so no input is built to defeat it
        std::random_device rd;
        c->sym_key = ((unsigned long long)rd() << 32) ^ rd();
    }
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e != cudaSuccess) {
        delete c;
        return fail(DMOLP_ERR_CUDA, std::string("stream/event: ") + cudaGetErrorString(e));
    }
    *out = c;
    return DMOLP_OK;
}

int dmolp_destroy(dmolp_ctx *c) {
    if (!c) return DMOLP_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    free_all(c);
    if (c->arena) cudaFree(c->arena);
    c->scratch.release();
    for (int i = 0; i < kPinSlots; ++i) {
        if (c->pin[i]) cudaFreeHost(c->pin[i]);
        if (c->pin_ev[i]) cudaEventDestroy(c->pin_ev[i]);
    }
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return DMOLP_OK;
}

int dmolp_graph_upload(dmolp_ctx *c, int64_t nv, int64_t narcs, const int64_t *off, const int32_t *col,
                       const int32_t *raw) {
    if (!c) return fail(DMOLP_ERR_ARG, "null context");
    if (nv < 0 || nv > 0x7ffffffe || narcs < 0 || (!off && nv >= 0) || (!col && narcs > 0))
        return fail(DMOLP_ERR_ARG, "bad graph sizes or null arrays");
    if (off[0] != 0 || off[nv] != narcs) return fail(DMOLP_ERR_ARG, "offsets must start at 0 and end at narcs");
    DMOLP_CUDA(cudaSetDevice(c->device));
    // The arrays go as they are to device staging buffers (from pinned memory at the link's rate) and are
    // checked there: every row bound, every id, whether rows are strictly increasing, the degree classes.
    // They reach the graph only once the check passed, so a rejected upload leaves the previous graph.
    std::string err;
    int64_t *s_off = (int64_t *)c->scratch.get(ingest::kEndTok, (size_t)(nv + 1) * sizeof(int64_t), err);
    int32_t *s_col = narcs ? (int32_t *)c->scratch.get(ingest::kTok, (size_t)narcs * sizeof(int32_t), err) : nullptr;
    int32_t *s_raw = raw && nv ? (int32_t *)c->scratch.get(ingest::kBadrow, (size_t)nv * sizeof(int32_t), err) : nullptr;
    if (!s_off || (narcs && !s_col) || (raw && nv && !s_raw)) return fail(DMOLP_ERR_NOMEM, err);
    DMOLP_CUDA(cudaMemcpyAsync(s_off, off, (size_t)(nv + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
    if (s_raw) DMOLP_CUDA(cudaMemcpyAsync(s_raw, raw, (size_t)nv * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    if (narcs)
        DMOLP_CUDA(cudaMemcpyAsync(s_col, col, (size_t)narcs * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    ingest::CsrInfo ci;
    if (ingest::check_csr(c->stream, s_off, s_col, s_raw, nv, narcs, c->scratch, ci, err)) {
        cudaGetLastError();
        return fail(DMOLP_ERR_CUDA, err);
    }
    c->launches += ci.launches;
    if (ci.bad & 1) return fail(DMOLP_ERR_ARG, "offsets are not non-decreasing");
    if (ci.bad & 2) return fail(DMOLP_ERR_ARG, "a neighbour id is outside [0, nv)");
    if (ci.bad & 4) return fail(DMOLP_ERR_ARG, "negative raw degree");
    const int64_t maxraw = raw ? ci.maxraw : ci.maxdeg;
    int st = graph_alloc(c, nv, narcs, ci.maxdeg, maxraw, ci.nb);
    if (st) return st;
    Buffers &b = c->b;
    DMOLP_CUDA(cudaMemcpyAsync(b.off, s_off, (size_t)(nv + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, c->stream));
    if (narcs)
        DMOLP_CUDA(cudaMemcpyAsync(b.col, s_col, (size_t)narcs * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    // raw degrees from the caller's array, or the CSR degrees; the host mirror the phase-1 hub sort reads is
    // fetched when phase 1 first needs it
    if (s_raw) DMOLP_CUDA(cudaMemcpyAsync(b.rawdeg, s_raw, (size_t)nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    else lp_degrees(c, b.off, nv, b.rawdeg);
    c->h_rawdeg.clear();
    c->h_rawdeg_valid = false;
    int32_t *const bucket[3] = {b.bucket[0], b.bucket[1], b.bucket[2]};
    if (ingest::csr_classes(c->stream, b.off, nv, ci, bucket, err)) return fail(DMOLP_ERR_CUDA, err);
    if (nv > 0) c->launches++;
    st = graph_finish(c, ci.sorted != 0);  // ends with a stream sync: the staging copies are done
    c->scratch.trim(ingest::kKeepScratch);
    return st;
}

int dmolp_graph_upload_adjtext(dmolp_ctx *c, const char *text, int64_t len, dmolp_ingest_info *info) {
    if (!c) return fail(DMOLP_ERR_ARG, "null context");
    if (len < 0 || (!text && len > 0)) return fail(DMOLP_ERR_ARG, "bad text buffer");
    const auto t0 = std::chrono::steady_clock::now();
    const char *nl = len > 0 ? (const char *)memchr(text, '\n', (size_t)len) : nullptr;
    if (!nl) return fail(DMOLP_ERR_ARG, "missing header line");
    const int64_t body0 = (int64_t)(nl - text) + 1;
    int64_t body1 = len;  // anything after the last newline is an unterminated line: dropped
    while (body1 > body0 && text[body1 - 1] != '\n') --body1;
    DMOLP_CUDA(cudaSetDevice(c->device));
    uint8_t *d_txt = nullptr;
    int st = text_buffer(c, len, &d_txt);
    if (st) return st;
    DMOLP_CUDA(cudaEventRecord(c->ev0, c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(d_txt, text, (size_t)len, cudaMemcpyHostToDevice, c->stream));
    DMOLP_CUDA(cudaEventRecord(c->ev1, c->stream));
    DMOLP_CUDA(cudaEventSynchronize(c->ev1));
    float copy_ms = 0.f;
    cudaEventElapsedTime(&copy_ms, c->ev0, c->ev1);
    st = ingest_text(c, d_txt, len, body0, body1, info);
    c->scratch.trim(ingest::kKeepScratch);
    if (info) {
        info->read_ms = copy_ms;
        info->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return st;
}

int dmolp_graph_upload_adjtext_device(dmolp_ctx *c, const char *d_text, int64_t len, dmolp_ingest_info *info) {
    if (!c) return fail(DMOLP_ERR_ARG, "null context");
    if (len < 0 || (!d_text && len > 0)) return fail(DMOLP_ERR_ARG, "bad text buffer");
    const auto t0 = std::chrono::steady_clock::now();
    DMOLP_CUDA(cudaSetDevice(c->device));
    // the header's newline and the last newline, from pieces of the two ends of the text
    constexpr int64_t kPiece = 1 << 16;
    std::vector<char> piece((size_t)kPiece);
    int64_t body0 = -1, body1 = -1;
    for (int64_t pos = 0; pos < len && body0 < 0; pos += kPiece) {
        const int64_t n = std::min(kPiece, len - pos);
        DMOLP_CUDA(cudaMemcpy(piece.data(), d_text + pos, (size_t)n, cudaMemcpyDeviceToHost));
        const char *q = (const char *)memchr(piece.data(), '\n', (size_t)n);
        if (q) body0 = pos + (q - piece.data()) + 1;
    }
    if (body0 < 0) return fail(DMOLP_ERR_ARG, "missing header line");
    for (int64_t end = len; end > body0 && body1 < 0; end -= kPiece) {
        const int64_t a = std::max(body0, end - kPiece);
        DMOLP_CUDA(cudaMemcpy(piece.data(), d_text + a, (size_t)(end - a), cudaMemcpyDeviceToHost));
        for (int64_t j = end - a; j > 0; --j)
            if (piece[(size_t)j - 1] == '\n') {
                body1 = a + j;
                break;
            }
    }
    if (body1 < 0) body1 = body0;
    uint8_t *d_txt = nullptr;
    int st = text_buffer(c, len, &d_txt);
    if (st) return st;
    DMOLP_CUDA(cudaMemcpyAsync(d_txt, d_text, (size_t)len, cudaMemcpyDeviceToDevice, c->stream));
    const double read_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    st = ingest_text(c, d_txt, len, body0, body1, info);
    c->scratch.trim(ingest::kKeepScratch);
    if (info) {
        info->read_ms = read_ms;
        info->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return st;
}

int dmolp_graph_load_adjtext(dmolp_ctx *c, const char *path, dmolp_ingest_info *info) {
    if (!c || !path) return fail(DMOLP_ERR_ARG, "null context or path");
    const auto t0 = std::chrono::steady_clock::now();
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return fail(DMOLP_ERR_ARG, std::string("cannot open ") + path);
    struct stat sb;
    if (fstat(fd, &sb) != 0) {
        close(fd);
        return fail(DMOLP_ERR_ARG, std::string("cannot stat ") + path);
    }
    const int64_t len = (int64_t)sb.st_size;
    int st = DMOLP_OK;
    uint8_t *d_txt = nullptr;
    if (cudaSetDevice(c->device) != cudaSuccess) st = fail(DMOLP_ERR_CUDA, "cudaSetDevice failed");
    if (!st) st = text_buffer(c, len, &d_txt);
    if (!st) st = pinned_ring(c);
    // Read slot-sized pieces with all host threads into pinned memory and copy each to the device while
    // the next is read; note the first and the last newline on the way.
    int64_t body0 = -1, body1 = -1;
    for (int64_t pos = 0, i = 0; !st && pos < len; pos += kPinSlot, ++i) {
        const int s = (int)(i % kPinSlots);
        if (i >= kPinSlots && cudaEventSynchronize(c->pin_ev[s]) != cudaSuccess) {
            st = fail(DMOLP_ERR_CUDA, "pinned copy failed");
            break;
        }
        const int64_t n = std::min<int64_t>(kPinSlot, len - pos);
        char *dst = c->pin[s];
        int ok = 1;
        const int T = std::max(1, std::min(omp_get_max_threads(), 16));
#pragma omp parallel for num_threads(T) reduction(& : ok) schedule(static, 1)
        for (int t = 0; t < T; ++t) {
            int64_t a = n * t / T;
            const int64_t z = n * (t + 1) / T;
            while (a < z) {
                const ssize_t r = pread(fd, dst + a, (size_t)(z - a), (off_t)(pos + a));
                if (r <= 0) {
                    ok = 0;
                    break;
                }
                a += r;
            }
        }
        if (!ok) {
            st = fail(DMOLP_ERR_ARG, std::string("short read of ") + path);
            break;
        }
        if (body0 < 0) {
            const char *q = (const char *)memchr(dst, '\n', (size_t)n);
            if (q) body0 = pos + (q - dst) + 1;
        }
        for (int64_t j = n; j > 0; --j)
            if (dst[j - 1] == '\n') {
                body1 = pos + j;
                break;
            }
        if (cudaMemcpyAsync(d_txt + pos, dst, (size_t)n, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
            cudaEventRecord(c->pin_ev[s], c->stream) != cudaSuccess)
            st = fail(DMOLP_ERR_CUDA, "text copy failed");
    }
    close(fd);
    if (!st && cudaStreamSynchronize(c->stream) != cudaSuccess) st = fail(DMOLP_ERR_CUDA, "text copy failed");
    const double read_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (!st && body0 < 0) st = fail(DMOLP_ERR_ARG, "missing header line");
    if (!st) st = ingest_text(c, d_txt, len, body0, std::max(body0, body1), info);
    c->scratch.trim(ingest::kKeepScratch);
    if (info) {
        info->read_ms = read_ms;
        info->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return st;
}

int dmolp_graph_size(dmolp_ctx *c, int64_t *nv, int64_t *narcs) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (nv) *nv = c->nv;
    if (narcs) *narcs = c->narcs;
    return DMOLP_OK;
}

int dmolp_graph_get(dmolp_ctx *c, int64_t *offsets, int32_t *indices, int32_t *raw_degree) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    DMOLP_CUDA(cudaSetDevice(c->device));
    if (offsets)
        DMOLP_CUDA(cudaMemcpyAsync(offsets, c->b.off, (size_t)(c->nv + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                   c->stream));
    if (indices && c->narcs)
        DMOLP_CUDA(cudaMemcpyAsync(indices, c->b.col, (size_t)c->narcs * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                   c->stream));
    if (raw_degree && c->nv)
        DMOLP_CUDA(cudaMemcpyAsync(raw_degree, c->b.rawdeg, (size_t)c->nv * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                   c->stream));
    return sync(c);
}

int dmolp_labels_get(dmolp_ctx *c, int32_t *labels) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (!labels && c->nv) return fail(DMOLP_ERR_ARG, "null labels");
    DMOLP_CUDA(cudaSetDevice(c->device));
    DMOLP_CUDA(cudaMemcpyAsync(labels, c->b.label, (size_t)c->nv * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    return sync(c);
}

int dmolp_labels_set(dmolp_ctx *c, const int32_t *labels) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (!labels && c->nv) return fail(DMOLP_ERR_ARG, "null labels");
    DMOLP_CUDA(cudaSetDevice(c->device));
    DMOLP_CUDA(cudaMemcpyAsync(c->b.label, labels, (size_t)c->nv * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    return sync(c);
}

int dmolp_device_labels(dmolp_ctx *c, int32_t **labels_device) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    *labels_device = c->b.label;
    return DMOLP_OK;
}

int64_t dmolp_kernel_launches(const dmolp_ctx *c) { return c ? c->launches : 0; }

void *dmolp_stream(dmolp_ctx *c) { return c ? (void *)c->stream : nullptr; }

int dmolp_labels_save(dmolp_ctx *c) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    DMOLP_CUDA(cudaSetDevice(c->device));
    if (!c->saved_labels) {
        int st = dalloc(c, &c->saved_labels, (size_t)c->nv + 1);
        if (st) return st;
    }
    DMOLP_CUDA(cudaMemcpyAsync(c->saved_labels, c->b.label, (size_t)c->nv * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                               c->stream));
    return DMOLP_OK;
}

int dmolp_labels_restore(dmolp_ctx *c) {
    if (!c || !c->has_graph || !c->saved_labels) return fail(DMOLP_ERR_STATE, "no saved labels");
    DMOLP_CUDA(cudaSetDevice(c->device));
    DMOLP_CUDA(cudaMemcpyAsync(c->b.label, c->saved_labels, (size_t)c->nv * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                               c->stream));
    return DMOLP_OK;
}

int dmolp_set_wait_limit(dmolp_ctx *c, uint32_t polls) {
    if (!c) return fail(DMOLP_ERR_ARG, "null context");
    const unsigned int v = polls ? polls : kDefaultWaitPolls;
    if (v != c->wait_polls) {
        drop_graphs(c);  // captured launches carry the limit as an argument
        c->wait_polls = v;
    }
    return DMOLP_OK;
}

int dmolp_graph_symmetric(dmolp_ctx *c, int *symmetric) {
    if (!c || !symmetric) return fail(DMOLP_ERR_ARG, "null argument");
    if (!c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    DMOLP_CUDA(cudaSetDevice(c->device));
    const int st = ensure_symmetry(c);
    if (st) return st;
    *symmetric = c->symmetric ? 1 : 0;
    return DMOLP_OK;
}

int dmolp_set_symmetry_test(dmolp_ctx *c, int exact) {
    if (!c) return fail(DMOLP_ERR_ARG, "null context");
    if ((exact != 0) != c->symmetry_exact) {
        c->symmetry_exact = exact != 0;
        c->symmetry_known = false;  // the resident graph is tested again, the chosen way, when next needed
        drop_graphs(c);
    }
    return DMOLP_OK;
}

int dmolp_set_profiling(dmolp_ctx *c, int enable) {
    if (!c) return fail(DMOLP_ERR_ARG, "null context");
    c->profiling = enable != 0;
    for (int i = 0; i < 5; ++i) {
        c->prof_ms[i] = 0;
        c->prof_launches[i] = 0;
        c->prof_bytes[i] = 0;
    }
    return DMOLP_OK;
}

int dmolp_kernel_profile(dmolp_ctx *c, int kernel, double *total_ms, int64_t *launches, double *bytes) {
    if (!c || kernel < 0 || kernel > 4) return fail(DMOLP_ERR_ARG, "bad context or kernel id");
    if (total_ms) *total_ms = c->prof_ms[kernel];
    if (launches) *launches = c->prof_launches[kernel];
    if (bytes) *bytes = c->prof_bytes[kernel];
    return DMOLP_OK;
}

int dmolp_metrics(dmolp_ctx *c, int k, int64_t *edge_cut, int64_t *vertex_counts, int64_t *edge_counts) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (k < 1 || k > DMOLP_MAX_K) return fail(DMOLP_ERR_ARG, "k out of range");
    DMOLP_CUDA(cudaSetDevice(c->device));
    unsigned long long arcs = 0;
    std::vector<long long> vc, intra;
    int bad = 0;
    int st = run_stats(c, k, &arcs, vc, intra, &bad);
    if (st) return st;
    if (edge_cut) *edge_cut = (int64_t)(arcs >> 1);
    for (int p = 0; p < k; ++p) {
        if (vertex_counts) vertex_counts[p] = vc[p];
        if (edge_counts) edge_counts[p] = intra[p] / 2;
    }
    if (bad || (arcs & 1ull)) return fail(DMOLP_ERR_BAD_LABELS, "label outside [0,k) or odd cut-arc count");
    return DMOLP_OK;
}

// Seeds by the reference rule (seed.cpp:138-242) from a given hub list and first seed; no completion.
static int find_seeds_impl(dmolp_ctx *c, int k, int first, const std::vector<int> &hubs, std::vector<int> &seeds) {
    Buffers &b = c->b;
    const int64_t nv = c->nv;
    seeds.clear();
    if (nv <= 0) return DMOLP_OK;
    seeds.push_back(first);
    if (hubs.empty() || k <= 1) return DMOLP_OK;
    DMOLP_CUDA(cudaMemcpyAsync(b.hubs, hubs.data(), hubs.size() * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.hub_used, 0, hubs.size(), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.covered, 0, (size_t)nv, c->stream));
    auto fi = std::find(hubs.begin(), hubs.end(), first);
    if (fi != hubs.end()) DMOLP_CUDA(cudaMemsetAsync(b.hub_used + (fi - hubs.begin()), 1, 1, c->stream));
    size_t balls = 0;
    for (int p = 1; p < k; ++p) {  // seed.cpp:206-226
        for (; balls < seeds.size(); ++balls) p1_mark_ball(c, seeds[balls]);
        p1_hub_argmax(c, (int64_t)hubs.size());
        unsigned long long best = 0;
        DMOLP_CUDA(cudaMemcpyAsync(&best, b.best, sizeof(best), cudaMemcpyDeviceToHost, c->stream));
        int st = sync(c);
        if (st) return st;
        if (best == 0) break;
        const int64_t idx = (int64_t)(0xffffffffu - (unsigned)(best & 0xffffffffull));
        seeds.push_back(hubs[idx]);
        DMOLP_CUDA(cudaMemsetAsync(b.hub_used + idx, 1, 1, c->stream));
    }
    return DMOLP_OK;
}

// Seed completion: where the reference rule found fewer than k seeds the reference reads past its seed
// vector (partition.cpp:347).  Remaining seeds: unused hubs by raw degree (first in hub order on ties),
// then other vertices by raw degree (lowest id on ties).
static void complete_seeds(dmolp_ctx *c, int k, const std::vector<int> &hubs, std::vector<int> &seeds) {
    const int64_t nv = c->nv;
    if ((int64_t)seeds.size() >= k || nv <= 0) return;
    std::vector<char> used(hubs.size(), 0), is_seed(nv, 0);
    for (int s : seeds) {
        is_seed[s] = 1;
        auto it = std::find(hubs.begin(), hubs.end(), s);
        if (it != hubs.end()) used[it - hubs.begin()] = 1;
    }
    while ((int)seeds.size() < k) {
        int bestv = -1, bd = -1;
        int64_t bi = -1;
        for (size_t i = 0; i < hubs.size(); ++i)
            if (!used[i] && c->h_rawdeg[hubs[i]] > bd) {
                bd = c->h_rawdeg[hubs[i]];
                bestv = hubs[i];
                bi = (int64_t)i;
            }
        if (bestv == -1)
            for (int64_t v = 0; v < nv; ++v)
                if (!is_seed[v] && c->h_rawdeg[v] > bd) {
                    bd = c->h_rawdeg[v];
                    bestv = (int)v;
                }
        if (bestv == -1) break;
        seeds.push_back(bestv);
        is_seed[bestv] = 1;
        if (bi >= 0) used[bi] = 1;
        else {
            auto it = std::find(hubs.begin(), hubs.end(), bestv);
            if (it != hubs.end()) used[it - hubs.begin()] = 1;
        }
    }
}

// Growth rounds (partition.cpp:335-604); seedk[p] = -1 for a part without a seed.
static int expand_impl(dmolp_ctx *c, int k, int theta, const std::vector<int32_t> &seedk, int *rounds_out) {
    Buffers &b = c->b;
    const int64_t nv = c->nv;
    p1_init_labels(c);
    DMOLP_CUDA(cudaMemsetAsync(b.psize, 0, DMOLP_MAX_K * sizeof(long long), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.npart, 0, DMOLP_MAX_K * sizeof(int32_t), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.p1cnt, 0, 8 * sizeof(int), c->stream));
    // the seeds go through the need[] buffer as staging (k ints)
    DMOLP_CUDA(cudaMemcpyAsync(b.need, seedk.data(), k * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    p1_set_seeds(c, b.need, k);
    int cur = 0, rounds = 0;
    std::vector<long long> psize(k);
    while (nv > 0) {
        int cnt[8];
        DMOLP_CUDA(cudaMemcpyAsync(cnt, b.p1cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
        DMOLP_CUDA(cudaMemcpyAsync(psize.data(), b.psize, k * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
        int st = sync(c);
        if (st) return st;
        if (cnt[3] >= nv) break;
        if (cnt[0] == 0) {  // every frontier empty: all unlabelled vertices go to the smallest part
            int best = 0;
            for (int p = 1; p < k; ++p)
                if (psize[p] < psize[best]) best = p;
            p1_fallback(c, best, cur);
        }
        p1_round(c, k, theta, cur);
        cur ^= 1;
        ++rounds;
    }
    *rounds_out = rounds;
    return DMOLP_OK;
}

static int check_seed_args(dmolp_ctx *c, int k) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (k < 1 || k > DMOLP_MAX_K) return fail(DMOLP_ERR_ARG, "k out of range [1, 1024]");
    return DMOLP_OK;
}

int dmolp_find_seeds(dmolp_ctx *c, int k, int32_t first_seed, const int32_t *hubs, int64_t nhubs, int32_t *seeds_out,
                     int32_t *nseeds) {
    int st = check_seed_args(c, k);
    if (st) return st;
    if (nhubs < 0 || (nhubs && !hubs) || !seeds_out || !nseeds) return fail(DMOLP_ERR_ARG, "bad arguments");
    if (c->nv > 0 && (first_seed < 0 || first_seed >= c->nv)) return fail(DMOLP_ERR_ARG, "first seed out of range");
    for (int64_t i = 0; i < nhubs; ++i)
        if (hubs[i] < 0 || hubs[i] >= c->nv) return fail(DMOLP_ERR_ARG, "hub id out of range");
    DMOLP_CUDA(cudaSetDevice(c->device));
    DMOLP_CUDA(cudaMemsetAsync(c->b.p1te, 0, sizeof(unsigned long long), c->stream));
    std::vector<int> hv(hubs, hubs + nhubs), seeds;
    st = find_seeds_impl(c, k, first_seed, hv, seeds);
    if (st) return st;
    for (size_t i = 0; i < seeds.size(); ++i) seeds_out[i] = seeds[i];
    *nseeds = (int32_t)seeds.size();
    return DMOLP_OK;
}

int dmolp_expand_partitions(dmolp_ctx *c, int k, int theta, const int32_t *seeds, int32_t nseeds, int32_t *rounds) {
    int st = check_seed_args(c, k);
    if (st) return st;
    if (theta < 1) return fail(DMOLP_ERR_ARG, "theta must be >= 1 (with theta = 0 the reference never ends)");
    if (nseeds < 0 || (nseeds && !seeds)) return fail(DMOLP_ERR_ARG, "bad seeds");
    std::vector<int32_t> seedk(k, -1);
    std::vector<char> seen(c->nv, 0);
    for (int p = 0; p < k && p < nseeds; ++p) {
        if (seeds[p] < 0 || seeds[p] >= c->nv) return fail(DMOLP_ERR_ARG, "seed out of range");
        if (seen[seeds[p]]) return fail(DMOLP_ERR_ARG, "a vertex is the seed of two parts");
        seen[seeds[p]] = 1;
        seedk[p] = seeds[p];
    }
    DMOLP_CUDA(cudaSetDevice(c->device));
    int r = 0;
    st = expand_impl(c, k, theta, seedk, &r);
    if (rounds) *rounds = r;
    return st ? st : check_waits(c);
}

int dmolp_phase1(dmolp_ctx *c, int k, int theta, int32_t *seeds_out, int64_t *vertex_counts, int64_t *edge_counts,
                 dmolp_phase1_info *info) {
    int st = check_seed_args(c, k);
    if (st) return st;
    if (theta < 1)
        return fail(DMOLP_ERR_ARG, "theta must be >= 1 (with theta = 0 the reference expands nothing and never ends)");
    DMOLP_CUDA(cudaSetDevice(c->device));
    Buffers &b = c->b;
    const int64_t nv = c->nv;
    if (!c->h_rawdeg_valid) {  // a device-parsed graph: fetch the raw degrees once
        c->h_rawdeg.resize(nv);
        if (nv)
            DMOLP_CUDA(cudaMemcpyAsync(c->h_rawdeg.data(), b.rawdeg, (size_t)nv * sizeof(int32_t),
                                       cudaMemcpyDeviceToHost, c->stream));
        int s0 = sync(c);
        if (s0) return s0;
        c->h_rawdeg_valid = true;
    }
    dmolp_phase1_info inf;
    std::memset(&inf, 0, sizeof(inf));
    DMOLP_CUDA(cudaEventRecord(c->ev0, c->stream));

    // ---- hubs and first seed on the host (order-dependent; see the top of this file) ----
    const auto th0 = std::chrono::steady_clock::now();
    std::vector<int> hubs = find_hubs(c->h_rawdeg);
    // init.cpp:179-187, including its id-vs-degree tie test
    const std::pair<int, int> first = dmolp::first_seed_of(c->h_rawdeg.data(), nv);
    inf.num_hubs = (int64_t)hubs.size();
    DMOLP_CUDA(cudaMemsetAsync(b.p1te, 0, sizeof(unsigned long long), c->stream));
    const auto th1 = std::chrono::steady_clock::now();
    inf.hubs_ms = std::chrono::duration<double, std::milli>(th1 - th0).count();
    std::vector<int> seeds;
    st = find_seeds_impl(c, k, first.first, hubs, seeds);
    if (st) return st;
    inf.num_seeds_found = (int32_t)seeds.size();
    complete_seeds(c, k, hubs, seeds);
    const auto th2 = std::chrono::steady_clock::now();
    inf.seeds_ms = std::chrono::duration<double, std::milli>(th2 - th1).count();
    std::vector<int32_t> seedk(k, -1);
    for (int p = 0; p < k && p < (int)seeds.size(); ++p) seedk[p] = seeds[p];
    if (seeds_out) std::copy(seedk.begin(), seedk.end(), seeds_out);
    int rounds = 0;
    st = expand_impl(c, k, theta, seedk, &rounds);
    if (st) return st;
    inf.rounds = rounds;

    // ---- initial metrics (phase1.cpp:83-153) ----
    unsigned long long arcs = 0;
    std::vector<long long> vc, intra;
    int bad = 0;
    st = run_stats(c, k, &arcs, vc, intra, &bad);
    if (st) return st;
    DMOLP_CUDA(cudaEventRecord(c->ev1, c->stream));
    unsigned long long te = 0;
    DMOLP_CUDA(cudaMemcpyAsync(&te, b.p1te, sizeof(te), cudaMemcpyDeviceToHost, c->stream));
    st = sync(c);
    if (st) return st;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    inf.gpu_ms = ms;
    inf.expand_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - th2).count();
    inf.traversed_edges = te;
    inf.initial_edge_cut = (int64_t)(arcs / 2);
    const double ev = (double)nv / k;
    double mv = 0;
    for (int p = 0; p < k; ++p) mv = std::max(mv, vc[p] / ev);
    double tot = 0;
    std::vector<long long> ec(k);
    for (int p = 0; p < k; ++p) {
        ec[p] = intra[p] / 2;
        tot += (double)ec[p];
    }
    const double ee = tot / k;
    double me = 0;
    for (int p = 0; p < k; ++p) me = std::max(me, ec[p] / ee);
    inf.initial_vertex_balance = mv;
    inf.initial_edge_balance = me;
    for (int p = 0; p < k; ++p) {
        if (vertex_counts) vertex_counts[p] = vc[p];
        if (edge_counts) edge_counts[p] = ec[p];
    }
    if (info) *info = inf;
    if (bad) return fail(DMOLP_ERR_BAD_LABELS, "phase 1 left a label outside [0,k)");
    return check_waits(c);
}

int dmolp_lp_run(dmolp_ctx *c, int k, const dmolp_lp_config *cfg, dmolp_lp_result *res, dmolp_lp_record *records,
                 int max_records) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (k < 1 || k > DMOLP_MAX_K) return fail(DMOLP_ERR_ARG, "k out of range [1, 1024]");
    if (!cfg) return fail(DMOLP_ERR_ARG, "null config");
    if (cfg->mode != DMOLP_LP_MODE_REF && cfg->mode != DMOLP_LP_MODE_FIXED) return fail(DMOLP_ERR_ARG, "bad mode");
    if (cfg->mode == DMOLP_LP_MODE_FIXED && (cfg->iterations < 0 || cfg->iterations > kMaxIter))
        return fail(DMOLP_ERR_ARG, "iterations must be in [0, 500]");
    if (cfg->cap != DMOLP_LP_CAP_REF && cfg->cap != DMOLP_LP_CAP_FULL) return fail(DMOLP_ERR_ARG, "bad cap");
    DMOLP_CUDA(cudaSetDevice(c->device));
    int st = ensure_symmetry(c);
    if (st) return st;
    Buffers &b = c->b;
    LpLaunch L;
    L.k = k;
    L.eff = cfg->cap == DMOLP_LP_CAP_FULL ? k : std::min(k, 32);
    L.mode = cfg->mode;
    const int max_iter = cfg->mode == DMOLP_LP_MODE_REF ? kMaxIter : cfg->iterations;

    DMOLP_CUDA(cudaEventRecord(c->ev0, c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.stamp, 0, (size_t)(c->nv + 1) * sizeof(int32_t), c->stream));
    DMOLP_CUDA(cudaMemsetAsync(b.sstamp, 0, (size_t)(c->nv + 1) * sizeof(int32_t), c->stream));
    st = clear_select_bins(c);
    if (st) return st;
    DMOLP_CUDA(cudaMemsetAsync(b.ndiff, 0, (size_t)(c->nv + 1) * sizeof(int32_t), c->stream));
    if (c->nb[2] > 0) {
        DMOLP_CUDA(cudaMemsetAsync(b.hubwin, 0, (size_t)(c->nv + 1) * sizeof(int32_t), c->stream));
        DMOLP_CUDA(cudaMemsetAsync(b.hub_in, 0, (size_t)c->nb[2] * sizeof(int32_t), c->stream));
    }
    // symmetric graphs with at most 32 scored labels decide from kept label counts (no label gathers)
    c->counts_kept = c->symmetric && L.eff <= 32;
    // The hot set (the labels of the highest-degree vertices in shared memory, a full pass over the arcs to
    // build) pays off when the decisions gather labels, or over several runs on the graph; the first run of
    // a kept-count graph goes without it.
    if (!c->counts_kept || c->lp_runs > 0) {
        st = lp_hot_prepare(c);
        if (st) return st;
    }
    ++c->lp_runs;
    lp_hot_refresh(c);
    lp_reset_stats(c, k, nullptr);
    // the run-start pass also counts every hub's row into hh on symmetric graphs (kept from the movers after)
    lp_stats(c, k, nullptr, nullptr, true, c->counts_kept ? L.eff : 0, c->symmetric ? L.eff : 0);
    lp_init_end(c, cfg->mode);
    st = check_launch(c);
    if (st) return st;
    int stopped = 0;
    // Iterations in blocks: FIXED mode one block of all iterations, REF mode blocks of 8 with a check of
    // the stop flag in between.  Each block is captured into a CUDA graph once and replayed afterwards.
    const int block = cfg->mode == DMOLP_LP_MODE_REF ? 8 : std::max(1, max_iter);
    for (int t0 = 1; t0 <= max_iter; t0 += block) {
        const int cnt = std::min(block, max_iter - t0 + 1);
        if (c->use_graphs) {
            st = run_block_graph(c, L, t0, cnt);
            if (st) return st;
        } else {
            for (int t = t0; t < t0 + cnt; ++t) lp_iteration(c, L, t, t == t0, t == t0 + cnt - 1);
        }
        if (cfg->mode == DMOLP_LP_MODE_REF && t0 + cnt <= max_iter) {
            DMOLP_CUDA(cudaMemcpyAsync(&stopped, &b.ctrl->stopped, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
            st = sync(c);
            if (st) return st;
            if (stopped) break;
        }
    }
    DMOLP_CUDA(cudaEventRecord(c->ev1, c->stream));
    LpControl ctl;
    DMOLP_CUDA(cudaMemcpyAsync(&ctl, b.ctrl, sizeof(ctl), cudaMemcpyDeviceToHost, c->stream));
    std::vector<unsigned long long> hv(k), hi(k);
    DMOLP_CUDA(cudaMemcpyAsync(hv.data(), b.vc, k * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(hi.data(), b.intra, k * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    std::vector<LpRecordDev> recs(kMaxIter);
    DMOLP_CUDA(cudaMemcpyAsync(recs.data(), b.rec, kMaxIter * sizeof(LpRecordDev), cudaMemcpyDeviceToHost, c->stream));
    st = sync(c);
    if (st) return st;
    if (ctl.wait_timeout || c->launch_error != cudaSuccess) return check_waits(c);
    if (ctl.error) return fail(DMOLP_ERR_BAD_LABELS, "label outside [0,k) or odd cut-arc count");
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    std::vector<long long> vc(k), ec(k);
    for (int p = 0; p < k; ++p) {
        vc[p] = (long long)hv[p];
        ec[p] = (long long)(hi[p] / 2);
    }
    if (c->profiling) {
        // Algorithmic bytes per launch of the design (ids and labels are 4 B, offsets 8 B):
        //  bnd    : per record slot (every vertex with arcs) its id, own label, boundary count and the record
        //           label written, from iteration 2 also its stamp (push) or window stamp (pull) and, on
        //           graphs with hubs, its hub-window count; offsets per candidate; the key written per
        //           boundary record; id + window stamp per arc of a pull-mode walk
        //  decide : list id + offsets + own label per selected vertex, id + label per arc, 8 B per mover;
        //           with kept counts 64 B of counts per selected vertex and no arcs
        //  mark   : list id + offsets per window vertex, id read + stamp write per arc of a walked row
        //           (window rows up to 4096 arcs; hub rows only when the hub enters or leaves the window)
        //  update : offsets + labels per mover, id + label + pending label + hub index per arc (+ 8 B of
        //           count updates per arc with kept counts)
        //  select : label + key of every record slot (one pass), and per selected vertex its stamp, window
        //           entry and decision-class entry
        const double nbk = (double)c->nb[0] + c->nb[1] + c->nb[2];
        dmolp_ctx::ProfEvents &pe = c->prof_pending;
        for (size_t i = 0; i < pe.kind.size(); ++i) {
            const int t = pe.iter[i], kind = pe.kind[i];
            float ems = 0;
            if (t <= ctl.iters_run && cudaEventElapsedTime(&ems, pe.ev[2 * i], pe.ev[2 * i + 1]) == cudaSuccess) {
                const LpRecordDev &d = recs[t - 1];
                const double ncand = t == 1 ? nbk : (double)d.candidates;
                double bytes = 0;
                if (kind == 0)
                    bytes = (16.0 + (t > 1 ? 4.0 : 0.0) + (t > 1 && c->nb[2] > 0 ? 4.0 : 0.0)) * nbk + 16.0 * ncand +
                            8.0 * d.boundary + 8.0 * (double)d.arcs_bnd;
                else if (kind == 1)
                    bytes = (c->counts_kept ? 88.0 : 24.0) * d.window + 8.0 * (double)d.arcs_dec + 8.0 * d.changes;
                else if (kind == 2) bytes = (t > 1 ? 20.0 * recs[t - 2].window : 0.0) + 8.0 * (double)d.arcs_mark;
                else if (kind == 3) bytes = 28.0 * d.changes + (c->counts_kept ? 24.0 : 16.0) * (double)d.arcs_upd;
            else bytes = 12.0 * nbk + 12.0 * (double)d.window;  // select
                c->prof_ms[kind] += ems;
                c->prof_launches[kind] += 1;
                c->prof_bytes[kind] += bytes;
            }
            cudaGetLastError();
            if (c->prof_owned[i]) {
                cudaEventDestroy(pe.ev[2 * i]);
                cudaEventDestroy(pe.ev[2 * i + 1]);
            }
        }
        c->prof_pending = dmolp_ctx::ProfEvents();
        c->prof_owned.clear();
    }
    dmolp_lp_result r;
    std::memset(&r, 0, sizeof(r));
    r.edge_cut = ctl.prev_cut;
    r.iterations_run = ctl.iters_run;
    r.stop_reason = ctl.stop_reason;
    balances(vc, ec, k, &r.vertex_balance, &r.edge_balance, &r.total_vertices, &r.total_edges);
    r.gpu_ms = ms;
    for (int i = 0; i < ctl.iters_run; ++i) {
        const LpRecordDev &d = recs[i];
        r.traversed_edges += d.te_prev + d.te_cand + d.te_sel + d.te_stats;
        if (records && i < max_records) {
            dmolp_lp_record &o = records[i];
            o.iteration = d.iteration;
            o.window = d.window;
            o.candidates = d.candidates < 0 ? (int32_t)c->nv : d.candidates;
            o.changes = d.changes;
            o.boundary = d.boundary;
            o.reserved = 0;
            o.arcs_read = d.arcs_bnd + d.arcs_dec + d.arcs_upd + d.arcs_mark;
            o.edge_cut = d.edge_cut;
            o.te_prev = d.te_prev;
            o.te_cand = d.te_cand;
            o.te_sel = d.te_sel;
            o.te_stats = d.te_stats;
            o.window_sum = d.win_sum;
        }
    }
    if (res) *res = r;
    return DMOLP_OK;
}

// Per-iteration history of the last dmolp_lp_run: penalties[iters][k] and counts[iters][2k] (vertex counts,
// then intra-part edge counts).  Not part of the reference interface; used by the parity tests.
int dmolp_lp_history(dmolp_ctx *c, int k, int iters, double *penalties, int64_t *counts) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (k < 1 || k > DMOLP_MAX_K || iters < 0 || iters > kMaxIter) return fail(DMOLP_ERR_ARG, "bad k/iters");
    DMOLP_CUDA(cudaSetDevice(c->device));
    std::vector<double> ph((size_t)iters * DMOLP_MAX_K);
    std::vector<long long> ch((size_t)iters * 2 * DMOLP_MAX_K);
    if (iters) {
        DMOLP_CUDA(cudaMemcpyAsync(ph.data(), c->b.penhist, ph.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream));
        DMOLP_CUDA(cudaMemcpyAsync(ch.data(), c->b.cnthist, ch.size() * sizeof(long long), cudaMemcpyDeviceToHost,
                                   c->stream));
    }
    int st = sync(c);
    if (st) return st;
    for (int t = 0; t < iters; ++t)
        for (int p = 0; p < k; ++p) {
            if (penalties) penalties[(size_t)t * k + p] = ph[(size_t)t * DMOLP_MAX_K + p];
            if (counts) {
                counts[(size_t)t * 2 * k + p] = ch[(size_t)t * 2 * DMOLP_MAX_K + p];
                counts[(size_t)t * 2 * k + k + p] = ch[(size_t)t * 2 * DMOLP_MAX_K + DMOLP_MAX_K + p];
            }
        }
    return DMOLP_OK;
}

int dmolp_window_select(dmolp_ctx *c, int k, int iteration, const double *RE, const int32_t *prev, int64_t nprev,
                        int32_t *out, int64_t *nout) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (k < 1 || k > DMOLP_MAX_K || iteration < 1 || iteration > kMaxIter || !RE || !out || !nout || nprev < 0 ||
        (nprev && !prev))
        return fail(DMOLP_ERR_ARG, "bad arguments");
    // keep only in-range previous vertices, deduplicated (gpu_lp_boundary.cu:210 skips the others)
    std::vector<int32_t> pv;
    pv.reserve(nprev);
    for (int64_t i = 0; i < nprev; ++i)
        if (prev[i] >= 0 && prev[i] < c->nv) pv.push_back(prev[i]);
    std::sort(pv.begin(), pv.end());
    pv.erase(std::unique(pv.begin(), pv.end()), pv.end());
    DMOLP_CUDA(cudaSetDevice(c->device));
    {  // the selection indexes per-label arrays by label: check every label is in [0,k) first
        unsigned long long arcs = 0;
        std::vector<long long> vc, intra;
        int bad = 0;
        int st0 = run_stats(c, k, &arcs, vc, intra, &bad);
        if (st0) return st0;
        if (bad) return fail(DMOLP_ERR_BAD_LABELS, "label outside [0,k)");
    }
    const int t = iteration;
    Buffers &b = c->b;
    DMOLP_CUDA(cudaMemsetAsync(b.stamp, 0, (size_t)(c->nv + 1) * sizeof(int32_t), c->stream));
    {
        const int st0 = clear_select_bins(c);
        if (st0) return st0;
    }
    if (!pv.empty())
        DMOLP_CUDA(cudaMemcpyAsync(b.win[(t - 1) & 1], pv.data(), pv.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                   c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(b.RE, RE, k * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    lp_window_from_list(c, k, t, b.RE, (int)pv.size());
    LpCounters cn;
    DMOLP_CUDA(cudaMemcpyAsync(&cn, b.cnt, sizeof(cn), cudaMemcpyDeviceToHost, c->stream));
    int st = sync(c);
    if (st) return st;
    const int n = cn.nwin[t & 1];
    if (n)
        DMOLP_CUDA(cudaMemcpyAsync(out, b.win[t & 1], (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    st = sync(c);
    if (st) return st;
    std::sort(out, out + n);
    *nout = n;
    return check_waits(c);
}

int dmolp_lp_apply(dmolp_ctx *c, int k, int cap, const double *penalty, const int32_t *window, int64_t nwindow,
                   int32_t *changed_nodes, int32_t *changed_labels, int64_t *nchanged) {
    if (!c || !c->has_graph) return fail(DMOLP_ERR_STATE, "no graph uploaded");
    if (k < 1 || k > DMOLP_MAX_K || !penalty || nwindow < 0 || (nwindow && !window) || !nchanged)
        return fail(DMOLP_ERR_ARG, "bad arguments");
    if (cap != DMOLP_LP_CAP_REF && cap != DMOLP_LP_CAP_FULL) return fail(DMOLP_ERR_ARG, "bad cap");
    std::vector<int32_t> w;
    w.reserve(nwindow);
    for (int64_t i = 0; i < nwindow; ++i)
        if (window[i] >= 0 && window[i] < c->nv) w.push_back(window[i]);
    std::sort(w.begin(), w.end());
    w.erase(std::unique(w.begin(), w.end()), w.end());
    std::vector<double> tp(k);
    for (int p = 0; p < k; ++p) tp[p] = 1.0 + penalty[p];
    DMOLP_CUDA(cudaSetDevice(c->device));
    Buffers &b = c->b;
    const int n = (int)w.size();
    if (n) DMOLP_CUDA(cudaMemcpyAsync(b.cand, w.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    DMOLP_CUDA(cudaMemcpyAsync(b.tpen, tp.data(), k * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const int eff = cap == DMOLP_LP_CAP_FULL ? k : std::min(k, 32);
    lp_apply_list(c, k, eff, n);
    LpCounters cn;
    DMOLP_CUDA(cudaMemcpyAsync(&cn, b.cnt, sizeof(cn), cudaMemcpyDeviceToHost, c->stream));
    int st = sync(c);
    if (st) return st;
    const int m = cn.nchanged;
    std::vector<int32_t> mv(m), ml(m);
    if (m) {
        DMOLP_CUDA(cudaMemcpyAsync(mv.data(), b.bv, m * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        DMOLP_CUDA(cudaMemcpyAsync(ml.data(), b.bnew, m * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    }
    st = sync(c);
    if (st) return st;
    for (int i = 0; i < m; ++i) {
        if (changed_nodes) changed_nodes[i] = mv[i];
        if (changed_labels) changed_labels[i] = ml[i];
    }
    *nchanged = m;
    return DMOLP_OK;
}

}  // extern "C"
