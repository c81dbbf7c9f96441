// C-ABI of the learned initial-partition proposal (include/dmolp_b200.h, dmolp_mpnn_* and
// dmolp_batch_propose): the network's parameters and Adam state, its per-batch workspace, features,
// forward, backward, one training step and the decoder into a batch's labels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/dmolp_b200.h"
#include "mpnn.cuh"

namespace dmolp {
void set_last_error(const std::string &msg);  // dmolp_cabi.cu
}

using namespace dmolp;
using namespace dmolp::mpnn;

namespace {

// Offsets of each layer's weights and biases in the flat parameter vector.
constexpr int kOffW[3] = {0, 2 * kIn * kHidden + kHidden, 2 * kIn * kHidden + kHidden + 2 * kHidden * kHidden + kHidden};
constexpr int kOffB[3] = {kOffW[0] + 2 * kIn * kHidden, kOffW[1] + 2 * kHidden * kHidden, kOffW[2] + 2 * kHidden * kOut};
static_assert(kOffB[2] + kOut == kNumParams, "parameter layout");

int fail(int code, const std::string &msg) {
    set_last_error(msg);
    return code;
}

#define MCUDA(call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(e_ == cudaErrorMemoryAllocation ? DMOLP_ERR_NOMEM : DMOLP_ERR_CUDA,           \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

#define MTRY(x)             \
    do {                    \
        int r_ = (x);       \
        if (r_) return r_;  \
    } while (0)

}  // namespace

struct dmolp_mpnn {
    int device = 0, num_sms = 148;
    float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *W[3] = {}, *Wt[3] = {};
    int *err = nullptr;
    uint32_t wait_polls = 1u << 24;  // GEMM completion-barrier polls before it gives up (dmolp_mpnn_set_wait_limit)
    double *loss = nullptr;
    int step = 0;
    std::vector<void *> fixed;
    // per-batch workspace
    int64_t cap_nv = -1;
    int cap_inst = -1;
    bool cap_train = false;
    std::vector<void *> ws;
    __nv_bfloat16 *C1 = nullptr, *C2 = nullptr, *C3 = nullptr, *G = nullptr, *G3 = nullptr;
    float *Z3 = nullptr, *dC = nullptr, *Xf = nullptr, *Pc = nullptr, *Y = nullptr;
    int32_t *vinst = nullptr, *dist = nullptr, *mind = nullptr, *f0 = nullptr, *f1 = nullptr, *cnt = nullptr;
    unsigned long long *akey = nullptr;
    int32_t *anchor = nullptr, *ecc = nullptr, *status = nullptr, *target = nullptr, *dl0 = nullptr, *dl1 = nullptr;
    uint8_t *skip = nullptr;  // [ninst] graphs the decoder leaves to phase 1
    int *next = nullptr;
    float *P0 = nullptr, *Q0 = nullptr, *P1 = nullptr, *Q1 = nullptr;
    double *stats = nullptr, *gscore = nullptr;
    float *ggrad = nullptr;
    bool have_z = false;
};

namespace {

template <typename T>
int alloc_into(std::vector<void *> &owner, T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DMOLP_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    owner.push_back(q);
    *p = (T *)q;
    return DMOLP_OK;
}

void free_ws(dmolp_mpnn *m) {
    for (void *p : m->ws) cudaFree(p);
    m->ws.clear();
    m->cap_nv = -1;
    m->cap_inst = -1;
    m->have_z = false;
}

// Workspace for a batch of nv vertices and ninst graphs (reallocated only when it must grow).
int ensure_ws(dmolp_mpnn *m, const batch::View &b, bool train) {
    if (b.nv <= m->cap_nv && b.ninst <= m->cap_inst && (!train || m->cap_train)) return DMOLP_OK;
    cudaStreamSynchronize(b.stream);
    free_ws(m);
    const size_t n = (size_t)b.nv;
    auto &o = m->ws;
    MTRY(alloc_into(o, &m->C1, n * 32));
    MTRY(alloc_into(o, &m->C2, n * 128));
    MTRY(alloc_into(o, &m->C3, n * 128));
    MTRY(alloc_into(o, &m->Z3, n * 16));
    MTRY(alloc_into(o, &m->Xf, n * 16));
    MTRY(alloc_into(o, &m->Pc, n * 16));
    MTRY(alloc_into(o, &m->Y, n * 4));
    MTRY(alloc_into(o, &m->G3, n * 16));
    MTRY(alloc_into(o, &m->vinst, n));
    MTRY(alloc_into(o, &m->dist, n));
    MTRY(alloc_into(o, &m->mind, n));
    MTRY(alloc_into(o, &m->f0, n));
    MTRY(alloc_into(o, &m->f1, n));
    MTRY(alloc_into(o, &m->dl0, n));
    MTRY(alloc_into(o, &m->dl1, n));
    MTRY(alloc_into(o, &m->target, n));
    MTRY(alloc_into(o, &m->cnt, 4));
    MTRY(alloc_into(o, &m->next, 1));
    MTRY(alloc_into(o, &m->akey, b.ninst));
    MTRY(alloc_into(o, &m->anchor, (size_t)kAnchors * b.ninst));
    MTRY(alloc_into(o, &m->ecc, b.ninst));
    MTRY(alloc_into(o, &m->status, b.ninst));
    MTRY(alloc_into(o, &m->skip, b.ninst));
    MTRY(alloc_into(o, &m->stats, (size_t)16 * b.ninst));
    MTRY(alloc_into(o, &m->gscore, b.ninst));
    MTRY(alloc_into(o, &m->ggrad, b.ninst));
    MTRY(alloc_into(o, &m->P0, n * 8));
    MTRY(alloc_into(o, &m->Q0, n * 8));
    MTRY(alloc_into(o, &m->P1, n * 8));
    MTRY(alloc_into(o, &m->Q1, n * 8));
    if (train) {
        MTRY(alloc_into(o, &m->G, n * 64));
        MTRY(alloc_into(o, &m->dC, n * 128));
    }
    m->cap_nv = b.nv;
    m->cap_inst = b.ninst;
    m->cap_train = train;
    return DMOLP_OK;
}

int get_view(dmolp_mpnn *m, dmolp_batch *b, batch::View *v) {
    if (!m) return fail(DMOLP_ERR_ARG, "null model");
    if (!batch::view(b, v)) return fail(DMOLP_ERR_STATE, "no batch uploaded");
    if (v->device != m->device) return fail(DMOLP_ERR_ARG, "model and batch are on different devices");
    MCUDA(cudaSetDevice(m->device));
    return DMOLP_OK;
}

int sync_check(dmolp_mpnn *m, cudaStream_t s, const char *what) {
    MCUDA(cudaStreamSynchronize(s));
    MCUDA(cudaGetLastError());
    int e = 0;
    MCUDA(cudaMemcpy(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(m->err, 0, sizeof(int));
        return fail(DMOLP_ERR_CUDA, std::string(what) + ": a tensor-core wait timed out");
    }
    return DMOLP_OK;
}

GemmArgs base_args(dmolp_mpnn *m, int rows) {
    GemmArgs g;
    std::memset(&g, 0, sizeof(g));
    g.rows = rows;
    g.err = m->err;
    g.polls = m->wait_polls;
    return g;
}

void run_forward(dmolp_mpnn *m, const batch::View &b) {
    const int nv = (int)b.nv;
    cudaStream_t s = b.stream;
    agg_fwd(b.off, b.col, nv, m->C1, kIn, b.num_sms, s);
    __nv_bfloat16 *in[3] = {m->C1, m->C2, m->C3};
    __nv_bfloat16 *out[2] = {m->C2, m->C3};
    for (int l = 0; l < 3; ++l) {
        GemmArgs g = base_args(m, nv);
        g.kind = kFwd;
        g.K = kK[l];
        g.nb = kN[l];
        g.A = in[l];
        g.lda = kK[l];
        g.B = m->Wt[l];
        g.ldb = kK[l];
        g.bias = m->params + kOffB[l];
        if (l < 2) {
            g.relu = 1;
            g.out_bf16 = out[l];
            g.ldo = 2 * kHidden;
        } else {
            g.out_f32 = m->Z3;
            g.ldo32 = kOut;
        }
        gemm(g, kN[l], l == 0 ? 32 : 64, b.num_sms, s);
        if (l < 2) agg_fwd(b.off, b.col, nv, out[l], kHidden, b.num_sms, s);
    }
    m->have_z = true;
}

// Backward from G3 (bf16 dL/dZ3, with db3 already in grads): parameter gradients into m->grads.
void run_backward(dmolp_mpnn *m, const batch::View &b) {
    const int nv = (int)b.nv;
    cudaStream_t s = b.stream;
    const int per = (int)((b.nv + (int64_t)b.num_sms * 4 - 1) / ((int64_t)b.num_sms * 4));
    const int chunk = std::max(64, (per + 63) / 64 * 64);
    __nv_bfloat16 *C[3] = {m->C1, m->C2, m->C3};
    const __nv_bfloat16 *Gin = m->G3;
    int ldg = kOut;
    for (int l = 2; l >= 0; --l) {
        GemmArgs w = base_args(m, nv);
        w.kind = kBwdWeight;
        w.chunk = chunk;
        w.A = C[l];
        w.lda = kK[l];
        w.m_valid = kK[l];
        w.B = Gin;
        w.ldb = ldg;
        w.nb = kN[l];
        w.out_w = m->grads + kOffW[l];
        gemm(w, kN[l], 64, b.num_sms, s);
        if (l == 0) break;
        GemmArgs d = base_args(m, nv);
        d.kind = kBwdData;
        d.K = kN[l];
        d.A = Gin;
        d.lda = ldg;
        d.B = m->W[l];
        d.ldb = kN[l];
        d.nb = kK[l];
        d.out_f32 = m->dC;
        d.ldo32 = 2 * kHidden;
        gemm(d, 2 * kHidden, kN[l] == 16 ? 16 : 64, b.num_sms, s);
        agg_bwd(b.off, b.col, nv, m->dC, C[l], kK[l], m->G, m->grads + kOffB[l - 1], b.num_sms, s);
        Gin = m->G;
        ldg = kHidden;
    }
}

}  // namespace

extern "C" {

int64_t dmolp_mpnn_num_params(void) { return kNumParams; }

int dmolp_mpnn_create(int device, dmolp_mpnn **out) {
    if (!out) return fail(DMOLP_ERR_ARG, "null output");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(DMOLP_ERR_NO_GPU, "no CUDA device");
    }
    if (device < 0 || device >= n) return fail(DMOLP_ERR_ARG, "device index out of range");
    MCUDA(cudaSetDevice(device));
    dmolp_mpnn *m = new dmolp_mpnn();
    m->device = device;
    cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device);
    auto &o = m->fixed;
    int r = alloc_into(o, &m->params, kNumParams);
    if (!r) r = alloc_into(o, &m->grads, kNumParams);
    if (!r) r = alloc_into(o, &m->m, kNumParams);
    if (!r) r = alloc_into(o, &m->v, kNumParams);
    for (int l = 0; l < 3 && !r; ++l) {
        r = alloc_into(o, &m->W[l], (size_t)kK[l] * kN[l]);
        if (!r) r = alloc_into(o, &m->Wt[l], (size_t)kK[l] * kN[l]);
    }
    if (!r) r = alloc_into(o, &m->err, 1);
    if (!r) r = alloc_into(o, &m->loss, 1);
    if (r) {
        dmolp_mpnn_destroy(m);
        return r;
    }
    // Glorot-uniform weights from a fixed seed for the hidden layers, zero biases; the output layer starts at
    // zero, so the untrained proposal is the random-walk features themselves (the network learns a residual)
    std::vector<float> p(kNumParams, 0.f);
    std::mt19937 rng(12345);
    for (int l = 0; l < 2; ++l) {
        const float a = std::sqrt(6.f / (float)(kK[l] + kN[l]));
        std::uniform_real_distribution<float> U(-a, a);
        for (int i = 0; i < kK[l] * kN[l]; ++i) p[kOffW[l] + i] = U(rng);
    }
    r = dmolp_mpnn_set_params(m, p.data());
    if (r) {
        dmolp_mpnn_destroy(m);
        return r;
    }
    cudaMemset(m->err, 0, sizeof(int));
    *out = m;
    return DMOLP_OK;
}

int dmolp_mpnn_set_wait_limit(dmolp_mpnn *m, uint32_t polls) {
    if (!m) return fail(DMOLP_ERR_ARG, "null network");
    m->wait_polls = polls ? polls : (1u << 24);
    return DMOLP_OK;
}

int dmolp_mpnn_destroy(dmolp_mpnn *m) {
    if (!m) return DMOLP_OK;
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    free_ws(m);
    for (void *p : m->fixed) cudaFree(p);
    delete m;
    return DMOLP_OK;
}

int dmolp_mpnn_set_params(dmolp_mpnn *m, const float *params) {
    if (!m || !params) return fail(DMOLP_ERR_ARG, "null argument");
    MCUDA(cudaSetDevice(m->device));
    MCUDA(cudaMemcpy(m->params, params, kNumParams * sizeof(float), cudaMemcpyHostToDevice));
    MCUDA(cudaMemset(m->m, 0, kNumParams * sizeof(float)));
    MCUDA(cudaMemset(m->v, 0, kNumParams * sizeof(float)));
    m->step = 0;
    cast_weights(m->params, m->W, m->Wt, 0);
    MCUDA(cudaDeviceSynchronize());
    return DMOLP_OK;
}

int dmolp_mpnn_get_params(dmolp_mpnn *m, float *params) {
    if (!m || !params) return fail(DMOLP_ERR_ARG, "null argument");
    MCUDA(cudaSetDevice(m->device));
    MCUDA(cudaDeviceSynchronize());
    MCUDA(cudaMemcpy(params, m->params, kNumParams * sizeof(float), cudaMemcpyDeviceToHost));
    return DMOLP_OK;
}

int dmolp_mpnn_features(dmolp_mpnn *m, dmolp_batch *b, float *features) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    MTRY(ensure_ws(m, v, m->cap_train));
    FeatWork w;
    w.off = v.off;
    w.col = v.col;
    w.inst = v.inst;
    w.ninst = v.ninst;
    w.nv = (int)v.nv;
    w.vinst = m->vinst;
    w.dist = m->dist;
    w.mind = m->mind;
    w.front0 = m->f0;
    w.front1 = m->f1;
    w.cnt = m->cnt;
    w.akey = m->akey;
    w.anchor = m->anchor;
    w.ecc = m->ecc;
    w.P0 = m->P0;
    w.Q0 = m->Q0;
    w.P1 = m->P1;
    w.Q1 = m->Q1;
    w.stats = m->stats;
    w.Xf = m->Xf;
    w.X = m->C1;
    w.ldx = 2 * kIn;
    const int e = mpnn::features(w, v.num_sms, v.stream);
    if (e) return fail(DMOLP_ERR_CUDA, std::string("features: ") + cudaGetErrorString((cudaError_t)e));
    if (features)
        MCUDA(cudaMemcpyAsync(features, m->Xf, (size_t)v.nv * 16 * sizeof(float), cudaMemcpyDeviceToHost, v.stream));
    m->have_z = false;
    return sync_check(m, v.stream, "features");
}

int dmolp_mpnn_set_features(dmolp_mpnn *m, dmolp_batch *b, const float *features) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    if (!features) return fail(DMOLP_ERR_ARG, "null features");
    MTRY(ensure_ws(m, v, m->cap_train));
    MCUDA(cudaMemcpyAsync(m->Xf, features, (size_t)v.nv * 16 * sizeof(float), cudaMemcpyHostToDevice, v.stream));
    features_to_input(m->Xf, (int)v.nv, m->C1, 2 * kIn, v.stream);
    m->have_z = false;
    return sync_check(m, v.stream, "set_features");
}

int dmolp_mpnn_forward(dmolp_mpnn *m, dmolp_batch *b, float *embedding) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    if (m->cap_nv < v.nv) return fail(DMOLP_ERR_STATE, "no features for this batch");
    run_forward(m, v);
    if (embedding)
        MCUDA(cudaMemcpyAsync(embedding, m->Z3, (size_t)v.nv * 16 * sizeof(float), cudaMemcpyDeviceToHost, v.stream));
    return sync_check(m, v.stream, "forward");
}

int dmolp_mpnn_backward(dmolp_mpnn *m, dmolp_batch *b, const float *d_embedding, float *grads) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    if (!d_embedding) return fail(DMOLP_ERR_ARG, "null upstream gradient");
    if (m->cap_nv < v.nv) return fail(DMOLP_ERR_STATE, "no features for this batch");
    if (!m->cap_train) return fail(DMOLP_ERR_STATE, "call dmolp_mpnn_prepare_training before the features");
    if (!m->have_z) return fail(DMOLP_ERR_STATE, "run forward first");
    MCUDA(cudaMemsetAsync(m->grads, 0, kNumParams * sizeof(float), v.stream));
    MCUDA(cudaMemcpyAsync(m->dC, d_embedding, (size_t)v.nv * 16 * sizeof(float), cudaMemcpyHostToDevice, v.stream));
    grad_out(m->dC, (int)v.nv, m->G3, m->grads + kOffB[2], v.num_sms, v.stream);
    run_backward(m, v);
    if (grads) MCUDA(cudaMemcpyAsync(grads, m->grads, kNumParams * sizeof(float), cudaMemcpyDeviceToHost, v.stream));
    return sync_check(m, v.stream, "backward");
}

int dmolp_mpnn_prepare_training(dmolp_mpnn *m, dmolp_batch *b) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    return ensure_ws(m, v, true);
}

int dmolp_mpnn_train_step(dmolp_mpnn *m, dmolp_batch *b, const int32_t *target, float lr, double *loss) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    if (!target) return fail(DMOLP_ERR_ARG, "null target");
    if (!m->cap_train || m->cap_nv < v.nv) return fail(DMOLP_ERR_STATE, "call dmolp_mpnn_prepare_training first");
    cudaStream_t s = v.stream;
    MCUDA(cudaMemcpyAsync(m->target, target, (size_t)v.nv * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    run_forward(m, v);
    MCUDA(cudaMemsetAsync(m->grads, 0, kNumParams * sizeof(float), s));
    MCUDA(cudaMemsetAsync(m->loss, 0, sizeof(double), s));
    coords(m->Xf, m->Z3, (int)v.nv, m->Pc, v.num_sms, s);
    mpnn::loss(v.off, v.col, (int)v.nv, m->Pc, m->target, v.narcs > 0 ? 1.0 / (double)v.narcs : 0.0, m->G3,
               m->grads + kOffB[2], m->loss, v.num_sms, s);
    run_backward(m, v);
    adam(m->params, m->grads, m->m, m->v, kNumParams, lr, ++m->step, s);
    cast_weights(m->params, m->W, m->Wt, s);
    double h = 0;
    MCUDA(cudaMemcpyAsync(&h, m->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    MTRY(sync_check(m, s, "train_step"));
    if (loss) *loss = v.narcs > 0 ? h / (double)v.narcs : 0.0;
    m->have_z = false;
    return DMOLP_OK;
}

// Decoder over the batch; graphs marked in skip_host (may be null) keep their labels and get status 2.
static int decode_impl(dmolp_mpnn *m, dmolp_batch *b, const float *embedding, const uint8_t *skip_host,
                       int32_t *status) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    if (m->cap_nv < v.nv) return fail(DMOLP_ERR_STATE, "no workspace for this batch");
    if (embedding)
        MCUDA(cudaMemcpyAsync(m->Z3, embedding, (size_t)v.nv * 16 * sizeof(float), cudaMemcpyHostToDevice, v.stream));
    else if (!m->have_z)
        return fail(DMOLP_ERR_STATE, "run forward first or pass an embedding");
    coords(m->Xf, m->Z3, (int)v.nv, m->Pc, v.num_sms, v.stream);
    DecodeWork w;
    w.inst = v.inst;
    w.order = v.order;
    w.ninst = v.ninst;
    w.Z = m->Pc;
    w.Y = m->Y;
    w.label = v.label;
    w.l0 = m->dl0;
    w.l1 = m->dl1;
    w.status = m->status;
    w.next = m->next;
    w.skip = nullptr;
    if (skip_host) {
        MCUDA(cudaMemcpyAsync(m->skip, skip_host, v.ninst, cudaMemcpyHostToDevice, v.stream));
        w.skip = m->skip;
    }
    decode(w, std::max(1, std::min(v.ninst, v.num_sms * 2)), v.stream);
    if (status) MCUDA(cudaMemcpyAsync(status, m->status, v.ninst * sizeof(int32_t), cudaMemcpyDeviceToHost, v.stream));
    return sync_check(m, v.stream, "decode");
}

int dmolp_mpnn_decode(dmolp_mpnn *m, dmolp_batch *b, const float *embedding, int32_t *status) {
    return decode_impl(m, b, embedding, nullptr, status);
}

int dmolp_mpnn_gate(dmolp_mpnn *m, dmolp_batch *b, double *scores) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    if (!scores) return fail(DMOLP_ERR_ARG, "null scores");
    if (!m->have_z) return fail(DMOLP_ERR_STATE, "run forward first");
    MCUDA(cudaMemsetAsync(m->gscore, 0, v.ninst * sizeof(double), v.stream));
    gate_scores(m->Z3, m->vinst, (int)v.nv, m->gscore, v.num_sms, v.stream);
    MCUDA(cudaMemcpyAsync(scores, m->gscore, v.ninst * sizeof(double), cudaMemcpyDeviceToHost, v.stream));
    MTRY(sync_check(m, v.stream, "gate"));
    std::vector<batch::Inst> hi(v.ninst);
    MCUDA(cudaMemcpy(hi.data(), v.inst, v.ninst * sizeof(batch::Inst), cudaMemcpyDeviceToHost));
    for (int i = 0; i < v.ninst; ++i) scores[i] = hi[i].nv > 0 ? scores[i] / (double)hi[i].nv : 0.0;
    return DMOLP_OK;
}

int dmolp_mpnn_train_gate(dmolp_mpnn *m, dmolp_batch *b, const float *target, float lr, double *loss) {
    batch::View v;
    MTRY(get_view(m, b, &v));
    if (!target) return fail(DMOLP_ERR_ARG, "null target");
    if (!m->cap_train || m->cap_nv < v.nv) return fail(DMOLP_ERR_STATE, "call dmolp_mpnn_prepare_training first");
    cudaStream_t s = v.stream;
    run_forward(m, v);
    std::vector<double> sc(v.ninst);
    MTRY(dmolp_mpnn_gate(m, b, sc.data()));
    std::vector<batch::Inst> hi(v.ninst);
    MCUDA(cudaMemcpy(hi.data(), v.inst, v.ninst * sizeof(batch::Inst), cudaMemcpyDeviceToHost));
    // binary cross-entropy of sigmoid(score) against the target, mean over graphs
    std::vector<float> g(v.ninst, 0.f);
    double L = 0.0;
    int ng = 0;
    for (int i = 0; i < v.ninst; ++i) ng += hi[i].nv > 0;
    for (int i = 0; i < v.ninst; ++i) {
        if (hi[i].nv == 0) continue;
        const double p = 1.0 / (1.0 + std::exp(-sc[i])), y = target[i];
        L += -(y * std::log(std::max(p, 1e-12)) + (1.0 - y) * std::log(std::max(1.0 - p, 1e-12)));
        g[i] = (float)((p - y) / (double)std::max(1, ng) / (double)hi[i].nv);
    }
    MCUDA(cudaMemcpyAsync(m->ggrad, g.data(), v.ninst * sizeof(float), cudaMemcpyHostToDevice, s));
    MCUDA(cudaMemsetAsync(m->grads, 0, kNumParams * sizeof(float), s));
    gate_grad(m->ggrad, m->vinst, (int)v.nv, m->dC, v.num_sms, s);
    grad_out(m->dC, (int)v.nv, m->G3, m->grads + kOffB[2], v.num_sms, s);
    run_backward(m, v);
    adam(m->params, m->grads, m->m, m->v, kNumParams, lr, ++m->step, s);
    cast_weights(m->params, m->W, m->Wt, s);
    MTRY(sync_check(m, s, "train_gate"));
    if (loss) *loss = ng > 0 ? L / ng : 0.0;
    m->have_z = false;
    return DMOLP_OK;
}

int dmolp_batch_propose(dmolp_batch *b, dmolp_mpnn *m, int32_t *status) {
    MTRY(dmolp_mpnn_features(m, b, nullptr));
    MTRY(dmolp_mpnn_forward(m, b, nullptr));
    batch::View v;
    MTRY(get_view(m, b, &v));
    std::vector<double> sc(v.ninst);
    MTRY(dmolp_mpnn_gate(m, b, sc.data()));
    // only the graphs the gate accepts are decoded; the others keep their labels for phase 1 (status 2)
    std::vector<uint8_t> skip(v.ninst);
    for (int i = 0; i < v.ninst; ++i) skip[i] = sc[i] < 0.0;
    std::vector<int32_t> st(v.ninst);
    MTRY(decode_impl(m, b, nullptr, skip.data(), st.data()));
    if (status) std::memcpy(status, st.data(), v.ninst * sizeof(int32_t));
    return DMOLP_OK;
}

}  // extern "C"
