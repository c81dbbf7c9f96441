// Learned initial-partition proposal: shared declarations of the network kernels (mpnn_kernels.cu) and the
// C-ABI (mpnn_cabi.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "batch.cuh"

namespace dmolp {
namespace mpnn {

constexpr int kIn = 16, kHidden = 64, kOut = 16;
constexpr int kAnchors = 8;
constexpr int kTMax = 96;
constexpr float kMargin = 1.0f;
constexpr float kPFloor = 1e-30f;
// layer l: [K_l x N_l] weights + N_l biases, K_l = 2 * (input width)
constexpr int kK[3] = {2 * kIn, 2 * kHidden, 2 * kHidden};
constexpr int kN[3] = {kHidden, kHidden, kOut};
constexpr int kNumParams = 2 * kIn * kHidden + kHidden + 2 * kHidden * kHidden + kHidden + 2 * kHidden * kOut + kOut;

enum GemmKind { kFwd = 0, kBwdData = 1, kBwdWeight = 2 };

struct GemmArgs {
    int kind;
    int rows;        // vertices
    int K;           // kFwd / kBwdData: reduction length (multiple of 16)
    int nb;          // valid B rows (kFwd / kBwdData) or valid output columns
    int m_valid;     // kBwdWeight: valid rows of dW
    int chunk;       // kBwdWeight: vertices per work item (multiple of the K tile)
    const __nv_bfloat16 *A;
    int lda;
    const __nv_bfloat16 *B;
    int ldb;
    const float *bias;
    int relu;
    __nv_bfloat16 *out_bf16;
    int ldo;
    float *out_f32;
    int ldo32;
    float *out_w;
    int *err;
    uint32_t polls;  // polls of the MMA completion barrier before the GEMM gives up (then: err, TMEM freed)
};

// One launch of the tensor-core GEMM: N = output tile width, KT = K tile.
void gemm(const GemmArgs &g, int n, int kt, int num_sms, cudaStream_t s);

void agg_fwd(const int64_t *off, const int32_t *col, int nv, __nv_bfloat16 *buf, int C, int num_sms, cudaStream_t s);
void agg_bwd(const int64_t *off, const int32_t *col, int nv, const float *dC, const __nv_bfloat16 *Hbuf, int ldh,
             __nv_bfloat16 *G, float *db, int num_sms, cudaStream_t s);
void loss(const int64_t *off, const int32_t *col, int nv, const float *Z, const int32_t *target, double inv_arcs,
          __nv_bfloat16 *G, float *db, double *loss_sum, int num_sms, cudaStream_t s);
void grad_out(const float *dZ, int nv, __nv_bfloat16 *G, float *db, int num_sms, cudaStream_t s);
void adam(float *p, const float *g, float *m, float *v, int n, float lr, int step, cudaStream_t s);
void cast_weights(const float *params, __nv_bfloat16 *const W[3], __nv_bfloat16 *const Wt[3], cudaStream_t s);

struct FeatWork {
    const int64_t *off;
    const int32_t *col;
    const batch::Inst *inst;
    int ninst;
    int nv;
    int32_t *vinst, *dist, *mind, *front0, *front1, *cnt;  // cnt[4]
    unsigned long long *akey;                              // [ninst]
    int32_t *anchor;                                       // [kAnchors * ninst]
    int32_t *ecc;                                          // [ninst]
    float *P0, *Q0, *P1, *Q1;                              // [nv * 8]
    double *stats;                                         // [ninst * 16]
    float *Xf;                                             // [nv * 16] features before rounding
    __nv_bfloat16 *X;                                      // [nv * ldx] bf16 input of layer 1
    int ldx;
};
int features(const FeatWork &w, int num_sms, cudaStream_t s);  // returns a CUDA error code (0 = ok)
void features_to_input(const float *Xf, int nv, __nv_bfloat16 *X, int ldx, cudaStream_t s);

struct DecodeWork {
    const batch::Inst *inst;
    const int32_t *order;
    int ninst;
    const float *Z;  // [nv * 16] proposal coordinates (first 8 columns used)
    float *Y;        // [nv * 4] principal coordinates (work)
    int32_t *label;
    int32_t *l0, *l1;  // [nv] each
    int32_t *status;   // [ninst]
    int *next;
    const uint8_t *skip;  // [ninst] or null: graphs left alone (status 2, labels untouched)
};
void decode(const DecodeWork &w, int grid, cudaStream_t s);
void coords(const float *Xf, const float *Z, int nv, float *P, int num_sms, cudaStream_t s);
void gate_scores(const float *Z, const int32_t *vinst, int nv, double *score, int num_sms, cudaStream_t s);
void gate_grad(const float *g, const int32_t *vinst, int nv, float *dZ, int num_sms, cudaStream_t s);

}  // namespace mpnn
}  // namespace dmolp
