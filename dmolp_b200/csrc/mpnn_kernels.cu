// Learned initial-partition proposal: the kernels of a 3-layer mean-aggregation message-passing network
// (BF16 weights and activations, FP32 accumulation on the tcgen05 tensor cores), its training step, its
// input features and the decoder that turns its embedding into k balanced labels per graph.
//
//   layer l:  Z_l = [H_l | mean over neighbours of H_l] @ W_l + b_l,   H_{l+1} = ReLU(Z_l)  (l = 1, 2)
//   sizes:    16 -> 64 -> 64 -> 16;  inputs: degree / mean degree, log(1 + degree), 8 random-walk
//             features, k / 64 (the remaining input columns are 0)
//
// The concatenation [H | mean H] is one BF16 buffer per layer: the GEMM epilogue of layer l writes H_{l+1}
// into the left half of layer l+1's buffer and the aggregation kernel fills its right half.  The GEMMs
// stage 128-row tiles of A and the B tile into shared memory in the no-swizzle K-major core-matrix layout
// (umma.cuh), one thread issues tcgen05.mma into a tensor-memory accumulator, completion is signalled on an
// mbarrier (bounded wait: a stuck MMA sets an error flag instead of hanging), and the epilogue reads the
// accumulator with tcgen05.ld.  The weight gradient is the same GEMM with vertices as the reduction axis,
// staged transposed, each CTA adding its partial sums to dW with atomics.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "mpnn.cuh"
#include "umma.cuh"

namespace dmolp {
namespace mpnn {
namespace {

// Polls of the MMA completion barrier after a GEMM gave up (GemmArgs::polls): the MMA in flight still
// completes before its TMEM is freed; far above any real MMA's time.
constexpr uint32_t kWaitLimit = 1u << 24;

__device__ __forceinline__ uint4 zero4() { return make_uint4(0, 0, 0, 0); }

// ------------------------------------------------------------------------------------------------ GEMM
template <int N, int KT>
__global__ void __launch_bounds__(128) k_gemm(GemmArgs g) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tslot;
    constexpr uint32_t NCOL = N < 32 ? 32 : N;
    constexpr int CH = KT / 8;  // 16-byte chunks per tile row
    uint8_t *sA = smem, *sB = smem + 128 * KT * 2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) umma::tmem_alloc(&tslot, NCOL);
    if (tid == 0) {
        umma::mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    constexpr uint32_t idesc = umma::idesc_bf16_f32(128, N);
    uint32_t phase = 0;
    int ok = 1;
    const bool wgt = g.kind == kBwdWeight;
    const int nitems = wgt ? (g.rows + g.chunk - 1) / g.chunk : (g.rows + 127) / 128;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int r0 = wgt ? item * g.chunk : item * 128;
        const int ktot = wgt ? min(g.chunk, g.rows - r0) : g.K;
        for (int kc = 0; kc < ktot; kc += KT) {
            // ---- stage the A (128 x KT) and B (N x KT) tiles ----
            if (!wgt) {
                for (int q = tid; q < 128 * CH; q += 128) {
                    const int r = q / CH, c = q % CH, row = r0 + r, kk = kc + c * 8;
                    uint4 x = zero4();
                    if (row < g.rows && kk < g.K) x = *reinterpret_cast<const uint4 *>(g.A + (size_t)row * g.lda + kk);
                    *reinterpret_cast<uint4 *>(sA + umma::tile_offset(r, c * 8, KT)) = x;
                }
                for (int q = tid; q < N * CH; q += 128) {
                    const int n = q / CH, c = q % CH, kk = kc + c * 8;
                    uint4 x = zero4();
                    if (n < g.nb && kk < g.K) x = *reinterpret_cast<const uint4 *>(g.B + (size_t)n * g.ldb + kk);
                    *reinterpret_cast<uint4 *>(sB + umma::tile_offset(n, c * 8, KT)) = x;
                }
            } else {
                // A(m, k) = C[vertex r0+kc+k][feature m], B(n, k) = G[vertex r0+kc+k][n]: transposed staging
                for (int q = tid; q < KT * 16; q += 128) {
                    const int k = q / 16, m = (q % 16) * 8, v = kc + k;
                    uint4 x = zero4();
                    if (v < ktot && m < g.m_valid)
                        x = *reinterpret_cast<const uint4 *>(g.A + (size_t)(r0 + v) * g.lda + m);
                    const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&x);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        *reinterpret_cast<__nv_bfloat16 *>(sA + umma::tile_offset(m + j, k, KT)) = e[j];
                }
                for (int q = tid; q < KT * (N / 8); q += 128) {
                    const int k = q / (N / 8), n = (q % (N / 8)) * 8, v = kc + k;
                    uint4 x = zero4();
                    if (v < ktot) x = *reinterpret_cast<const uint4 *>(g.B + (size_t)(r0 + v) * g.ldb + n);
                    const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&x);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        *reinterpret_cast<__nv_bfloat16 *>(sB + umma::tile_offset(n + j, k, KT)) = e[j];
                }
            }
            umma::fence_async_smem();
            umma::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                umma::fence_after_sync();
                const uint32_t a0 = umma::smem_addr(sA), b0 = umma::smem_addr(sB);
#pragma unroll
                for (int s = 0; s < KT / 16; ++s)
                    umma::mma_bf16(tmem, umma::smem_desc(a0 + 256 * s, 128, KT * 16),
                                   umma::smem_desc(b0 + 256 * s, 128, KT * 16), idesc, kc > 0 || s > 0);
                umma::mma_commit(&mbar);
            }
            const bool done = umma::mbar_wait(&mbar, phase, g.polls);
            ok = __syncthreads_and(done);
            if (!ok) break;
            phase ^= 1;
            umma::fence_after_sync();
        }
        if (!ok) break;
        // ---- epilogue: warp w owns accumulator rows (TMEM lanes) 32w .. 32w+31 ----
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        const int r = warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            umma::tmem_ld16(trow + c0, v);
            if (wgt) {
                if (r < g.m_valid)
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (c0 + i < g.nb && v[i] != 0.0f) atomicAdd(&g.out_w[(size_t)r * g.nb + c0 + i], v[i]);
            } else {
                const int row = r0 + r;
                if (row < g.rows) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        if (g.bias) v[i] = __fadd_rn(v[i], g.bias[c0 + i]);
                        if (g.relu) v[i] = fmaxf(v[i], 0.0f);
                    }
                    if (g.out_bf16) {
                        __align__(16) __nv_bfloat16 h[16];
#pragma unroll
                        for (int i = 0; i < 16; ++i) h[i] = __float2bfloat16_rn(v[i]);
                        uint4 *dst = reinterpret_cast<uint4 *>(g.out_bf16 + (size_t)row * g.ldo + c0);
                        dst[0] = reinterpret_cast<const uint4 *>(h)[0];
                        dst[1] = reinterpret_cast<const uint4 *>(h)[1];
                    }
                    if (g.out_f32) {
                        float4 *dst = reinterpret_cast<float4 *>(g.out_f32 + (size_t)row * g.ldo32 + c0);
#pragma unroll
                        for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                    }
                }
            }
        }
        umma::fence_before_sync();
        __syncthreads();  // the accumulator is read before the next tile's first MMA overwrites it
    }
    if (!ok) {
        umma::mbar_wait(&mbar, phase, kWaitLimit);  // let an MMA still in flight finish before the free
        if (tid == 0) atomicExch(g.err, 1);
    }
    __syncthreads();
    if (warp == 0) umma::tmem_free(tmem, NCOL);
}

// ------------------------------------------------------------------------------------ aggregation
// Right half of buf (row stride 2C) = bf16(mean over neighbours of the left half), fp32 sums in row order.
template <int C>
__global__ void k_agg_fwd(const int64_t *__restrict__ off, const int32_t *__restrict__ col, int nv,
                          __nv_bfloat16 *__restrict__ buf) {
    constexpr int G = C / 2;  // lanes per vertex, two channels each
    const int lane = threadIdx.x & 31, sub = lane / G, sl = lane % G;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = ((int64_t)gridDim.x * blockDim.x >> 5) * (32 / G);
    for (int64_t v = gw * (32 / G) + sub; v < nv; v += stride) {
        const int64_t s = off[v], e = off[v + 1];
        float a0 = 0.f, a1 = 0.f;
        for (int64_t j = s; j < e; ++j) {
            const int u = __ldg(col + j);
            const __nv_bfloat162 x = *reinterpret_cast<const __nv_bfloat162 *>(buf + (size_t)u * 2 * C + 2 * sl);
            a0 = __fadd_rn(a0, __bfloat162float(x.x));
            a1 = __fadd_rn(a1, __bfloat162float(x.y));
        }
        const float inv = e > s ? (float)(1.0 / (double)(e - s)) : 0.f;
        *reinterpret_cast<__nv_bfloat162 *>(buf + (size_t)v * 2 * C + C + 2 * sl) =
            __floats2bfloat162_rn(__fmul_rn(a0, inv), __fmul_rn(a1, inv));
    }
}

// Backward of one layer's input (64 channels): dH = dC[:, :64] + sum over neighbours v of dC[v, 64:] / deg(v)
// (the transpose of the mean for a symmetric graph); G = bf16(dH * [H > 0]); db += column sums of G.
__global__ void k_agg_bwd(const int64_t *__restrict__ off, const int32_t *__restrict__ col, int nv,
                          const float *__restrict__ dC, const __nv_bfloat16 *__restrict__ H, int ldh,
                          __nv_bfloat16 *__restrict__ G, float *__restrict__ db) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = (int64_t)gridDim.x * blockDim.x >> 5;
    float s0 = 0.f, s1 = 0.f;
    for (int64_t u = gw; u < nv; u += nw) {
        const int64_t s = off[u], e = off[u + 1];
        float a0 = 0.f, a1 = 0.f;
        for (int64_t j = s; j < e; ++j) {
            const int v = __ldg(col + j);
            const int64_t dv = off[v + 1] - off[v];
            const float inv = dv > 0 ? (float)(1.0 / (double)dv) : 0.f;
            const float2 x = *reinterpret_cast<const float2 *>(dC + (size_t)v * 128 + 64 + 2 * lane);
            a0 = __fadd_rn(a0, __fmul_rn(x.x, inv));
            a1 = __fadd_rn(a1, __fmul_rn(x.y, inv));
        }
        const float2 l = *reinterpret_cast<const float2 *>(dC + (size_t)u * 128 + 2 * lane);
        const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162 *>(H + (size_t)u * ldh + 2 * lane);
        const float g0 = __bfloat162float(h.x) > 0.f ? __fadd_rn(l.x, a0) : 0.f;
        const float g1 = __bfloat162float(h.y) > 0.f ? __fadd_rn(l.y, a1) : 0.f;
        const __nv_bfloat162 q = __floats2bfloat162_rn(g0, g1);
        *reinterpret_cast<__nv_bfloat162 *>(G + (size_t)u * 64 + 2 * lane) = q;
        s0 += __bfloat162float(q.x);
        s1 += __bfloat162float(q.y);
    }
    if (s0 != 0.f) atomicAdd(&db[2 * lane], s0);
    if (s1 != 0.f) atomicAdd(&db[2 * lane + 1], s1);
}

// Edge-contrastive loss over arcs (v, u): y * d2 + (1 - y) * max(0, margin - d2), y = same target label,
// d2 = |z_v - z_u|^2.  Four lanes per vertex (4 channels each).  G3 = bf16(dL/dz), db3 += its column sums.
__global__ void k_loss(const int64_t *__restrict__ off, const int32_t *__restrict__ col, int nv,
                       const float *__restrict__ Z, const int32_t *__restrict__ target, float scale,
                       __nv_bfloat16 *__restrict__ G, float *__restrict__ db, double *__restrict__ loss_sum) {
    const int lane = threadIdx.x & 31, sub = lane >> 2, q = lane & 3;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = ((int64_t)gridDim.x * blockDim.x >> 5) * 8;
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    double ls = 0.0;
    for (int64_t v0 = gw * 8; v0 < nv; v0 += stride) {
        const int64_t v = v0 + sub;
        const bool act = v < nv;
        const int64_t b = act ? off[v] : 0, e = act ? off[v + 1] : 0;
        const float4 zv = act ? *reinterpret_cast<const float4 *>(Z + (size_t)v * 16 + 4 * q) : make_float4(0, 0, 0, 0);
        const int tv = act ? target[v] : 0;
        float g[4] = {0.f, 0.f, 0.f, 0.f};
        // every lane of the warp runs the longest row of its 8 vertices (the shuffles need all lanes)
        int64_t len = e - b, mx = len;
        for (int o = 4; o < 32; o <<= 1) mx = max(mx, (int64_t)__shfl_xor_sync(DMOLP_FULL_MASK, (long long)mx, o));
        for (int64_t t = 0; t < mx; ++t) {
            const bool on = t < len;
            const int u = on ? __ldg(col + b + t) : 0;
            float4 zu = make_float4(0, 0, 0, 0);
            if (on) zu = *reinterpret_cast<const float4 *>(Z + (size_t)u * 16 + 4 * q);
            const float d[4] = {__fsub_rn(zv.x, zu.x), __fsub_rn(zv.y, zu.y), __fsub_rn(zv.z, zu.z),
                                __fsub_rn(zv.w, zu.w)};
            float p = 0.f;
#pragma unroll
            for (int i = 0; i < 4; ++i) p = __fadd_rn(p, __fmul_rn(d[i], d[i]));
            p += __shfl_xor_sync(DMOLP_FULL_MASK, p, 1);
            p += __shfl_xor_sync(DMOLP_FULL_MASK, p, 2);
            if (on) {
                const bool y = target[u] == tv;
                const float coef = y ? 2.f : (p < kMargin ? -2.f : 0.f);
#pragma unroll
                for (int i = 0; i < 4; ++i) g[i] = __fadd_rn(g[i], __fmul_rn(coef, d[i]));
                if (q == 0) ls += y ? (double)p : (double)fmaxf(0.f, kMargin - p);
            }
        }
        if (act) {
            __align__(8) __nv_bfloat16 h[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                h[i] = __float2bfloat16_rn(__fmul_rn(g[i], scale));
                s[i] += __bfloat162float(h[i]);
            }
            *reinterpret_cast<uint2 *>(G + (size_t)v * 16 + 4 * q) = *reinterpret_cast<const uint2 *>(h);
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (s[i] != 0.f) atomicAdd(&db[4 * q + i], s[i]);
    if (q == 0 && ls != 0.0) atomicAdd(loss_sum, ls);
}

// An upstream gradient given in FP32: G = bf16(dZ) [nv x 16], db += its column sums.
__global__ void k_grad_out(const float *dZ, int nv, __nv_bfloat16 *G, float *db) {
    const int c = threadIdx.x & 15;
    float s = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)nv * 16;
         i += (int64_t)gridDim.x * blockDim.x) {
        const __nv_bfloat16 h = __float2bfloat16_rn(dZ[i]);
        G[i] = h;
        s += __bfloat162float(h);
    }
    if (s != 0.f) atomicAdd(&db[c], s);
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

__global__ void k_cast(const float *params, __nv_bfloat16 *W0, __nv_bfloat16 *W1, __nv_bfloat16 *W2,
                       __nv_bfloat16 *T0, __nv_bfloat16 *T1, __nv_bfloat16 *T2) {
    int o = 0;
    __nv_bfloat16 *W[3] = {W0, W1, W2}, *T[3] = {T0, T1, T2};
    const int Ks[3] = {2 * kIn, 2 * kHidden, 2 * kHidden}, Ns[3] = {kHidden, kHidden, kOut};
    for (int l = 0; l < 3; ++l) {
        const int K = Ks[l], N = Ns[l];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < K * N; i += gridDim.x * blockDim.x) {
            const int r = i / N, c = i % N;
            const __nv_bfloat16 h = __float2bfloat16_rn(params[o + i]);
            W[l][i] = h;
            T[l][c * K + r] = h;
        }
        o += K * N + N;
    }
}

// ------------------------------------------------------------------------------------ features
__device__ __forceinline__ int inst_of(const batch::Inst *inst, int ninst, int v) {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (inst[mid].vbase <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_vinst(const batch::Inst *inst, int ninst, int nv, int32_t *vinst) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        int i = inst_of(inst, ninst, v);
        while (i + 1 < ninst && inst[i + 1].vbase <= v && inst[i].nv == 0) ++i;  // empty instances share vbase
        vinst[v] = i;
    }
}

// Candidate keys for the next anchor: (value << 32) | (~local id), maximum = largest value, lowest id.
__global__ void k_anchor_key(const FeatWork w, int j) {
    const int lane = threadIdx.x & 31;
    for (int v0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); v0 < w.nv; v0 += gridDim.x * blockDim.x) {
        const int v = v0 + lane;
        int i = -1;
        unsigned long long key = 0;
        if (v < w.nv) {
            i = w.vinst[v];
            const unsigned lid = (unsigned)(v - (int)w.inst[i].vbase);
            const long long val = j == 0 ? (long long)(w.off[v + 1] - w.off[v]) : (long long)w.mind[v];
            if (val >= 0) key = ((unsigned long long)val << 32) | (unsigned long long)(0xFFFFFFFFu - lid);
            else i = -1;
        }
        const int i0 = __shfl_sync(DMOLP_FULL_MASK, i, 0);
        if (__all_sync(DMOLP_FULL_MASK, i == i0) && i0 >= 0) {  // one graph: one atomic per warp
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long y = __shfl_xor_sync(DMOLP_FULL_MASK, key, o);
                key = y > key ? y : key;
            }
            if (lane == 0) atomicMax(&w.akey[i0], key);
        } else if (i >= 0) {
            atomicMax(&w.akey[i], key);
        }
    }
}

__global__ void k_anchor_pick(const FeatWork w, int j) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w.ninst; i += gridDim.x * blockDim.x) {
        const batch::Inst I = w.inst[i];
        int a = -1;
        if (I.nv > 0) a = (int)I.vbase + (int)(0xFFFFFFFFu - (unsigned)(w.akey[i] & 0xFFFFFFFFull));
        w.anchor[j * w.ninst + i] = a;
        w.akey[i] = 0;
        if (a >= 0) {
            w.dist[a] = 0;
            w.front0[atomicAdd(&w.cnt[0], 1)] = a;
        }
    }
}

__global__ void k_fill_i32(int32_t *p, int n, int32_t x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = x;
}

// One BFS level: unvisited neighbours of the frontier get level + 1.  The frontier counts rotate over three
// counters: level L reads cnt[L%3], appends to cnt[(L+1)%3] and clears cnt[(L+2)%3], the count the next
// level appends to (nothing reads it now), so levels run back to back with no host work in between; a level
// after the frontier has emptied does nothing.
__global__ void k_bfs_level(const int64_t *__restrict__ off, const int32_t *__restrict__ col, int32_t *dist,
                            const int32_t *fin, int32_t *fout, int *cnt, int level) {
    const int n = cnt[level % 3];
    int *nout = cnt + (level + 1) % 3;
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[(level + 2) % 3] = 0;
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < n; i += nw) {
        const int v = fin[i];
        const int64_t s = off[v], e = off[v + 1];
        for (int64_t j0 = s; j0 < e; j0 += 32) {  // warp-uniform trip count: one append per warp and step
            const int64_t j = j0 + lane;
            int u = 0;
            bool found = false;
            if (j < e) {
                u = __ldg(col + j);
                found = dist[u] < 0 && atomicCAS(&dist[u], -1, level + 1) == -1;
            }
            const int slot = warp_append(nout, found);
            if (found) fout[slot] = u;
        }
    }
}

__global__ void k_mind(const FeatWork w, int j) {
    const int lane = threadIdx.x & 31;
    for (int v0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); v0 < w.nv; v0 += gridDim.x * blockDim.x) {
        const int v = v0 + lane;
        const int d = v < w.nv ? w.dist[v] : -1;
        if (j == 0) {
            const int i = v < w.nv ? w.vinst[v] : -1;
            if (v < w.nv) w.mind[v] = d;
            const int i0 = __shfl_sync(DMOLP_FULL_MASK, i, 0);
            if (__all_sync(DMOLP_FULL_MASK, i == i0)) {
                int m = d;
                for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(DMOLP_FULL_MASK, m, o));
                if (lane == 0 && m > 0) atomicMax(&w.ecc[i0], m);
            } else if (d > 0) {
                atomicMax(&w.ecc[i], d);
            }
        } else if (v < w.nv) {
            const int m = w.mind[v];
            if (m >= 0 && d >= 0 && d < m) w.mind[v] = d;
        }
    }
}

// Random walk state: P (landing probabilities, 8 channels), Q = P / deg.
__global__ void k_rw_init(const FeatWork w) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < w.nv; v += gridDim.x * blockDim.x) {
        float p[8];
        const int i = w.vinst[v];
        for (int j = 0; j < 8; ++j) p[j] = w.anchor[j * w.ninst + i] == v ? 1.f : 0.f;
        const int64_t d = w.off[v + 1] - w.off[v];
        const float inv = d > 0 ? (float)(1.0 / (double)d) : 0.f;
        float4 *P = reinterpret_cast<float4 *>(w.P0 + (size_t)v * 8), *Q = reinterpret_cast<float4 *>(w.Q0 + (size_t)v * 8);
        P[0] = make_float4(p[0], p[1], p[2], p[3]);
        P[1] = make_float4(p[4], p[5], p[6], p[7]);
        Q[0] = make_float4(__fmul_rn(p[0], inv), __fmul_rn(p[1], inv), __fmul_rn(p[2], inv), __fmul_rn(p[3], inv));
        Q[1] = make_float4(__fmul_rn(p[4], inv), __fmul_rn(p[5], inv), __fmul_rn(p[6], inv), __fmul_rn(p[7], inv));
    }
}

// One lazy step P' = P/2 + (sum over neighbours of Q)/2 for graphs that still walk (step < T of the graph).
__global__ void k_rw_step(const FeatWork w, const float *Pin, const float *Qin, float *Pout, float *Qout, int step) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < w.nv; v += gridDim.x * blockDim.x) {
        const int i = w.vinst[v];
        const int T = min(max(w.ecc[i], 1), kTMax);
        const float4 *pi = reinterpret_cast<const float4 *>(Pin + (size_t)v * 8);
        float4 *po = reinterpret_cast<float4 *>(Pout + (size_t)v * 8), *qo = reinterpret_cast<float4 *>(Qout + (size_t)v * 8);
        if (step >= T) continue;  // the graph has walked its T steps: its result stays in the buffer of step T-1
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const int64_t b = w.off[v], e = w.off[v + 1];
        for (int64_t j = b; j < e; ++j) {
            const int u = __ldg(w.col + j);
            const float4 a = reinterpret_cast<const float4 *>(Qin + (size_t)u * 8)[0];
            const float4 c = reinterpret_cast<const float4 *>(Qin + (size_t)u * 8)[1];
            s[0] = __fadd_rn(s[0], a.x);
            s[1] = __fadd_rn(s[1], a.y);
            s[2] = __fadd_rn(s[2], a.z);
            s[3] = __fadd_rn(s[3], a.w);
            s[4] = __fadd_rn(s[4], c.x);
            s[5] = __fadd_rn(s[5], c.y);
            s[6] = __fadd_rn(s[6], c.z);
            s[7] = __fadd_rn(s[7], c.w);
        }
        const float4 p0 = pi[0], p1 = pi[1];
        const float p[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
        float r[8], q[8];
        const float inv = e > b ? (float)(1.0 / (double)(e - b)) : 0.f;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            r[j] = __fadd_rn(__fmul_rn(0.5f, p[j]), __fmul_rn(0.5f, s[j]));
            q[j] = __fmul_rn(r[j], inv);
        }
        po[0] = make_float4(r[0], r[1], r[2], r[3]);
        po[1] = make_float4(r[4], r[5], r[6], r[7]);
        qo[0] = make_float4(q[0], q[1], q[2], q[3]);
        qo[1] = make_float4(q[4], q[5], q[6], q[7]);
    }
}

// log landing probabilities, their per-graph sums and sums of squares (double).  A graph that walked T steps
// left its probabilities in P0 (T even) or P1 (T odd): steps alternate the two buffers.
__global__ void k_rw_log(const FeatWork w) {
    const int lane = threadIdx.x & 31;
    for (int v0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); v0 < w.nv; v0 += gridDim.x * blockDim.x) {
        const int v = v0 + lane;
        const int i = v < w.nv ? w.vinst[v] : -1;
        const int i0 = __shfl_sync(DMOLP_FULL_MASK, i, 0);
        const bool uni = __all_sync(DMOLP_FULL_MASK, i == i0);
        for (int j = 0; j < 8; ++j) {
            double a = 0.0, b = 0.0;
            if (v < w.nv) {
                const float *P = (min(max(w.ecc[i], 1), kTMax) & 1) ? w.P1 : w.P0;
                const float L = logf(fmaxf(P[(size_t)v * 8 + j], kPFloor));
                w.Xf[(size_t)v * 16 + 2 + j] = L;
                a = (double)L;
                b = (double)L * (double)L;
            }
            if (uni) {
                for (int o = 16; o > 0; o >>= 1) {
                    a += __shfl_xor_sync(DMOLP_FULL_MASK, a, o);
                    b += __shfl_xor_sync(DMOLP_FULL_MASK, b, o);
                }
                if (lane == 0) {
                    atomicAdd(&w.stats[i0 * 16 + j], a);
                    atomicAdd(&w.stats[i0 * 16 + 8 + j], b);
                }
            } else if (i >= 0) {
                atomicAdd(&w.stats[i * 16 + j], a);
                atomicAdd(&w.stats[i * 16 + 8 + j], b);
            }
        }
    }
}

__global__ void k_feat_final(const FeatWork w) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < w.nv; v += gridDim.x * blockDim.x) {
        const int i = w.vinst[v];
        const batch::Inst I = w.inst[i];
        float *x = w.Xf + (size_t)v * 16;
        const int64_t deg = w.off[v + 1] - w.off[v];
        const float mdeg = I.narcs > 0 ? (float)((double)I.narcs / (double)I.nv) : 1.f;
        x[0] = __fdiv_rn((float)deg, mdeg);
        x[1] = log1pf((float)deg);
        for (int j = 0; j < 8; ++j) {
            const double n = (double)I.nv;
            const double mu = w.stats[i * 16 + j] / n;
            const double var = fmax(w.stats[i * 16 + 8 + j] / n - mu * mu, 0.0);
            const float muf = (float)mu, sdf = (float)sqrt(var);
            x[2 + j] = __fdiv_rn(__fsub_rn(x[2 + j], muf), sdf > 0.f ? sdf : 1.f);
        }
        x[10] = __fdiv_rn((float)I.k, 64.f);
        for (int j = 11; j < 16; ++j) x[j] = 0.f;
    }
}

__global__ void k_to_input(const float *Xf, int nv, __nv_bfloat16 *X, int ldx) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        for (int j = 0; j < 16; ++j) X[(size_t)v * ldx + j] = __float2bfloat16_rn(Xf[(size_t)v * 16 + j]);
}

// Gate scores: per graph, the mean of the network's output column 8 over its vertices (double sums).
__global__ void k_gate_scores(const float *Z, const int32_t *vinst, int nv, double *score) {
    const int lane = threadIdx.x & 31;
    for (int v0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); v0 < nv; v0 += gridDim.x * blockDim.x) {
        const int v = v0 + lane;
        const int i = v < nv ? vinst[v] : -1;
        double x = v < nv ? (double)Z[(size_t)v * 16 + 8] : 0.0;
        const int i0 = __shfl_sync(DMOLP_FULL_MASK, i, 0);
        if (__all_sync(DMOLP_FULL_MASK, i == i0)) {
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(DMOLP_FULL_MASK, x, o);
            if (lane == 0) atomicAdd(&score[i0], x);
        } else if (i >= 0) {
            atomicAdd(&score[i], x);
        }
    }
}

// Upstream gradient of the gate loss: column 8 of vertex v gets g[graph of v], the other columns 0.
__global__ void k_gate_grad(const float *g, const int32_t *vinst, int nv, float *dZ) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)nv * 16;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i >> 4;
        dZ[i] = (i & 15) == 8 ? g[vinst[v]] : 0.f;
    }
}

// Proposal coordinates: random-walk features + the network's first 8 outputs (its residual); 16 wide, the
// upper 8 columns 0.
__global__ void k_coords(const float *__restrict__ Xf, const float *__restrict__ Z, int nv, float *__restrict__ P) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)nv * 16;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i >> 4;
        const int j = (int)(i & 15);
        P[i] = j < 8 ? __fadd_rn(Xf[v * 16 + 2 + j], Z[v * 16 + j]) : 0.f;
    }
}

// ------------------------------------------------------------------------------------ decoder
// Recursive inertial bisection of the proposal coordinates P (8 wide), one CTA per graph: every part with
// kp >= 2 labels splits (all parts of a level at once) into kl = kp/2 and kp - kl labels; the left child takes
// the floor(n * kl / kp) vertices with the smallest (projection, id) on the part's principal axis.  The axis:
// mean and covariance of the part in double (thread partials in a fixed order, then a fixed reduction
// tree), cyclic Jacobi on the 8x8 covariance by one thread, the eigenvector of the largest eigenvalue signed
// so that its largest-magnitude component is positive.  The selection is an MSD radix select over 64-bit keys
// (orderable float bits of the projection, id) with 6-bit digits, segmented by part.
constexpr int kDecThreads = 512;
constexpr int kDecDigits = 64;
constexpr int kPcaDims = 8;

// Eigen-decomposition of a symmetric 8x8 matrix (cyclic Jacobi, double); eigenvalues on the diagonal of A,
// eigenvectors in the columns of V.
__device__ void jacobi8(double (&A)[kPcaDims][kPcaDims], double (&V)[kPcaDims][kPcaDims]) {
    for (int i = 0; i < kPcaDims; ++i)
        for (int j = 0; j < kPcaDims; ++j) V[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < kPcaDims; ++p)
            for (int q = p + 1; q < kPcaDims; ++q) off += A[p][q] * A[p][q];
        if (off < 1e-30) break;
        for (int p = 0; p < kPcaDims; ++p)
            for (int q = p + 1; q < kPcaDims; ++q) {
                if (fabs(A[p][q]) < 1e-300) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
                for (int r = 0; r < kPcaDims; ++r) {
                    const double arp = A[r][p], arq = A[r][q];
                    A[r][p] = c * arp - sn * arq;
                    A[r][q] = sn * arp + c * arq;
                }
                for (int r = 0; r < kPcaDims; ++r) {
                    const double apr = A[p][r], aqr = A[q][r];
                    A[p][r] = c * apr - sn * aqr;
                    A[q][r] = sn * apr + c * aqr;
                }
                for (int r = 0; r < kPcaDims; ++r) {
                    const double vrp = V[r][p], vrq = V[r][q];
                    V[r][p] = c * vrp - sn * vrq;
                    V[r][q] = sn * vrp + c * vrq;
                }
            }
    }
}

__device__ __forceinline__ unsigned orderable(float x) {
    const unsigned u = __float_as_uint(x);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct DecSmem {
    int kp[64], dim[64], cnt[64], need[64], below[64], keep[64];
    double part[kDecThreads / 32][kPcaDims * kPcaDims];
    double mean[kPcaDims], axis[kPcaDims][2];  // principal axis of the current part, its mean
    int hist[64 * kDecDigits];
    int nact[2], open, inst, bad;
};

__device__ __forceinline__ int dec_push(int *ctr, bool pred) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(DMOLP_FULL_MASK, pred);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(ctr, __popc(m));
    base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
    return base + __popc(m & ((1u << lane) - 1));
}

__global__ void __launch_bounds__(kDecThreads) k_decode(DecodeWork w) {
    __shared__ DecSmem sm;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) sm.inst = atomicAdd(w.next, 1);
        __syncthreads();
        const int q = sm.inst;
        if (q >= w.ninst) break;
        const int ii = w.order[q];
        if (w.skip && w.skip[ii]) {  // the gate prefers phase-1 seeding: nothing to decode
            if (threadIdx.x == 0) w.status[ii] = 2;
            __syncthreads();
            continue;
        }
        const batch::Inst I = w.inst[ii];
        const int k = I.k, nv = I.nv, vb = (int)I.vbase;
        for (int p = threadIdx.x; p < 64; p += blockDim.x) sm.kp[p] = 0;
        if (threadIdx.x == 0) {
            sm.kp[0] = k;
            sm.bad = 0;
        }
        __syncthreads();
        for (int v = threadIdx.x; v < nv; v += blockDim.x) {
            w.label[vb + v] = 0;
            for (int d = 0; d < kPcaDims; ++d)
                if (!isfinite(w.Z[(size_t)(vb + v) * 16 + d])) sm.bad = 1;
        }
        __syncthreads();
        if (sm.bad || nv < k) {
            if (threadIdx.x == 0) w.status[ii] = 1;  // not usable: the caller falls back
            __syncthreads();
            continue;
        }
        for (int level = 0; level < 7; ++level) {
            // ---- per splitting part: vertex count, mean, covariance, principal axis (fixed-order double
            //      reductions, so the result does not depend on scheduling); Y = projection on the axis ----
            for (int p = threadIdx.x; p < 64; p += blockDim.x) sm.cnt[p] = 0;
            __syncthreads();
            for (int i0 = (int)(threadIdx.x & ~31u); i0 < nv; i0 += blockDim.x) {
                const int v = i0 + lane;
                int lo = v < nv ? w.label[vb + v] : -1;
                if (lo >= 0 && sm.kp[lo] < 2) lo = -1;
                const unsigned m = __match_any_sync(DMOLP_FULL_MASK, lo);
                if (lo >= 0 && lane == __ffs(m) - 1) atomicAdd(&sm.cnt[lo], __popc(m));
            }
            __syncthreads();
            for (int lo = 0; lo < 64; ++lo) {
                if (sm.kp[lo] < 2 || sm.cnt[lo] == 0) continue;  // block-uniform
                // mean of the part
                {
                    double acc[kPcaDims];
#pragma unroll
                    for (int d = 0; d < kPcaDims; ++d) acc[d] = 0.0;
                    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
                        if (w.label[vb + v] != lo) continue;
                        const float4 *z = reinterpret_cast<const float4 *>(w.Z + (size_t)(vb + v) * 16);
                        const float4 z0 = z[0], z1 = z[1];
                        const float x[kPcaDims] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
#pragma unroll
                        for (int d = 0; d < kPcaDims; ++d) acc[d] += (double)x[d];
                    }
#pragma unroll
                    for (int d = 0; d < kPcaDims; ++d) {
                        double y = acc[d];
                        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(DMOLP_FULL_MASK, y, o);
                        if (lane == 0) sm.part[wib][d] = y;
                    }
                    __syncthreads();
                    if (threadIdx.x < kPcaDims) {
                        double t = 0.0;
                        for (int ww = 0; ww < kDecThreads / 32; ++ww) t += sm.part[ww][threadIdx.x];
                        sm.mean[threadIdx.x] = t / (double)sm.cnt[lo];
                    }
                    __syncthreads();
                }
                // covariance (upper triangle, 36 entries), then the principal axis
                {
                    constexpr int kTri = kPcaDims * (kPcaDims + 1) / 2;
                    double acc[kTri];
#pragma unroll
                    for (int i = 0; i < kTri; ++i) acc[i] = 0.0;
                    double mu[kPcaDims];
#pragma unroll
                    for (int d = 0; d < kPcaDims; ++d) mu[d] = sm.mean[d];
                    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
                        if (w.label[vb + v] != lo) continue;
                        const float4 *z = reinterpret_cast<const float4 *>(w.Z + (size_t)(vb + v) * 16);
                        const float4 z0 = z[0], z1 = z[1];
                        const float xf[kPcaDims] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
                        double x[kPcaDims];
#pragma unroll
                        for (int d = 0; d < kPcaDims; ++d) x[d] = (double)xf[d] - mu[d];
                        int i = 0;
#pragma unroll
                        for (int a2 = 0; a2 < kPcaDims; ++a2)
#pragma unroll
                            for (int b2 = a2; b2 < kPcaDims; ++b2) acc[i++] += x[a2] * x[b2];
                    }
#pragma unroll
                    for (int i = 0; i < kTri; ++i) {
                        double y = acc[i];
                        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(DMOLP_FULL_MASK, y, o);
                        if (lane == 0) sm.part[wib][i] = y;
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) {
                        double A[kPcaDims][kPcaDims], V[kPcaDims][kPcaDims];
                        int i = 0;
                        for (int a2 = 0; a2 < kPcaDims; ++a2)
                            for (int b2 = a2; b2 < kPcaDims; ++b2, ++i) {
                                double t = 0.0;
                                for (int ww = 0; ww < kDecThreads / 32; ++ww) t += sm.part[ww][i];
                                A[a2][b2] = t;
                                A[b2][a2] = t;
                            }
                        jacobi8(A, V);
                        int bi = 0;  // largest eigenvalue, lowest index on ties
                        for (int r = 1; r < kPcaDims; ++r)
                            if (A[r][r] > A[bi][bi]) bi = r;
                        int mi = 0;
                        for (int r = 1; r < kPcaDims; ++r)
                            if (fabs(V[r][bi]) > fabs(V[mi][bi])) mi = r;
                        const double sg = V[mi][bi] < 0 ? -1.0 : 1.0;
                        for (int r = 0; r < kPcaDims; ++r) {
                            sm.axis[r][0] = sg * V[r][bi];
                            sm.axis[r][1] = sm.mean[r];
                        }
                    }
                    __syncthreads();
                }
                for (int v = threadIdx.x; v < nv; v += blockDim.x) {
                    if (w.label[vb + v] != lo) continue;
                    double y = 0.0;
                    for (int d = 0; d < kPcaDims; ++d)
                        y += ((double)w.Z[(size_t)(vb + v) * 16 + d] - sm.axis[d][1]) * sm.axis[d][0];
                    w.Y[(size_t)(vb + v) * 4] = (float)y;
                }
                __syncthreads();
            }
            if (threadIdx.x < 64) {
                const int p = threadIdx.x;
                sm.need[p] = 0;
                sm.dim[p] = 0;
                if (sm.kp[p] >= 2 && sm.cnt[p] > 0) sm.need[p] = (int)(((long long)sm.cnt[p] * (sm.kp[p] / 2)) / sm.kp[p]);
            }
            for (int i = threadIdx.x; i < 64 * kDecDigits; i += blockDim.x) sm.hist[i] = 0;
            if (threadIdx.x == 0) {
                int any = 0;
                for (int p = 0; p < 64; ++p) any |= sm.kp[p] >= 2;
                sm.open = any;
            }
            __syncthreads();
            if (!sm.open) break;
            // ---- select the need[p] smallest keys of each splitting part: selected -> l1 marks ----
            // l0 holds the active records; pass 0 runs over all vertices.  Selected vertices are flagged by
            // writing -1 - lo into label (restored to lo below); the rest move to lo + kl.
            int nlist = nv;
            const int32_t *list = nullptr;
            for (int pass = 0; pass < 11; ++pass) {
                const int shift = 64 - 6 * (pass + 1);
                const int sh = shift < 0 ? 0 : shift;
                const unsigned long long dmask = shift < 0 ? ((1ull << (6 + shift)) - 1) : 63ull;
                for (int i0 = (int)(threadIdx.x & ~31u); i0 < nlist; i0 += blockDim.x) {
                    const int i = i0 + lane;
                    int bin = -(lane + 1);
                    if (i < nlist) {
                        const int v = list ? list[i] : i;
                        const int lo = w.label[vb + v];
                        if (lo >= 0 && sm.kp[lo] >= 2 && sm.need[lo] > 0) {
                            const unsigned long long key =
                                ((unsigned long long)orderable(w.Y[(size_t)(vb + v) * 4 + sm.dim[lo]]) << 32) |
                                (unsigned)v;
                            bin = lo * kDecDigits + (int)((key >> sh) & dmask);
                        }
                    }
                    const unsigned m = __match_any_sync(DMOLP_FULL_MASK, bin);
                    if (bin >= 0 && lane == __ffs(m) - 1) atomicAdd(&sm.hist[bin], __popc(m));
                }
                if (threadIdx.x == 0) {
                    sm.open = 0;
                    sm.nact[pass & 1] = 0;
                }
                __syncthreads();
                for (int p = wib; p < 64; p += kDecThreads / 32) {
                    int *h = sm.hist + p * kDecDigits;
                    const int c0 = h[2 * lane], c1 = h[2 * lane + 1];
                    h[2 * lane] = 0;
                    h[2 * lane + 1] = 0;
                    const int sum = c0 + c1;
                    int incl = sum;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
                        if (lane >= o) incl += y;
                    }
                    const int total = __shfl_sync(DMOLP_FULL_MASK, incl, 31);
                    const int nd = sm.need[p];
                    __syncwarp();
                    if (sm.kp[p] < 2 || nd <= 0) {
                        if (lane == 0) {
                            sm.below[p] = 0;
                            sm.keep[p] = -1;
                        }
                    } else if (nd >= total) {
                        if (lane == 0) {
                            sm.below[p] = kDecDigits;
                            sm.keep[p] = -1;
                            sm.need[p] = 0;
                        }
                    } else {
                        const int ex0 = incl - sum, in0 = ex0 + c0, in1 = in0 + c1;
                        int d = -1, r = 0, cnt = 0;
                        if (ex0 < nd && nd <= in0) {
                            d = 2 * lane;
                            r = nd - ex0;
                            cnt = c0;
                        } else if (in0 < nd && nd <= in1) {
                            d = 2 * lane + 1;
                            r = nd - in0;
                            cnt = c1;
                        }
                        if (d >= 0) {
                            if (r == cnt) {
                                sm.below[p] = d + 1;
                                sm.keep[p] = -1;
                                sm.need[p] = 0;
                            } else {
                                sm.below[p] = d;
                                sm.keep[p] = d;
                                sm.need[p] = r;
                                atomicAdd(&sm.open, 1);
                            }
                        }
                    }
                }
                __syncthreads();
                int32_t *nxt = (pass & 1) ? w.l1 + vb : w.l0 + vb;
                for (int i0 = (int)(threadIdx.x & ~31u); i0 < nlist; i0 += blockDim.x) {
                    const int i = i0 + lane;
                    bool keepv = false;
                    int v = 0;
                    if (i < nlist) {
                        v = list ? list[i] : i;
                        const int lo = w.label[vb + v];
                        if (lo >= 0 && sm.kp[lo] >= 2) {
                            const unsigned long long key =
                                ((unsigned long long)orderable(w.Y[(size_t)(vb + v) * 4 + sm.dim[lo]]) << 32) |
                                (unsigned)v;
                            const int d = (int)((key >> sh) & dmask);
                            if (d < sm.below[lo]) w.label[vb + v] = -1 - lo;  // selected: stays in lo
                            else keepv = d == sm.keep[lo];
                        }
                    }
                    const int slot = dec_push(&sm.nact[pass & 1], keepv);
                    if (keepv) nxt[slot] = v;
                }
                __syncthreads();
                if (sm.open == 0) break;
                list = nxt;
                nlist = sm.nact[pass & 1];
                __syncthreads();
            }
            // ---- children: selected vertices keep lo, the others move to lo + kl ----
            for (int v = threadIdx.x; v < nv; v += blockDim.x) {
                const int lo = w.label[vb + v];
                if (lo < 0) w.label[vb + v] = -1 - lo;
                else if (sm.kp[lo] >= 2) w.label[vb + v] = lo + sm.kp[lo] / 2;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int nk[64];
                for (int p = 0; p < 64; ++p) nk[p] = 0;
                for (int p = 0; p < 64; ++p) {
                    const int kp = sm.kp[p];
                    if (kp >= 2) {
                        nk[p] = kp / 2;
                        nk[p + kp / 2] = kp - kp / 2;
                    } else if (kp == 1) {
                        nk[p] = 1;
                    }
                }
                for (int p = 0; p < 64; ++p) sm.kp[p] = nk[p];
            }
            __syncthreads();
        }
        // ---- usable only if no part ended empty ----
        for (int p = threadIdx.x; p < 64; p += blockDim.x) sm.cnt[p] = 0;
        __syncthreads();
        for (int v = threadIdx.x; v < nv; v += blockDim.x) atomicAdd(&sm.cnt[w.label[vb + v]], 1);
        __syncthreads();
        if (threadIdx.x == 0) {
            int st = 0;
            for (int p = 0; p < k; ++p) st |= sm.cnt[p] == 0;
            w.status[ii] = st;
        }
        __syncthreads();
    }
}

template <int N, int KT>
void launch_gemm(const GemmArgs &g, int num_sms, cudaStream_t s) {
    const size_t smem = (size_t)(128 + N) * KT * 2;
    const int items = g.kind == kBwdWeight ? (g.rows + g.chunk - 1) / g.chunk : (g.rows + 127) / 128;
    const int grid = std::max(1, std::min(items, num_sms * 4));
    k_gemm<N, KT><<<grid, 128, smem, s>>>(g);
}

inline int grid_for(int64_t n, int num_sms) {
    const int64_t b = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)num_sms * 16));
}

}  // namespace

void gemm(const GemmArgs &g, int n, int kt, int num_sms, cudaStream_t s) {
    if (n == 64 && kt == 32) launch_gemm<64, 32>(g, num_sms, s);
    else if (n == 64 && kt == 64) launch_gemm<64, 64>(g, num_sms, s);
    else if (n == 16 && kt == 64) launch_gemm<16, 64>(g, num_sms, s);
    else if (n == 128 && kt == 16) launch_gemm<128, 16>(g, num_sms, s);
    else if (n == 128 && kt == 64) launch_gemm<128, 64>(g, num_sms, s);
}

void agg_fwd(const int64_t *off, const int32_t *col, int nv, __nv_bfloat16 *buf, int C, int num_sms, cudaStream_t s) {
    const int per_warp = C == 16 ? 4 : 1;
    const int64_t warps = ((int64_t)nv + per_warp - 1) / per_warp;
    const int grid = grid_for(warps * 32, num_sms);
    if (C == 16) k_agg_fwd<16><<<grid, 256, 0, s>>>(off, col, nv, buf);
    else k_agg_fwd<64><<<grid, 256, 0, s>>>(off, col, nv, buf);
}

void agg_bwd(const int64_t *off, const int32_t *col, int nv, const float *dC, const __nv_bfloat16 *Hbuf, int ldh,
             __nv_bfloat16 *G, float *db, int num_sms, cudaStream_t s) {
    k_agg_bwd<<<grid_for((int64_t)nv * 32, num_sms), 256, 0, s>>>(off, col, nv, dC, Hbuf, ldh, G, db);
}

void loss(const int64_t *off, const int32_t *col, int nv, const float *Z, const int32_t *target, double inv_arcs,
          __nv_bfloat16 *G, float *db, double *loss_sum, int num_sms, cudaStream_t s) {
    k_loss<<<grid_for((int64_t)nv * 4, num_sms), 256, 0, s>>>(off, col, nv, Z, target, (float)(2.0 * inv_arcs), G,
                                                             db, loss_sum);
}

void grad_out(const float *dZ, int nv, __nv_bfloat16 *G, float *db, int num_sms, cudaStream_t s) {
    k_grad_out<<<grid_for((int64_t)nv * 16, num_sms), 256, 0, s>>>(dZ, nv, G, db);
}

void adam(float *p, const float *g, float *m, float *v, int n, float lr, int step, cudaStream_t s) {
    const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, s>>>(p, g, m, v, n, lr, c1, c2);
}

void cast_weights(const float *params, __nv_bfloat16 *const W[3], __nv_bfloat16 *const Wt[3], cudaStream_t s) {
    k_cast<<<32, 256, 0, s>>>(params, W[0], W[1], W[2], Wt[0], Wt[1], Wt[2]);
}

constexpr int kBfsChunk = 64;  // BFS levels launched between two looks at the frontier size

int features(const FeatWork &w, int num_sms, cudaStream_t s) {
    const int g = grid_for(w.nv, num_sms);
    k_vinst<<<g, 256, 0, s>>>(w.inst, w.ninst, w.nv, w.vinst);
    cudaMemsetAsync(w.akey, 0, sizeof(unsigned long long) * w.ninst, s);
    cudaMemsetAsync(w.ecc, 0, sizeof(int32_t) * w.ninst, s);
    cudaMemsetAsync(w.stats, 0, sizeof(double) * 16 * w.ninst, s);
    cudaMemsetAsync(w.Xf, 0, sizeof(float) * 16 * (size_t)w.nv, s);
    for (int j = 0; j < kAnchors; ++j) {
        k_anchor_key<<<g, 256, 0, s>>>(w, j);
        k_fill_i32<<<g, 256, 0, s>>>(w.dist, w.nv, -1);
        cudaMemsetAsync(w.cnt, 0, 4 * sizeof(int), s);
        k_anchor_pick<<<(w.ninst + 255) / 256, 256, 0, s>>>(w, j);
        // levels in chunks of kBfsChunk launches; the host looks at the frontier once per chunk
        const int gb = num_sms * 16;
        for (int level = 0;; level += kBfsChunk) {
            for (int l = level; l < level + kBfsChunk; ++l)
                k_bfs_level<<<gb, 256, 0, s>>>(w.off, w.col, w.dist, (l & 1) ? w.front1 : w.front0,
                                               (l & 1) ? w.front0 : w.front1, w.cnt, l);
            int h = 0;
            cudaMemcpyAsync(&h, w.cnt + (level + kBfsChunk) % 3, sizeof(int), cudaMemcpyDeviceToHost, s);
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return (int)e;
            if (h == 0) break;
        }
        k_mind<<<g, 256, 0, s>>>(w, j);
    }
    int tmax = 0;
    {
        std::vector<int32_t> ecc(w.ninst);
        cudaMemcpyAsync(ecc.data(), w.ecc, sizeof(int32_t) * w.ninst, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return (int)e;
        for (int x : ecc) tmax = std::max(tmax, std::min(std::max(x, 1), kTMax));
    }
    k_rw_init<<<g, 256, 0, s>>>(w);
    float *P = w.P0, *Q = w.Q0, *P2 = w.P1, *Q2 = w.Q1;
    for (int t = 0; t < tmax; ++t) {
        k_rw_step<<<g, 256, 0, s>>>(w, P, Q, P2, Q2, t);
        std::swap(P, P2);
        std::swap(Q, Q2);
    }
    k_rw_log<<<g, 256, 0, s>>>(w);
    k_feat_final<<<g, 256, 0, s>>>(w);
    if (w.X) k_to_input<<<g, 256, 0, s>>>(w.Xf, w.nv, w.X, w.ldx);
    return (int)cudaGetLastError();
}

void features_to_input(const float *Xf, int nv, __nv_bfloat16 *X, int ldx, cudaStream_t s) {
    k_to_input<<<grid_for(nv, 148), 256, 0, s>>>(Xf, nv, X, ldx);
}

void gate_scores(const float *Z, const int32_t *vinst, int nv, double *score, int num_sms, cudaStream_t s) {
    k_gate_scores<<<grid_for(nv, num_sms), 256, 0, s>>>(Z, vinst, nv, score);
}

void gate_grad(const float *g, const int32_t *vinst, int nv, float *dZ, int num_sms, cudaStream_t s) {
    k_gate_grad<<<grid_for((int64_t)nv * 16, num_sms), 256, 0, s>>>(g, vinst, nv, dZ);
}

void coords(const float *Xf, const float *Z, int nv, float *P, int num_sms, cudaStream_t s) {
    k_coords<<<grid_for((int64_t)nv * 16, num_sms), 256, 0, s>>>(Xf, Z, nv, P);
}

void decode(const DecodeWork &w, int grid, cudaStream_t s) {
    cudaMemsetAsync(w.next, 0, sizeof(int), s);
    k_decode<<<grid, kDecThreads, 0, s>>>(w);
}

}  // namespace mpnn
}  // namespace dmolp
