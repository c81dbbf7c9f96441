// Device helpers shared by the single-graph LP kernels and the batched LP kernel.
#pragma once

#include <cfloat>

#include "device_state.cuh"

namespace dmolp {

// Decision class of a selected vertex: 0 thread (short row, own label scored, at most kDecSmallK labels),
// 1 warp, 2 hub (row split into chunks).  A vertex whose own label is not scored goes to the warp class,
// whose histogram also sees absent labels.
__device__ __forceinline__ int dec_class(int deg, int own, int eff) {
    if (deg > kLargeDeg) return 2;
    return (deg > kDecSmall || (unsigned)own >= (unsigned)eff || eff > kDecSmallK) ? 1 : 0;
}

// SplitMix64 finaliser of a vertex id: summed over a window it gives an order-independent checksum of the
// set (the oracle and the reference harness report the same sum).
__device__ __forceinline__ unsigned long long window_mix(int v) {
    unsigned long long z = (unsigned long long)(unsigned)v + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ int tiekey(int c) { return (c & ~31) | (int)brev5((unsigned)c & 31u); }

__device__ __forceinline__ long long sll(unsigned long long x) { return (long long)x; }

// Better (score desc, tie key asc).
__device__ __forceinline__ bool better(double s, int key, double bs, int bkey) {
    return s > bs || (s == bs && key < bkey);
}

// Visit neighbour ids col[s..e) with the lanes of a warp: scalar head up to a 16-byte boundary, 128-bit
// loads for the body, scalar tail.  f(u) is called per neighbour; after each step `stop()` (evaluated
// warp-uniformly) may end the walk early.  Returns the number of arcs the warp read.
template <typename F, typename S>
__device__ __forceinline__ int64_t warp_row(const int32_t *__restrict__ col, int64_t s, int64_t e, int lane, F f,
                                            S stop) {
    int64_t a = (s + 3) & ~int64_t(3);
    if (a > e) a = e;
    if (s + lane < a) f(__ldg(col + s + lane));
    int64_t read = a - s;
    if (stop()) return read;
    const int64_t qe = e >> 2;  // body: int4 words [a/4, e/4)
    const int4 *c4 = reinterpret_cast<const int4 *>(col);
    for (int64_t q = (a >> 2) + lane, q0 = a >> 2; q0 < qe; q += 32, q0 += 32) {
        if (q < qe) {
            const int4 x = __ldcs(c4 + q);
            f(x.x);
            f(x.y);
            f(x.z);
            f(x.w);
        }
        read += 4 * (qe - q0 < 32 ? qe - q0 : (int64_t)32);
        if (stop()) return read;
    }
    const int64_t t0 = a > (qe << 2) ? a : (qe << 2);
    if (t0 + lane < e) f(__ldg(col + t0 + lane));
    return read + (e - t0);
}

// The arcs [s, e) of a row visited by the lanes of a warp with many loads in flight: each step loads, per
// lane, the row's scalar head and tail (first step only) and two 16-byte words of its body, then gathers
// g(u) for all of them, then calls f(u, g(u)) for each, so a row of up to 262 arcs costs one dependent
// load pair.  After each step stop() (evaluated warp-uniformly) may end the walk.  Returns the number of
// arcs the warp read.  Entries are ids (>= 0) or, in the hot-encoded rows, -(rank + 2); kNoArc marks an
// empty slot.
constexpr int kNoArc = -1;
template <typename G, typename F, typename S>
__device__ __forceinline__ int64_t warp_row_wide(const int32_t *__restrict__ col, int64_t s, int64_t e, int lane,
                                                 G g, F f, S stop) {
    int64_t a = (s + 3) & ~int64_t(3);
    if (a > e) a = e;
    const int64_t qe = e >> 2;  // body: int4 words [a/4, e/4)
    const int64_t t0 = a > (qe << 2) ? a : (qe << 2);
    const int4 *c4 = reinterpret_cast<const int4 *>(col);
    int64_t read = (a - s) + (e - t0);
    bool first = true;
    for (int64_t q0 = a >> 2; first || q0 < qe; q0 += 64) {
        int u[10];
        u[8] = first && s + lane < a ? __ldg(col + s + lane) : kNoArc;
        u[9] = first && t0 + lane < e ? __ldg(col + t0 + lane) : kNoArc;
        const int64_t q = q0 + lane;
        int4 x = make_int4(kNoArc, kNoArc, kNoArc, kNoArc), y = x;
        if (q < qe) x = __ldcs(c4 + q);
        if (q + 32 < qe) y = __ldcs(c4 + q + 32);
        u[0] = x.x; u[1] = x.y; u[2] = x.z; u[3] = x.w;
        u[4] = y.x; u[5] = y.y; u[6] = y.z; u[7] = y.w;
        decltype(g(0)) v[10];
#pragma unroll
        for (int r = 0; r < 10; ++r)
            if (u[r] != kNoArc) v[r] = g(u[r]);
#pragma unroll
        for (int r = 0; r < 10; ++r)
            if (u[r] != kNoArc) f(u[r], v[r]);
        if (q0 < qe) read += 4 * (qe - q0 < 64 ? qe - q0 : (int64_t)64);
        first = false;
        if (stop()) break;
    }
    return read;
}

// The same walk with f(u, value) called on every lane for every slot of a step, empty slots included
// (u == kNoArc, value = none), so that f may take warp-wide votes.  No early stop.
template <typename T, typename G, typename F>
__device__ __forceinline__ void warp_row_wide_all(const int32_t *__restrict__ col, int64_t s, int64_t e, int lane,
                                                  T none, G g, F f) {
    int64_t a = (s + 3) & ~int64_t(3);
    if (a > e) a = e;
    const int64_t qe = e >> 2;
    const int64_t t0 = a > (qe << 2) ? a : (qe << 2);
    const int4 *c4 = reinterpret_cast<const int4 *>(col);
    bool first = true;
    for (int64_t q0 = a >> 2; first || q0 < qe; q0 += 64) {
        int u[10];
        u[8] = first && s + lane < a ? __ldg(col + s + lane) : kNoArc;
        u[9] = first && t0 + lane < e ? __ldg(col + t0 + lane) : kNoArc;
        const int64_t q = q0 + lane;
        int4 x = make_int4(kNoArc, kNoArc, kNoArc, kNoArc), y = x;
        if (q < qe) x = __ldcs(c4 + q);
        if (q + 32 < qe) y = __ldcs(c4 + q + 32);
        u[0] = x.x; u[1] = x.y; u[2] = x.z; u[3] = x.w;
        u[4] = y.x; u[5] = y.y; u[6] = y.z; u[7] = y.w;
        T v[10];
#pragma unroll
        for (int r = 0; r < 10; ++r) v[r] = u[r] != kNoArc ? g(u[r]) : none;
#pragma unroll
        for (int r = 0; r < 10; ++r) f(u[r], v[r]);
        first = false;
    }
}

// Lane-private label counters of one warp for labels < 32: lane L counts label c in
// h[c*32 + ((L + c) & 31)].  Increments need no atomics and hit distinct banks for lanes sharing a label;
// the sum over row c (lane c, rotated start) is bank-conflict free as well.
__device__ __forceinline__ void priv_zero(int *h, int eff, int lane) {
    for (int c = 0; c < eff; ++c) h[c * 32 + ((lane + c) & 31)] = 0;
}
__device__ __forceinline__ int priv_total(const int *h, int eff, int lane) {
    int t = 0;
    if (lane < eff)
        for (int j = 0; j < 32; ++j) t += h[lane * 32 + ((j + lane) & 31)];
    return t;
}

// Count labels < eff of the arcs [s, e) into the calling warp's histogram: lane-private counters (eff <= 32,
// h has 32*32 ints) or a shared histogram h[eff] with one atomic per group of equal labels (__match_any).
__device__ __forceinline__ int64_t warp_count(const int32_t *__restrict__ col, const int32_t *__restrict__ label,
                                              int64_t s, int64_t e, int lane, int eff, int *h) {
    if (eff <= 32) {
        return warp_row(col, s, e, lane, [&](int u) {
            const int lu = label[u];
            if ((unsigned)lu < (unsigned)eff) h[lu * 32 + ((lane + lu) & 31)] += 1;
        }, [] { return false; });
    }
    for (int64_t j0 = s; j0 < e; j0 += 32) {
        const int64_t j = j0 + lane;
        const int lu = j < e ? label[__ldcs(col + j)] : -1;
        const bool ok = (unsigned)lu < (unsigned)eff;
        const unsigned m = __match_any_sync(DMOLP_FULL_MASK, ok ? lu : -(lane + 1));
        if (ok && lane == __ffs(m) - 1) atomicAdd(&h[lu], __popc(m));
    }
    return e - s;
}

// Warp argmax over labels < eff given per-label counts: lanes hold the counts of labels lane, lane+32, ...
// through cnt_of(c).  Returns (best score, best label) in every lane; (score desc, tie key asc).
template <typename C>
__device__ __forceinline__ void warp_argmax(int eff, const double *tpen, int lane, C cnt_of, double &best,
                                            int &blab) {
    best = -DBL_MAX;
    int bkey = 0x7fffffff;
    blab = -1;
    for (int c = lane; c < eff; c += 32) {
        const int cnt = cnt_of(c);
        const double sc = cnt > 0 ? __dmul_rn((double)cnt, tpen[c]) : 0.0;
        const int key = tiekey(c);
        if (better(sc, key, best, bkey)) {
            best = sc;
            bkey = key;
            blab = c;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(DMOLP_FULL_MASK, best, o);
        const int ok = __shfl_xor_sync(DMOLP_FULL_MASK, bkey, o);
        const int ol = __shfl_xor_sync(DMOLP_FULL_MASK, blab, o);
        if (better(ob, ok, best, bkey)) {
            best = ob;
            bkey = ok;
            blab = ol;
        }
    }
}

// calculatePenalties (src/phase2/phase2.cpp:158-209) by one warp, with the reference's operation order:
// per-part ratios and penalties in parallel, the means and variances summed in part order by lane 0.
// vc_of(p) = vertices of part p, ec_of(p) = its intra-part edges (arcs / 2); logt = log(iteration).
// Writes RE[p] and tpen[p] = 1 + penalty[p] (the kernel's score factor), and penalty[p] to pen_out if given.
template <typename VC, typename EC>
__device__ __forceinline__ void warp_penalties(int k, VC vc_of, EC ec_of, double logt, double *RE, double *tpen,
                                               double *pen_out) {
    const int lane = threadIdx.x & 31;
    long long tv = 0, te = 0;
    for (int p = lane; p < k; p += 32) {
        tv += vc_of(p);
        te += ec_of(p);
    }
    for (int o = 16; o > 0; o >>= 1) {
        tv += __shfl_xor_sync(DMOLP_FULL_MASK, tv, o);
        te += __shfl_xor_sync(DMOLP_FULL_MASK, te, o);
    }
    const double ev = __ddiv_rn((double)tv, (double)k);
    const double ee = te > 0 ? __ddiv_rn((double)te, (double)k) : 1.0;
    for (int p = lane; p < k; p += 32) {
        RE[p] = ee > 0 ? __ddiv_rn((double)ec_of(p), ee) : 1.0;
        tpen[p] = ev > 0 ? __ddiv_rn((double)vc_of(p), ev) : 1.0;  // RV until the penalties overwrite it
    }
    __syncwarp();
    double imb_rv = 0.0, imb_re = 0.0;
    if (lane == 0) {
        double rv_mean = 0.0, re_mean = 0.0;
        for (int p = 0; p < k; ++p) {
            rv_mean = __dadd_rn(rv_mean, tpen[p]);
            re_mean = __dadd_rn(re_mean, RE[p]);
        }
        rv_mean = __ddiv_rn(rv_mean, (double)k);
        re_mean = __ddiv_rn(re_mean, (double)k);
        double rv_var = 0.0, re_var = 0.0;
        for (int p = 0; p < k; ++p) {
            const double dv = __dsub_rn(tpen[p], rv_mean), de = __dsub_rn(RE[p], re_mean);
            rv_var = __dadd_rn(rv_var, __dmul_rn(dv, dv));
            re_var = __dadd_rn(re_var, __dmul_rn(de, de));
        }
        rv_var = __ddiv_rn(rv_var, (double)k);
        re_var = __ddiv_rn(re_var, (double)k);
        const double total_var = __dadd_rn(rv_var, re_var);
        imb_rv = total_var > 0 ? __ddiv_rn(rv_var, total_var) : 0.0;
        imb_re = total_var > 0 ? __ddiv_rn(re_var, total_var) : 0.0;
    }
    imb_rv = __shfl_sync(DMOLP_FULL_MASK, imb_rv, 0);
    imb_re = __shfl_sync(DMOLP_FULL_MASK, imb_re, 0);
    const double g = __dadd_rn(1.0, logt);
    for (int p = lane; p < k; p += 32) {
        const double grv = __dmul_rn(__dsub_rn(1.0, tpen[p]), g);
        const double gre = __dmul_rn(__dsub_rn(1.0, RE[p]), g);
        const double pen = __dadd_rn(__dmul_rn(imb_rv, grv), __dmul_rn(imb_re, gre));
        if (pen_out) pen_out[p] = pen;
        tpen[p] = __dadd_rn(1.0, pen);
    }
    __syncwarp();
}

}  // namespace dmolp
