// Batched boundary label propagation: thousands of independent partition instances in one persistent
// launch, replayed from a captured CUDA graph.
//
// Each instance is one graph of the batch (its vertices are a contiguous range of the batch's union CSR)
// with its own part count k <= 64.  A CTA takes the next instance from a global queue (largest first) and
// runs the whole phase-2 loop of src/phase2/phase2.cpp:256-449 on it -- penalties, candidate marking,
// boundary test, per-label window selection, decisions, incremental cut / balance update, stopping rules --
// with block barriers between the steps, then takes the next instance.  The per-instance arithmetic is the
// single-graph path's: the same penalties (warp_penalties), the same selection keys (degree ascending, or
// max-degree minus degree when RE > 1, then the vertex's id within its graph), the same decision rule and
// tie order, so every instance ends bit-identical to a single-graph run of the same graph and labels.
//
// Work inside a CTA is scheduled per warp: a warp takes 32 list entries; rows of at most TD arcs are walked
// by their own lane, longer rows (and vertices whose own label is not scored) by the whole warp, one after
// another.  The window selection is an MSD radix select over the instance's boundary list with 6-bit
// digits and one shared-memory histogram of k x 64 counters.  Block size NT, the thread-row limit TD and
// the number of resident CTAs per SM are the autotuned shape.
#include <cfloat>

#include "batch.cuh"
#include "lp_device.cuh"

namespace dmolp {
namespace batch {
namespace {

constexpr int kDigitBits = 6;
constexpr int kDigits = 1 << kDigitBits;

template <int NT>
struct Smem {
    long long vc[kBatchMaxK], intra[kBatchMaxK];
    double tpen[kBatchMaxK], RE[kBatchMaxK];
    int bcnt[kBatchMaxK], need[kBatchMaxK], below[kBatchMaxK], keep[kBatchMaxK];
    int hist[kBatchMaxK * kDigits];
    int whist[NT / 32][kBatchMaxK];
    int ncand, nbnd, nwin, nmov, nact[2], open, bad, inst;
    unsigned long long te_cand, te_sel, arcs, visits;
    long long cut_arcs, dcut;
};

__device__ __forceinline__ int warp_push(int *ctr, bool pred) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(DMOLP_FULL_MASK, pred);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(ctr, __popc(m));
    base = __shfl_sync(DMOLP_FULL_MASK, base, 0);
    return base + __popc(m & ((1u << lane) - 1));
}

// Visit the n vertices vid(i), i in [0, n).  Every thread of the block calls it.  small(active, v, s, e) is
// called by all lanes of a warp (active marks the lanes that own a short row); rows with is_big(v, s, e)
// are passed one by one to wide(v, s, e), called by the whole warp.
template <typename Vid, typename Big, typename Small, typename Wide>
__device__ __forceinline__ void visit(const Args &a, int n, Vid vid, Big is_big, Small small, Wide wide) {
    const int lane = threadIdx.x & 31;
    for (int i0 = (int)(threadIdx.x & ~31u); i0 < n; i0 += blockDim.x) {
        const int i = i0 + lane;
        int v = -1;
        int64_t s = 0, e = 0;
        if (i < n) {
            v = vid(i);
            s = a.off[v];
            e = a.off[v + 1];
        }
        const bool big = v >= 0 && is_big(v, s, e);
        small(v >= 0 && !big, v, s, e);
        unsigned m = __ballot_sync(DMOLP_FULL_MASK, big);
        while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            wide(__shfl_sync(DMOLP_FULL_MASK, v, l), __shfl_sync(DMOLP_FULL_MASK, s, l),
                 __shfl_sync(DMOLP_FULL_MASK, e, l));
        }
    }
}

__device__ __forceinline__ long long block_sum_into(long long x, long long *dst) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(DMOLP_FULL_MASK, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd((unsigned long long *)dst, (unsigned long long)x);
    return x;
}

// Label counts and same-label / cut arcs of the instance's current labels (phase2.cpp:55-117, 214-253).
template <int NT, int TD>
__device__ void full_stats(const Args &a, const Inst &I, Smem<NT> &sm) {
    const int lane = threadIdx.x & 31;
    long long cut = 0;
    int bad = 0;
    visit(a, I.nv, [&](int i) { return (int)I.vbase + i; },
          [&](int, int64_t s, int64_t e) { return e - s > TD; },
          [&](bool act, int v, int64_t s, int64_t e) {
              if (!act) return;
              const int lv = a.label[v];
              if ((unsigned)lv >= (unsigned)I.k) {
                  bad = 1;
                  return;
              }
              int same = 0, diff = 0;
              for (int64_t j = s; j < e; ++j) {
                  const int lu = a.label[__ldg(a.col + j)];
                  same += lu == lv;
                  diff += lu != lv;
              }
              atomicAdd((unsigned long long *)&sm.vc[lv], 1ull);
              if (same) atomicAdd((unsigned long long *)&sm.intra[lv], (unsigned long long)same);
              cut += diff;
              a.ndiff[v] = diff;
          },
          [&](int v, int64_t s, int64_t e) {
              const int lv = a.label[v];
              int same = 0, diff = 0;
              warp_row(a.col, s, e, lane, [&](int u) {
                  const int lu = a.label[u];
                  same += lu == lv;
                  diff += lu != lv;
              }, [] { return false; });
              for (int o = 16; o > 0; o >>= 1) {
                  same += __shfl_xor_sync(DMOLP_FULL_MASK, same, o);
                  diff += __shfl_xor_sync(DMOLP_FULL_MASK, diff, o);
              }
              if (lane == 0) {
                  if ((unsigned)lv >= (unsigned)I.k) {
                      bad = 1;
                  } else {
                      atomicAdd((unsigned long long *)&sm.vc[lv], 1ull);
                      if (same) atomicAdd((unsigned long long *)&sm.intra[lv], (unsigned long long)same);
                      cut += diff;
                      a.ndiff[v] = diff;
                  }
              }
          });
    block_sum_into(cut, &sm.cut_arcs);
    if (__any_sync(DMOLP_FULL_MASK, bad) && lane == 0) sm.bad = 1;
}

// Selection key of a boundary vertex (as the single-graph path's sel_key, with the id inside its graph).
__device__ __forceinline__ uint64_t key_of(const Inst &I, bool desc, int deg, int v) {
    const uint64_t dk = desc ? (uint64_t)(I.maxdeg - deg) : (uint64_t)deg;
    return (dk << I.ibits) | (uint64_t)(v - (int)I.vbase);
}

template <int NT, int TD>
__device__ void run_instance(const Args &a, const int ii, Smem<NT> &sm) {
    const Inst I = a.inst[ii];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int k = I.k;
    const int eff = a.cap == DMOLP_LP_CAP_FULL ? k : (k < 32 ? k : 32);
    const int stamp0 = *a.stamp_base;
    int32_t *const cand = a.l_cand + I.vbase, *const bnd = a.l_bnd + I.vbase;
    int32_t *const act[2] = {a.l_cand + I.vbase, a.l_act + I.vbase};  // cand is dead once bnd is built
    int32_t *const win[2] = {a.l_win0 + I.vbase, a.l_win1 + I.vbase};
    int32_t *const mov = a.l_bnd + I.vbase;  // bnd is dead once the window is selected
    const int npass_raw = (I.dbits + I.ibits + kDigitBits - 1) / kDigitBits;
    const int npass = npass_raw > 0 ? npass_raw : 1;
    const int top = npass * kDigitBits;

    for (int p = threadIdx.x; p < k; p += blockDim.x) sm.vc[p] = sm.intra[p] = 0;
    if (threadIdx.x == 0) {
        sm.cut_arcs = 0;
        sm.bad = 0;
    }
    __syncthreads();
    full_stats<NT, TD>(a, I, sm);
    __syncthreads();
    Out o;
    o.edge_cut = sm.cut_arcs >> 1;
    o.te = o.arcs = o.visits = 0;
    o.iterations = o.stop_reason = o.changes = 0;
    o.status = (sm.bad || (sm.cut_arcs & 1)) ? DMOLP_ERR_BAD_LABELS : DMOLP_OK;
    const int max_iter = a.mode == DMOLP_LP_MODE_REF ? kMaxIter : a.iters;
    long long prev_cut = o.edge_cut;
    int conv = 0;
    unsigned long long te_prev_next = (unsigned long long)I.narcs;
    int nprev = I.nv;
    for (int t = 1; o.status == DMOLP_OK && t <= max_iter; ++t) {
        const int st = stamp0 + t;
        // ---- penalties (phase2.cpp:158-209) and per-iteration counters ----
        if (wib == 0)
            warp_penalties(k, [&](int p) { return sm.vc[p]; }, [&](int p) { return sm.intra[p] / 2; }, a.logtab[t],
                           sm.RE, sm.tpen, nullptr);
        for (int p = threadIdx.x; p < k; p += blockDim.x) sm.bcnt[p] = 0;
        for (int i = threadIdx.x; i < k * kDigits; i += blockDim.x) sm.hist[i] = 0;
        if (threadIdx.x == 32) {
            sm.ncand = sm.nbnd = sm.nwin = sm.nmov = 0;
            sm.te_cand = sm.te_sel = 0;
            sm.dcut = 0;
        }
        __syncthreads();
        const unsigned long long te_prev = te_prev_next;
        unsigned long long arcs = 0, visits = 0;
        // ---- candidates = previous window and its neighbours (gpu_lp_boundary.cu:196-214) ----
        if (t > 1) {
            const int32_t *prev = win[(t - 1) & 1];
            auto mark = [&](int u) {
                if (a.cstamp[u] != st && atomicExch(&a.cstamp[u], st) != st) cand[atomicAdd(&sm.ncand, 1)] = u;
            };
            visit(a, nprev, [&](int i) { return prev[i]; }, [&](int, int64_t s, int64_t e) { return e - s > TD; },
                  [&](bool act, int v, int64_t s, int64_t e) {
                      if (!act) return;
                      ++visits;
                      mark(v);
                      for (int64_t j = s; j < e; ++j) mark(__ldg(a.col + j));
                      arcs += (unsigned long long)(e - s);
                  },
                  [&](int v, int64_t s, int64_t e) {
                      if (lane == 0) {
                          ++visits;
                          mark(v);
                          arcs += (unsigned long long)(e - s);
                      }
                      warp_row(a.col, s, e, lane, mark, [] { return false; });
                  });
            __syncthreads();
        }
        // ---- boundary test: a neighbour with another label (gpu_lp_boundary.cu:216-236), i.e. ndiff > 0 ----
        {
            const int n = t == 1 ? I.nv : sm.ncand;
            unsigned long long tec = 0;
            for (int i0 = (int)(threadIdx.x & ~31u); i0 < n; i0 += blockDim.x) {
                const int i = i0 + lane;
                bool isb = false;
                int own = 0, v = 0;
                if (i < n) {
                    v = t == 1 ? (int)I.vbase + i : cand[i];
                    tec += (unsigned long long)(a.off[v + 1] - a.off[v]);
                    ++visits;
                    if (a.ndiff[v] > 0) {
                        isb = true;
                        own = a.label[v];
                    }
                }
                const int slot = warp_push(&sm.nbnd, isb);
                if (isb) {
                    bnd[slot] = v;
                    atomicAdd(&sm.bcnt[own], 1);
                }
            }
            tec = warp_sum_u64(tec);
            if (lane == 0 && tec) atomicAdd(&sm.te_cand, tec);
        }
        __syncthreads();
        // ---- per label keep ceil(e^(-t/5) * n_p) (gpu_lp_boundary.cu:238-300) ----
        {
            const double ratio = a.ratiotab[t];
            for (int p = threadIdx.x; p < k; p += blockDim.x) {
                const int n = sm.bcnt[p];
                const int m = (int)ceil(__dmul_rn(ratio, (double)n));
                sm.need[p] = m > n ? n : m;
            }
        }
        int32_t *const wout = win[t & 1];
        __syncthreads();
        int nlist = sm.nbnd;
        const int32_t *list = bnd;
        for (int pass = 0; pass < npass; ++pass) {
            const int shift = top - kDigitBits * (pass + 1);
            // histogram of the digit over the records of open labels
            for (int i0 = (int)(threadIdx.x & ~31u); i0 < nlist; i0 += blockDim.x) {
                const int i = i0 + lane;
                int bin = -(lane + 1);
                if (i < nlist) {
                    const int v = list[i];
                    const int p = a.label[v];
                    if (sm.need[p] > 0) {
                        const int deg = (int)(a.off[v + 1] - a.off[v]);
                        bin = p * kDigits + (int)((key_of(I, sm.RE[p] > 1.0, deg, v) >> shift) & (kDigits - 1));
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
            // per label: the digit where the running count crosses need (warp per label, 2 bins per lane)
            for (int p = wib; p < k; p += NT / 32) {
                int *h = sm.hist + p * kDigits;
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
                if (nd <= 0) {
                    if (lane == 0) {
                        sm.below[p] = 0;
                        sm.keep[p] = -1;
                    }
                } else if (nd >= total) {
                    if (lane == 0) {
                        sm.below[p] = kDigits;
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
            // records below the digit are selected; records on it stay for the next digit
            int32_t *const nxt = act[pass & 1];
            for (int i0 = (int)(threadIdx.x & ~31u); i0 < nlist; i0 += blockDim.x) {
                const int i = i0 + lane;
                bool take = false, keep = false;
                int v = 0;
                if (i < nlist) {
                    v = list[i];
                    const int p = a.label[v];
                    const int deg = (int)(a.off[v + 1] - a.off[v]);
                    const int d = (int)((key_of(I, sm.RE[p] > 1.0, deg, v) >> shift) & (kDigits - 1));
                    take = d < sm.below[p];
                    keep = d == sm.keep[p];
                }
                const int ws = warp_push(&sm.nwin, take);
                if (take) wout[ws] = v;
                const int ks = warp_push(&sm.nact[pass & 1], keep);
                if (keep) nxt[ks] = v;
            }
            __syncthreads();
            if (sm.open == 0) break;
            list = nxt;
            nlist = sm.nact[pass & 1];
            __syncthreads();  // nact of the next pass is reset by thread 0 only after everyone read it
        }
        const int nwin = sm.nwin;
        // ---- decisions for the window (boundaryLPKernel_unified, gpu_lp_boundary.cu:327-427) ----
        {
            unsigned long long tes = 0;
            int *h = sm.whist[wib];
            visit(a, nwin, [&](int i) { return wout[i]; },
                  [&](int v, int64_t s, int64_t e) { return e - s > TD || a.label[v] >= eff; },
                  [&](bool act, int v, int64_t s, int64_t e) {
                      int nl = -1;
                      if (act) {
                          const int own = a.label[v];
                          const int deg = (int)(e - s);
                          tes += (unsigned long long)deg;
                          arcs += (unsigned long long)deg;
                          ++visits;
                          int l[TD];
#pragma unroll
                          for (int j = 0; j < TD; ++j) l[j] = j < deg ? a.label[__ldg(a.col + s + j)] : -1;
                          int own_cnt = 0;
                          double best = -DBL_MAX;
                          int bkey = 0x7fffffff, blab = -1;
#pragma unroll
                          for (int j = 0; j < TD; ++j) {
                              own_cnt += (l[j] == own);
                              const int c = l[j];
                              if ((unsigned)c < (unsigned)eff) {
                                  int cnt = 0;
#pragma unroll
                                  for (int q = 0; q < TD; ++q) cnt += (l[q] == c);
                                  const double sc = __dmul_rn((double)cnt, sm.tpen[c]);
                                  const int key = tiekey(c);
                                  if (better(sc, key, best, bkey)) {
                                      best = sc;
                                      bkey = key;
                                      blab = c;
                                  }
                              }
                          }
                          if (blab >= 0 && best > (double)own_cnt && blab != own) nl = blab;
                      }
                      const int slot = warp_push(&sm.nmov, nl >= 0);
                      if (nl >= 0) {
                          a.newlab[v] = nl;
                          mov[slot] = v;
                      }
                  },
                  [&](int v, int64_t s, int64_t e) {
                      const int own = a.label[v];
                      for (int c = lane; c < eff; c += 32) h[c] = 0;
                      __syncwarp();
                      for (int64_t j0 = s; j0 < e; j0 += 32) {
                          const int64_t j = j0 + lane;
                          const int lu = j < e ? a.label[__ldg(a.col + j)] : -1;
                          const bool ok = (unsigned)lu < (unsigned)eff;
                          const unsigned m = __match_any_sync(DMOLP_FULL_MASK, ok ? lu : -(lane + 1));
                          if (ok && lane == __ffs(m) - 1) atomicAdd(&h[lu], __popc(m));
                      }
                      __syncwarp();
                      double best;
                      int blab;
                      warp_argmax(eff, sm.tpen, lane, [&](int c) { return h[c]; }, best, blab);
                      const double own_raw = (unsigned)own < (unsigned)eff ? (double)h[own] : -1e300;
                      __syncwarp();
                      if (lane == 0) {
                          tes += (unsigned long long)(e - s);
                          arcs += (unsigned long long)(e - s);
                          ++visits;
                          const int nl = best > own_raw ? blab : own;
                          if (nl != own) {
                              a.newlab[v] = nl;
                              mov[atomicAdd(&sm.nmov, 1)] = v;
                          }
                      }
                  });
            tes = warp_sum_u64(tes);
            if (lane == 0 && tes) atomicAdd(&sm.te_sel, tes);
        }
        __syncthreads();
        const int nmov = sm.nmov;
        // ---- incremental cut / balance update from the movers (symmetric graphs) ----
        if (I.symmetric && nmov > 0) {
            long long dcut = 0;
            // cut / intra counts, and the differently-labelled neighbour counts: arc (u,v) seen from u, arc
            // (v,u) from v when u stays (a moving u updates v's count from its own row)
            auto upd = [&](int v, int u, long long &dc, long long &in_c, long long &out_a, int &dv) {
                const int a0 = a.label[v], c = a.newlab[v];
                const int lo = a.label[u], nu = a.newlab[u];
                const int ln = nu >= 0 ? nu : lo;
                const int w = nu >= 0 ? 1 : 2;
                dc += w * ((int)(c != ln) - (int)(a0 != lo));
                in_c += w * (int)(c == ln);
                out_a += w * (int)(a0 == lo);
                const int du = (int)(ln != c) - (int)(lo != a0);
                if (du) atomicAdd(&a.ndiff[u], du);
                if (nu < 0) dv += (int)(c != lo) - (int)(a0 != lo);
            };
            visit(a, nmov, [&](int i) { return mov[i]; }, [&](int, int64_t s, int64_t e) { return e - s > TD; },
                  [&](bool act, int v, int64_t s, int64_t e) {
                      if (!act) return;
                      long long in_c = 0, out_a = 0;
                      int dv = 0;
                      for (int64_t j = s; j < e; ++j) upd(v, __ldg(a.col + j), dcut, in_c, out_a, dv);
                      if (dv) atomicAdd(&a.ndiff[v], dv);
                      arcs += (unsigned long long)(e - s);
                      ++visits;
                      const int a0 = a.label[v], c = a.newlab[v];
                      atomicAdd((unsigned long long *)&sm.vc[a0], (unsigned long long)-1ll);
                      atomicAdd((unsigned long long *)&sm.vc[c], 1ull);
                      if (in_c) atomicAdd((unsigned long long *)&sm.intra[c], (unsigned long long)in_c);
                      if (out_a) atomicAdd((unsigned long long *)&sm.intra[a0], (unsigned long long)-out_a);
                  },
                  [&](int v, int64_t s, int64_t e) {
                      long long in_c = 0, out_a = 0, dc = 0;
                      int dv = 0;
                      warp_row(a.col, s, e, lane, [&](int u) { upd(v, u, dc, in_c, out_a, dv); }, [] { return false; });
                      for (int o = 16; o > 0; o >>= 1) {
                          in_c += __shfl_xor_sync(DMOLP_FULL_MASK, in_c, o);
                          out_a += __shfl_xor_sync(DMOLP_FULL_MASK, out_a, o);
                          dv += __shfl_xor_sync(DMOLP_FULL_MASK, dv, o);
                      }
                      if (lane == 0 && dv) atomicAdd(&a.ndiff[v], dv);
                      dcut += dc;
                      if (lane == 0) {
                          arcs += (unsigned long long)(e - s);
                          ++visits;
                          const int a0 = a.label[v], c = a.newlab[v];
                          atomicAdd((unsigned long long *)&sm.vc[a0], (unsigned long long)-1ll);
                          atomicAdd((unsigned long long *)&sm.vc[c], 1ull);
                          if (in_c) atomicAdd((unsigned long long *)&sm.intra[c], (unsigned long long)in_c);
                          if (out_a) atomicAdd((unsigned long long *)&sm.intra[a0], (unsigned long long)-out_a);
                      }
                  });
            block_sum_into(dcut, &sm.dcut);
        }
        __syncthreads();
        // ---- movers take their labels ----
        for (int i = threadIdx.x; i < nmov; i += blockDim.x) {
            const int v = mov[i];
            a.label[v] = a.newlab[v];
            a.newlab[v] = -1;
        }
        // ---- stopping rules (phase2.cpp:305-415) ----
        bool stats = true;
        int stop = 0;
        if (nwin == 0) {
            stats = false;
            if (a.mode == DMOLP_LP_MODE_REF) stop = 1;
        } else if (nmov == 0 && a.mode == DMOLP_LP_MODE_REF) {
            stats = false;
            stop = 2;
        }
        if (stats && !I.symmetric) {  // no reverse arcs to update from: recount
            __syncthreads();
            for (int p = threadIdx.x; p < k; p += blockDim.x) sm.vc[p] = sm.intra[p] = 0;
            if (threadIdx.x == 0) {
                sm.cut_arcs = 0;
                sm.dcut = 0;
            }
            __syncthreads();
            full_stats<NT, TD>(a, I, sm);
        }
        arcs = warp_sum_u64(arcs);
        visits = warp_sum_u64(visits);
        if (lane == 0) {
            atomicAdd(&sm.arcs, arcs);
            atomicAdd(&sm.visits, visits);
        }
        __syncthreads();
        const long long ca = sm.cut_arcs + sm.dcut;
        if (stats) {
            if (ca & 1) {
                o.status = DMOLP_ERR_BAD_LABELS;
                stop = 4;
            } else {
                const long long cur = ca >> 1;
                const double delta =
                    prev_cut > 0 ? fabs(__ddiv_rn((double)(cur - prev_cut), (double)prev_cut)) : 1.0;
                if (delta < 0.03) ++conv;
                else conv = 0;
                prev_cut = cur;
                if (a.mode == DMOLP_LP_MODE_REF && conv >= 10) stop = 3;
            }
        }
        o.te += te_prev + sm.te_cand + sm.te_sel + (stats ? (unsigned long long)I.narcs : 0ull);
        o.changes += nmov;
        o.iterations = t;
        te_prev_next = sm.te_sel;
        nprev = nwin;
        __syncthreads();  // every thread has read this iteration's shared counters
        if (threadIdx.x == 0 && stats) sm.cut_arcs = ca;
        if (stop) {
            o.stop_reason = stop;
            break;
        }
    }
    __syncthreads();
    o.edge_cut = prev_cut;
    o.arcs = sm.arcs;
    o.visits = sm.visits;
    if (threadIdx.x == 0) a.out[ii] = o;
    long long *cnt = a.counts + (size_t)ii * 2 * kBatchMaxK;
    for (int p = threadIdx.x; p < kBatchMaxK; p += blockDim.x) {
        cnt[p] = p < k ? sm.vc[p] : 0;
        cnt[kBatchMaxK + p] = p < k ? sm.intra[p] / 2 : 0;
    }
    __syncthreads();
}

template <int NT, int TD>
__global__ void __launch_bounds__(NT, 1024 / NT) k_batch_lp(Args a) {
    __shared__ Smem<NT> sm;
    for (;;) {
        if (threadIdx.x == 0) {
            sm.inst = atomicAdd(a.next, 1);
            sm.arcs = 0;
            sm.visits = 0;
        }
        __syncthreads();
        const int q = sm.inst;
        if (q >= a.ninst) break;
        run_instance<NT, TD>(a, a.order[q], sm);
    }
}

__global__ void k_batch_begin(int *next, int *stamp_base) {
    *next = 0;
    *stamp_base += kStampStride;
}

// Per instance: local neighbour ids -> union ids (with range check), maximum degree, key widths, and
// whether every row is sorted and every arc has its reverse (binary search in the neighbour's row).
__global__ void k_batch_prepare(const int64_t *off, int32_t *col, Inst *inst, int ninst, int *next, int *err) {
    __shared__ int s_i, s_maxdeg, s_unsym, s_bad;
    for (;;) {
        if (threadIdx.x == 0) {
            s_i = atomicAdd(next, 1);
            s_maxdeg = 0;
            s_unsym = 0;
            s_bad = 0;
        }
        __syncthreads();
        const int i = s_i;
        if (i >= ninst) break;
        Inst I = inst[i];
        const int64_t v0 = I.vbase, v1 = I.vbase + I.nv;
        for (int64_t v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
            const int64_t s = off[v], e = off[v + 1];
            atomicMax(&s_maxdeg, (int)(e - s));
            for (int64_t j = s; j < e; ++j) {
                const int u = col[j];
                if ((unsigned)u >= (unsigned)I.nv) s_bad = 1;
                else col[j] = u + (int)v0;
            }
        }
        __syncthreads();
        for (int64_t v = v0 + threadIdx.x; v < v1 && !s_bad; v += blockDim.x) {
            const int64_t s = off[v], e = off[v + 1];
            int prev = -1;
            bool sorted = true;
            for (int64_t j = s; j < e; ++j) {
                const int u = col[j];
                sorted &= u > prev;
                prev = u;
            }
            if (!sorted) {
                s_unsym = 1;
                continue;
            }
            for (int64_t j = s; j < e; ++j) {
                const int u = col[j];
                int64_t lo = off[u], hi = off[u + 1];
                while (lo < hi) {
                    const int64_t mid = (lo + hi) >> 1;
                    if (col[mid] < (int)v) lo = mid + 1;
                    else hi = mid;
                }
                if (lo >= off[u + 1] || col[lo] != (int)v) {
                    s_unsym = 1;
                    break;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_bad) atomicExch(err, i + 1);
            I.maxdeg = s_maxdeg;
            int ib = 1, db = 1;
            while (ib < 62 && (int64_t(1) << ib) <= (int64_t)(I.nv > 0 ? I.nv - 1 : 0)) ++ib;
            while (db < 62 && (int64_t(1) << db) <= (int64_t)s_maxdeg) ++db;
            I.ibits = ib;
            I.dbits = db;
            I.symmetric = !s_unsym && !s_bad;
            inst[i] = I;
        }
        __syncthreads();
    }
}

template <int NT, int TD>
void launch_variant(const Args &a, int grid, cudaStream_t s) {
    k_batch_lp<NT, TD><<<grid, NT, 0, s>>>(a);
}

}  // namespace

int occupancy(int nt, int td) {
    int n = 0;
    cudaError_t e = cudaSuccess;
#define DMOLP_OCC(NT_, TD_) \
    if (nt == NT_ && td == TD_) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_lp<NT_, TD_>, NT_, 0);
    DMOLP_OCC(256, 8) DMOLP_OCC(256, 16) DMOLP_OCC(512, 8) DMOLP_OCC(512, 16) DMOLP_OCC(1024, 8) DMOLP_OCC(1024, 16)
#undef DMOLP_OCC
    return e == cudaSuccess ? n : 0;
}

bool launch(const Args &a, int nt, int td, int grid, cudaStream_t s) {
    k_batch_begin<<<1, 1, 0, s>>>(a.next, a.stamp_base);
#define DMOLP_LAUNCH(NT_, TD_)              \
    if (nt == NT_ && td == TD_) {           \
        launch_variant<NT_, TD_>(a, grid, s); \
        return true;                        \
    }
    DMOLP_LAUNCH(256, 8) DMOLP_LAUNCH(256, 16) DMOLP_LAUNCH(512, 8) DMOLP_LAUNCH(512, 16) DMOLP_LAUNCH(1024, 8)
    DMOLP_LAUNCH(1024, 16)
#undef DMOLP_LAUNCH
    return false;
}

void prepare(const int64_t *off, int32_t *col, Inst *inst, int ninst, int *next, int *err, int grid, cudaStream_t s) {
    k_batch_prepare<<<grid, 256, 0, s>>>(off, col, inst, ninst, next, err);
}

}  // namespace batch
}  // namespace dmolp
