/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- the checker for the product's CUDA path, and the "port"
 * CPU baseline in bench.py.  It is never linked into or called by the product.
 *
 * A single-threaded CPU restatement of the reference's partitioning path as it behaves with one MPI
 * rank.  Each function cites the reference lines it follows (paths relative to the reference tree).
 * Floating point is IEEE double in the source's evaluation order (built without -ffast-math and
 * without FMA contraction, see oracle/Makefile).
 *
 * Pinned against the reference itself: tests/golden/ holds outputs of the reference sources run through
 * oracle/ref_harness.cpp (tests/golden/make_golden.py), and tests/test_oracle.py compares this file's
 * results with them.
 */
#include "dmolp_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

namespace {

thread_local std::string g_err;

uint64_t fnv1a(const void *data, size_t n) {
    uint64_t h = 1469598103934665603ULL;
    const unsigned char *p = (const unsigned char *)data;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// Order-independent checksum of a vertex set: sum (mod 2^64) of the SplitMix64 finaliser of each id.
uint64_t set_sum(const int *v, size_t n) {
    uint64_t s = 0;
    for (size_t i = 0; i < n; ++i) {
        uint64_t z = (uint64_t)(uint32_t)v[i] + 0x9e3779b97f4a7c15ULL;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        s += z ^ (z >> 31);
    }
    return s;
}

struct Csr {
    int64_t nv;
    const int64_t *off;
    const int32_t *col;
    int64_t deg(int64_t v) const { return off[v + 1] - off[v]; }
};

// ---------------------------------------------------------------- phase 1

// src/phase1/init.cpp:139-177.  Input order is global_degree's iteration order at one rank, which is
// vertex V-1 down to 0 (libstdc++ unordered_map, every key in its own bucket, iterated newest-first);
// the unstable std::sort then decides the order of equal-degree vertices.
std::vector<int> find_hubs(int64_t nv, const int32_t *rawdeg) {
    std::vector<std::pair<int, int>> sd;
    sd.reserve(nv);
    for (int64_t v = nv - 1; v >= 0; --v) sd.emplace_back((int)v, rawdeg[v]);
    std::sort(sd.begin(), sd.end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
        return a.second < b.second;
    });
    const int N = (int)sd.size();
    std::vector<int> hubs;
    if (N < 2) return hubs;
    std::vector<double> cum(N);
    double total = 0.0, run = 0.0;
    for (int i = 0; i < N; ++i) {
        total += sd[i].second;
        run += sd[i].second;
        cum[i] = run;
    }
    for (int i = 0; i < N; ++i) cum[i] /= total;
    const double inv_n = 1.0 / N;
    const double x1 = N * inv_n, y1 = cum[N - 1];
    const double x0 = (N - 1) * inv_n, y0 = cum[N - 2];
    const double slope = (y1 - y0) / (x1 - x0);
    const double x_int = x1 - y1 / slope;
    for (int i = N - 1; i >= 0; --i) {
        if ((i + 1) * inv_n > x_int) hubs.push_back(sd[i].first);
        else break;
    }
    return hubs;
}

// src/phase1/init.cpp:179-187, including its tie rule that compares a vertex id with the best DEGREE;
// iteration order V-1 .. 0 as above.
std::pair<int, int> first_seed(int64_t nv, const int32_t *rawdeg) {
    std::pair<int, int> best(-1, -1);
    for (int64_t v = nv - 1; v >= 0; --v) {
        int d = rawdeg[v];
        if (d > best.second || (d == best.second && (int)v < best.second)) best = std::make_pair((int)v, d);
    }
    return best;
}

// src/phase1/seed.cpp:20-101 with MAX_LEVELS = 3: the ball of radius 2 around s (levels 0, 1, 2).
void mark_ball(const Csr &g, int s, std::vector<char> &covered, uint64_t &te) {
    std::vector<char> seen(g.nv, 0);
    std::vector<int> level{ s }, next;
    seen[s] = 1;
    covered[s] = 1;
    for (int depth = 0; depth < 2; ++depth) {
        next.clear();
        for (int u : level) {
            te += (uint64_t)g.deg(u);
            for (int64_t e = g.off[u]; e < g.off[u + 1]; ++e) {
                int w = g.col[e];
                if (!seen[w]) {
                    seen[w] = 1;
                    covered[w] = 1;
                    next.push_back(w);
                }
            }
        }
        level.swap(next);
    }
}

// src/phase1/seed.cpp:138-242 at one rank.
std::vector<int> find_seeds(const Csr &g, int k, std::pair<int, int> first, const std::vector<int> &hubs,
                            const int32_t *rawdeg, uint64_t &te, int &found) {
    std::vector<int> seeds{ first.first };
    std::vector<char> used(hubs.size(), 0), covered(g.nv, 0);
    auto mark_used = [&](int s) {
        auto it = std::find(hubs.begin(), hubs.end(), s);
        if (it != hubs.end()) used[it - hubs.begin()] = 1;
    };
    mark_used(first.first);
    size_t balls = 0;
    for (int p = 1; p < k && !hubs.empty(); ++p) {  // seed.cpp:195-198: no hubs, no search
        for (; balls < seeds.size(); ++balls) mark_ball(g, seeds[balls], covered, te);
        int best = -1, best_deg = -1;
        for (size_t i = 0; i < hubs.size(); ++i) {
            if (used[i] || covered[hubs[i]]) continue;
            int d = rawdeg[hubs[i]];
            if (d > best_deg) {
                best_deg = d;
                best = hubs[i];
            }
        }
        if (best == -1) break;  // seed.cpp:214-217: fewer than k seeds
        seeds.push_back(best);
        mark_used(best);
    }
    found = (int)seeds.size();
    // Seed completion.  With fewer than k seeds the reference goes on to read seeds[p] past the end of
    // the vector (partition.cpp:347, undefined).  This path defines it: the next seed is the unused hub
    // of highest degree (first in hub order on ties); with no hub left, the non-seed vertex of highest
    // degree (lowest id on ties).
    std::vector<char> is_seed(g.nv, 0);
    for (int s : seeds)
        if (s >= 0) is_seed[s] = 1;
    while ((int)seeds.size() < k) {
        int best = -1, best_deg = -1;
        for (size_t i = 0; i < hubs.size(); ++i)
            if (!used[i] && rawdeg[hubs[i]] > best_deg) {
                best_deg = rawdeg[hubs[i]];
                best = hubs[i];
            }
        if (best == -1)
            for (int64_t v = 0; v < g.nv; ++v)
                if (!is_seed[v] && rawdeg[v] > best_deg) {
                    best_deg = rawdeg[v];
                    best = (int)v;
                }
        if (best == -1) break;  // fewer vertices than parts
        seeds.push_back(best);
        is_seed[best] = 1;
        mark_used(best);
    }
    return seeds;
}

// src/phase1/partition.cpp:323-604 at one rank.  Per round, each part expands the theta frontier
// vertices with the smallest (raw degree, id); an unlabelled neighbour goes to the lowest part that
// reaches it; with every frontier empty, all unlabelled vertices go to the smallest part (ties: lowest).
// Parts without a seed (fewer than k seeds, where the reference reads past its seed vector) start empty.
int expand_partitions(const Csr &g, int k, int theta, const std::vector<int> &seeds, const int32_t *rawdeg,
                      int32_t *label, uint64_t &te) {
    const int64_t nv = g.nv;
    std::fill(label, label + nv, -1);
    std::vector<std::vector<int>> frontier(k);
    for (int p = 0; p < k && p < (int)seeds.size(); ++p) {
        if (seeds[p] < 0 || seeds[p] >= nv) continue;
        label[seeds[p]] = p;
        frontier[p].push_back(seeds[p]);
    }
    std::vector<int64_t> size(k, 0);
    auto recount = [&]() -> int64_t {
        std::fill(size.begin(), size.end(), 0);
        int64_t n = 0;
        for (int64_t v = 0; v < nv; ++v)
            if (label[v] >= 0) {
                ++n;
                if (label[v] < k) ++size[label[v]];
            }
        return n;
    };
    int64_t labeled = recount();
    std::vector<char> claimed(nv, 0);
    int rounds = 0;
    while (labeled < nv) {
        bool all_empty = true;
        for (int p = 0; p < k; ++p)
            if (!frontier[p].empty()) all_empty = false;
        if (all_empty) {  // partition.cpp:376-394
            int best = 0;
            for (int p = 0; p < k; ++p)
                if (size[p] < size[best]) best = p;
            for (int64_t v = 0; v < nv; ++v)
                if (label[v] < 0) {
                    label[v] = best;
                    frontier[best].push_back((int)v);
                }
        }
        std::vector<std::vector<int>> sel(k), carry(k), fresh(k);
        for (int p = 0; p < k; ++p) {  // partition.cpp:400-441
            std::vector<int> &f = frontier[p];
            std::sort(f.begin(), f.end(), [&](int a, int b) {
                if (rawdeg[a] != rawdeg[b]) return rawdeg[a] < rawdeg[b];
                return a < b;
            });
            for (size_t i = 0; i < f.size(); ++i) ((int)i < theta ? sel[p] : carry[p]).push_back(f[i]);
        }
        for (int p = 0; p < k; ++p)  // partition.cpp:455-476
            for (int u : sel[p]) {
                te += (uint64_t)g.deg(u);
                for (int64_t e = g.off[u]; e < g.off[u + 1]; ++e) {
                    int v = g.col[e];
                    if (label[v] < 0 && !claimed[v]) {
                        claimed[v] = 1;
                        fresh[p].push_back(v);
                    }
                }
            }
        for (int p = 0; p < k; ++p)
            for (int v : fresh[p]) {
                label[v] = p;
                claimed[v] = 0;
            }
        labeled = recount();
        for (int p = 0; p < k; ++p) {
            frontier[p].swap(carry[p]);
            frontier[p].insert(frontier[p].end(), fresh[p].begin(), fresh[p].end());
        }
        ++rounds;
    }
    return rounds;
}

// ---------------------------------------------------------------- phase 2

struct Stats {
    std::vector<int64_t> vc, ec;  // vertex counts, intra-part edge counts (arcs / 2 per part)
    int64_t total_vertices = 0, total_edges = 0;
    double ev = 0, ee = 0;
};

// src/phase2/phase2.cpp:55-117.
Stats part_stats(const Csr &g, const int32_t *label, int k) {
    Stats s;
    s.vc.assign(k, 0);
    std::vector<int64_t> arcs(k, 0);
    for (int64_t u = 0; u < g.nv; ++u) {
        int lu = label[u];
        if (lu < 0 || lu >= k) continue;
        s.vc[lu]++;
        for (int64_t e = g.off[u]; e < g.off[u + 1]; ++e)
            if (label[g.col[e]] == lu) arcs[lu]++;
    }
    s.ec.assign(k, 0);
    for (int p = 0; p < k; ++p) {
        s.ec[p] = arcs[p] / 2;
        s.total_vertices += s.vc[p];
        s.total_edges += s.ec[p];
    }
    s.ev = (double)s.total_vertices / k;
    s.ee = (s.total_edges > 0) ? (double)s.total_edges / k : 1.0;
    return s;
}

// src/phase2/phase2.cpp:214-253: arcs with different labels, halved; -1 labels or an odd count abort there.
int64_t edge_cut(const Csr &g, const int32_t *label, bool *bad) {
    int64_t cut = 0, invalid = 0;
    for (int64_t u = 0; u < g.nv; ++u)
        for (int64_t e = g.off[u]; e < g.off[u + 1]; ++e) {
            int lu = label[u], lv = label[g.col[e]];
            if (lu == -1 || lv == -1) {
                ++invalid;
                continue;
            }
            if (lu != lv) ++cut;
        }
    *bad = invalid != 0 || (cut & 1);
    return cut >> 1;
}

// src/phase2/phase2.cpp:158-209.  Returns {penalty, RE}.
void penalties(const Stats &s, int k, int iter, std::vector<double> &pen, std::vector<double> &RE) {
    std::vector<double> RV(k);
    RE.assign(k, 0.0);
    pen.assign(k, 0.0);
    for (int i = 0; i < k; ++i) {
        RV[i] = (s.ev > 0) ? (double)s.vc[i] / s.ev : 1.0;
        RE[i] = (s.ee > 0) ? (double)s.ec[i] / s.ee : 1.0;
    }
    double rv_mean = 0.0, re_mean = 0.0;
    for (int i = 0; i < k; ++i) {
        rv_mean += RV[i];
        re_mean += RE[i];
    }
    rv_mean /= k;
    re_mean /= k;
    double rv_var = 0.0, re_var = 0.0;
    for (int i = 0; i < k; ++i) {
        rv_var += (RV[i] - rv_mean) * (RV[i] - rv_mean);
        re_var += (RE[i] - re_mean) * (RE[i] - re_mean);
    }
    rv_var /= k;
    re_var /= k;
    double total_var = rv_var + re_var;
    double imb_rv = (total_var > 0) ? rv_var / total_var : 0.0;
    double imb_re = (total_var > 0) ? re_var / total_var : 0.0;
    const double lg = std::log((double)iter);
    for (int i = 0; i < k; ++i) {
        double grv = (1.0 - RV[i]) * (1.0 + lg);
        double gre = (1.0 - RE[i]) * (1.0 + lg);
        pen[i] = imb_rv * grv + imb_re * gre;
    }
}

// The kernel's per-vertex rule, boundaryLPKernel_unified (src/phase2/gpu_lp_boundary.cu:354-426),
// stated by simulating its 32-lane shuffle-down reduction.  cap = 0 keeps its min(k, 32) label limit.
int lp_decide(int own, const int32_t *nl, int64_t deg, const double *pen, int k, int cap) {
    const int eff = cap == 0 ? std::min(k, 32) : k;
    std::vector<double> score(eff, 0.0);
    for (int64_t i = 0; i < deg; ++i)
        if (nl[i] >= 0 && nl[i] < eff) score[nl[i]] += 1.0;
    int best_label = own;
    double best = (own >= 0 && own < eff) ? score[own] : -1e300;
    for (int base = 0; base < eff; base += 32) {
        double cs[32];
        int cl[32];
        for (int lane = 0; lane < 32; ++lane) {
            cl[lane] = base + lane;
            cs[lane] = -1e300;
            if (cl[lane] < eff) {
                double s = score[cl[lane]];
                if (s > 0.0) s *= (1.0 + pen[cl[lane]]);
                cs[lane] = s;
            }
        }
        for (int off = 16; off > 0; off >>= 1)
            for (int lane = 0; lane + off < 32; ++lane)  // ascending lanes read not-yet-updated partners
                if (cs[lane + off] > cs[lane]) {
                    cs[lane] = cs[lane + off];
                    cl[lane] = cl[lane + off];
                }
        if (cs[0] > best) {
            best = cs[0];
            best_label = cl[0];
        }
    }
    return best_label;
}

// src/phase2/gpu_lp_boundary.cu:185-305.  Candidate set = prev window plus neighbours; keep vertices
// with a differently-labelled neighbour; per label keep ceil(e^(-iter/5) * n) ordered by degree (desc
// when RE[label] > 1, else asc), then id.  Returns the selected set (ascending id order).
std::vector<int> select_window(const Csr &g, const int32_t *label, const std::vector<int> &prev,
                               const std::vector<double> &RE, int iter, int k, uint64_t &te_prev,
                               uint64_t &te_cand, int64_t &ncand) {
    const int64_t nv = g.nv;
    std::vector<char> is_cand(nv, 0);
    for (int v : prev) {
        if (v < 0 || v >= nv) continue;
        is_cand[v] = 1;
        te_prev += (uint64_t)g.deg(v);
        for (int64_t e = g.off[v]; e < g.off[v + 1]; ++e) is_cand[g.col[e]] = 1;
    }
    std::vector<std::vector<std::pair<int, int>>> by_label(k);
    ncand = 0;
    for (int64_t v = 0; v < nv; ++v) {
        if (!is_cand[v]) continue;
        ++ncand;
        te_cand += (uint64_t)g.deg(v);
        const int lv = label[v];
        bool boundary = false;
        for (int64_t e = g.off[v]; e < g.off[v + 1]; ++e)
            if (label[g.col[e]] != lv) {
                boundary = true;
                break;
            }
        if (boundary && lv >= 0 && lv < k) by_label[lv].emplace_back((int)v, (int)g.deg(v));
    }
    const double ratio = std::exp((-iter) / (5.0));
    std::vector<int> sel;
    for (int p = 0; p < k; ++p) {
        auto &vec = by_label[p];
        if (vec.empty()) continue;
        if (RE[p] > 1.0)
            std::sort(vec.begin(), vec.end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
                if (a.second != b.second) return a.second > b.second;
                return a.first < b.first;
            });
        else
            std::sort(vec.begin(), vec.end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
                if (a.second != b.second) return a.second < b.second;
                return a.first < b.first;
            });
        int m = (int)std::ceil(ratio * (double)vec.size());
        if (m > (int)vec.size()) m = (int)vec.size();
        for (int i = 0; i < m; ++i) sel.push_back(vec[i].first);
    }
    std::sort(sel.begin(), sel.end());
    return sel;
}

double max_ratio(const std::vector<int64_t> &c, double expected_if_pos, bool use_expected) {
    double m = 0.0;
    for (int64_t x : c) {
        double r = use_expected ? (double)x / expected_if_pos : 1.0;
        m = std::max(m, r);
    }
    return m;
}

}  // namespace

extern "C" {

const char *oracle_last_error(void) { return g_err.c_str(); }

// src/phase1/init.cpp:8-100 (fast_atoi tokenisation; a final line without '\n' is dropped) and the CSR
// of src/phase1/partition.cpp:227-262 (sort_unique per row, self-loops kept).
int oracle_load_adjtext(const char *path, int64_t *nv_out, int64_t *narcs_out, int64_t *off, int32_t *col,
                        int32_t *rawdeg) {
    FILE *f = fopen(path, "rb");
    if (!f) {
        g_err = std::string("cannot open ") + path;
        return 1;
    }
    std::string data;
    {
        char buf[1 << 16];
        size_t n;
        while ((n = fread(buf, 1, sizeof buf, f)) > 0) data.append(buf, n);
        fclose(f);
    }
    size_t p = data.find('\n');
    if (p == std::string::npos) {
        g_err = "missing header line";
        return 1;
    }
    std::vector<std::vector<int>> rows;
    size_t start = p + 1;
    while (true) {
        size_t nl = data.find('\n', start);
        if (nl == std::string::npos) break;
        std::vector<int> r;
        size_t i = start;
        while (i < nl && data[i] != '\0') {
            int x = 0;
            while (i < nl && (unsigned)(data[i] - '0') <= 9) x = x * 10 + (data[i++] - '0');
            while (i < nl && data[i] != '\0' && (unsigned)(data[i] - '0') > 9) ++i;
            r.push_back(x);
        }
        rows.push_back(std::move(r));
        start = nl + 1;
    }
    const int64_t nv = (int64_t)rows.size();
    int64_t narcs = 0;
    for (auto &r : rows) {
        for (int x : r)
            if (x < 0 || x >= nv) {
                g_err = "neighbour id out of range";
                return 1;
            }
        std::vector<int> s(r);
        std::sort(s.begin(), s.end());
        narcs += std::unique(s.begin(), s.end()) - s.begin();
    }
    *nv_out = nv;
    *narcs_out = narcs;
    if (!off) return 0;
    off[0] = 0;
    for (int64_t v = 0; v < nv; ++v) {
        std::vector<int> s(rows[v]);
        std::sort(s.begin(), s.end());
        s.erase(std::unique(s.begin(), s.end()), s.end());
        std::copy(s.begin(), s.end(), col + off[v]);
        off[v + 1] = off[v] + (int64_t)s.size();
        if (rawdeg) rawdeg[v] = (int32_t)rows[v].size();
    }
    return 0;
}

// The permutation std::sort leaves on (id, degree) pairs ordered by degree: the sort of find_hub_nodes
// (src/phase1/init.cpp:142), run by this toolchain's libstdc++ itself.
int oracle_degree_order(int64_t n, int32_t *ids, int32_t *degrees) {
    std::vector<std::pair<int, int>> a(n);
    for (int64_t i = 0; i < n; ++i) a[i] = std::make_pair(ids[i], degrees[i]);
    std::sort(a.begin(), a.end(), [](const std::pair<int, int> &x, const std::pair<int, int> &y) {
        return x.second < y.second;
    });
    for (int64_t i = 0; i < n; ++i) {
        ids[i] = a[i].first;
        degrees[i] = a[i].second;
    }
    return 0;
}

int oracle_find_hubs(int64_t nv, const int32_t *rawdeg, int32_t *hubs_out, int64_t *nhubs) {
    std::vector<int> h = find_hubs(nv, rawdeg);
    *nhubs = (int64_t)h.size();
    if (hubs_out) std::copy(h.begin(), h.end(), hubs_out);
    return 0;
}

// src/phase1/phase1.cpp:18-161 at one rank.
int oracle_phase1(int64_t nv, const int64_t *off, const int32_t *col, const int32_t *rawdeg, int k, int theta,
                  int32_t *labels_out, int32_t *seeds_out, int64_t *vertex_counts, int64_t *edge_counts,
                  oracle_phase1_result *res) {
    if (k <= 0 || theta <= 0) {
        g_err = "k and theta must be positive";
        return 1;
    }
    Csr g{ nv, off, col };
    std::memset(res, 0, sizeof(*res));
    std::vector<int> hubs = find_hubs(nv, rawdeg);
    std::pair<int, int> first = first_seed(nv, rawdeg);
    uint64_t te = 0;
    int found = 0;
    std::vector<int> seeds = nv > 0 ? find_seeds(g, k, first, hubs, rawdeg, te, found) : std::vector<int>();
    res->num_hubs = (int64_t)hubs.size();
    res->first_seed = first.first;
    res->first_seed_degree = first.second;
    res->num_seeds = found;  // seeds found by the reference's rule; the rest come from seed completion
    for (int p = 0; p < k; ++p) seeds_out[p] = p < (int)seeds.size() ? seeds[p] : -1;
    res->rounds = expand_partitions(g, k, theta, seeds, rawdeg, labels_out, te);
    res->te = te;
    // phase1.cpp:83-153
    int64_t cut_arcs = 0;
    std::vector<int64_t> intra(k, 0);
    for (int p = 0; p < k; ++p) vertex_counts[p] = 0;
    for (int64_t u = 0; u < nv; ++u) {
        int lu = labels_out[u];
        if (lu >= 0) vertex_counts[lu]++;
        for (int64_t e = off[u]; e < off[u + 1]; ++e) {
            int lv = labels_out[col[e]];
            if (lu != -1 && lv != -1 && lu != lv) ++cut_arcs;
            if (lu >= 0 && lv == lu) intra[lu]++;
        }
    }
    res->initial_edge_cut = cut_arcs / 2;
    double ev = (double)nv / k;
    double mv = 0;
    for (int p = 0; p < k; ++p) mv = std::max(mv, vertex_counts[p] / ev);
    res->initial_vertex_balance = mv;
    double tot = 0;
    for (int p = 0; p < k; ++p) {
        edge_counts[p] = intra[p] / 2;
        tot += (double)edge_counts[p];
    }
    double ee = tot / k, me = 0;
    for (int p = 0; p < k; ++p) me = std::max(me, edge_counts[p] / ee);
    res->initial_edge_balance = me;
    return 0;
}

// src/phase2/phase2.cpp:256-449 at one rank (mode 0), or exactly `iters` iterations (mode 1).
int oracle_phase2(int64_t nv, const int64_t *off, const int32_t *col, int k, int32_t *label, int mode, int iters,
                  int cap, oracle_iter_record *records, int64_t *counts_out, double *penalty_out,
                  oracle_phase2_result *res) {
    if (k <= 0) {
        g_err = "k must be positive";
        return 1;
    }
    Csr g{ nv, off, col };
    std::memset(res, 0, sizeof(*res));
    bool bad = false;
    int64_t prev_cut = edge_cut(g, label, &bad);
    if (bad) {
        g_err = "invalid labels or odd edge cut";
        return 3;
    }
    Stats st = part_stats(g, label, k);
    std::vector<int> window(nv);
    for (int64_t v = 0; v < nv; ++v) window[v] = (int)v;
    const int max_iter = mode == 0 ? 500 : iters;
    int conv = 0;
    std::vector<double> pen, RE;
    std::vector<int32_t> nl;
    std::vector<std::pair<int, int>> moves;
    int it = 0;
    res->stop_reason = 0;
    for (; it < max_iter; ++it) {
        penalties(st, k, it + 1, pen, RE);
        if (penalty_out) std::copy(pen.begin(), pen.end(), penalty_out + (size_t)it * k);
        uint64_t te_prev = 0, te_cand = 0, te_sel = 0, te_stats = 0;
        int64_t ncand = 0;
        window = select_window(g, label, window, RE, it + 1, k, te_prev, te_cand, ncand);
        int changes = 0;
        if (!window.empty()) {
            moves.clear();
            for (int v : window) {
                te_sel += (uint64_t)g.deg(v);
                nl.assign(col + off[v], col + off[v + 1]);
                for (auto &x : nl) x = label[x];
                int nlab = lp_decide(label[v], nl.data(), (int64_t)nl.size(), pen.data(), k, cap);
                if (nlab != label[v]) moves.emplace_back(v, nlab);
            }
            for (auto &m : moves) label[m.first] = m.second;
            changes = (int)moves.size();
        }
        bool stop = false;
        if (window.empty()) {
            if (mode == 0) {
                res->stop_reason = 1;
                stop = true;
            }
        } else if (changes == 0 && mode == 0) {
            res->stop_reason = 2;
            stop = true;
        } else {
            st = part_stats(g, label, k);
            int64_t cur = edge_cut(g, label, &bad);
            if (bad) {
                g_err = "invalid labels or odd edge cut";
                return 3;
            }
            te_stats = (uint64_t)off[nv];
            double delta = (prev_cut > 0) ? std::fabs((double)(cur - prev_cut) / (double)prev_cut) : 1.0;
            if (delta < 0.03) ++conv;
            else conv = 0;
            prev_cut = cur;
            if (mode == 0 && conv >= 10) {
                res->stop_reason = 3;
                stop = true;
            }
        }
        res->te_total += te_prev + te_cand + te_sel + te_stats;
        if (records) {
            oracle_iter_record &r = records[it];
            r.iteration = it + 1;
            r.window = (int32_t)window.size();
            r.candidates = (int32_t)ncand;
            r.changes = changes;
            r.edge_cut = prev_cut;
            r.window_hash = fnv1a(window.data(), window.size() * sizeof(int));
            r.window_sum = set_sum(window.data(), window.size());
            r.labels_hash = fnv1a(label, (size_t)nv * sizeof(int32_t));
            r.te_prev = te_prev;
            r.te_cand = te_cand;
            r.te_sel = te_sel;
            r.te_stats = te_stats;
        }
        if (counts_out) {
            for (int p = 0; p < k; ++p) {
                counts_out[(size_t)it * 2 * k + p] = st.vc[p];
                counts_out[(size_t)it * 2 * k + k + p] = st.ec[p];
            }
        }
        if (stop) {
            ++it;
            break;
        }
    }
    res->iterations_run = it;
    Stats fs = part_stats(g, label, k);
    res->edge_cut = prev_cut;
    res->vertex_balance = max_ratio(fs.vc, fs.ev, fs.ev > 0);
    res->edge_balance = max_ratio(fs.ec, fs.ee, fs.ee > 0);
    res->total_vertices = fs.total_vertices;
    res->total_edges = fs.total_edges;
    return 0;
}

uint64_t oracle_fnv1a(const void *data, size_t n) { return fnv1a(data, n); }

uint64_t oracle_set_sum(const int32_t *v, int64_t n) { return set_sum(v, (size_t)n); }

int32_t oracle_lp_decide(int32_t own, const int32_t *nbr_labels, int64_t deg, const double *penalty, int k, int cap) {
    return lp_decide(own, nbr_labels, deg, penalty, k, cap);
}

}  // extern "C"
