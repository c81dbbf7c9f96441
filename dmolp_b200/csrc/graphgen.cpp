// Seeded synthetic graph generators and graph file I/O (host C++, OpenMP).
//
// Every generator returns an undirected graph as a CSR with sorted, de-duplicated neighbour lists
// and no self-loops, the form the reference's tool/convert.sh produces (convert.sh:69-186) and that
// its loader reads (src/phase1/init.cpp:25-100).  Output is independent of the thread count: random
// streams are tied to fixed-size chunks of work, never to threads.
//
//   R-MAT (Chakrabarti et al. 2004): recursive quadrant sampling with probabilities (a,b,c,d),
//        symmetrised, optionally relabelled by a seeded random permutation (Graph500 practice).
//   k-NN geometric: n points uniform in [0,1)^dim, each joined to its k nearest (Euclidean, ties by
//        index), symmetrised (union).
//   Barabasi-Albert: preferential attachment, each new vertex joins m distinct earlier vertices
//        chosen with probability proportional to degree.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "graphgen.h"

namespace {

// splitmix64 (Steele, Lea, Flood 2014) for seeding; xoshiro256** (Blackman, Vigna 2018) for streams.
inline uint64_t splitmix64(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s[4];
    Rng(uint64_t seed, uint64_t stream) {
        uint64_t x = seed * 0x9E3779B97F4A7C15ULL + stream * 0xD1B54A32D192ED03ULL + 0x1234567ULL;
        for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
    }
    static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    inline uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    inline double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    inline uint64_t below(uint64_t n) {  // unbiased: Lemire's multiply-shift with rejection
        uint64_t x = next();
        __uint128_t m = (__uint128_t)x * n;
        uint64_t l = (uint64_t)m;
        if (l < n) {
            uint64_t t = (0 - n) % n;
            while (l < t) {
                x = next();
                m = (__uint128_t)x * n;
                l = (uint64_t)m;
            }
        }
        return (uint64_t)(m >> 64);
    }
};

thread_local std::string g_err;

}  // namespace

struct dmolp_csr {
    int64_t nv = 0;
    std::vector<int64_t> off;
    std::vector<int32_t> col;
};

namespace {

// Build a symmetric CSR (sorted, unique, no self-loops) from directed arcs (src[i] -> dst[i]); both
// directions must already be present in the arc list.
dmolp_csr *csr_from_arcs(int64_t nv, std::vector<int32_t> &src, std::vector<int32_t> &dst) {
    dmolp_csr *g = new dmolp_csr();
    g->nv = nv;
    const int64_t na = (int64_t)src.size();
    std::vector<int64_t> cnt(nv + 1, 0);
    {
        std::vector<std::atomic<int64_t>> acnt(nv);
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < nv; ++v) acnt[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < na; ++i)
            if (src[i] != dst[i]) acnt[src[i]].fetch_add(1, std::memory_order_relaxed);
        for (int64_t v = 0; v < nv; ++v) cnt[v + 1] = cnt[v] + acnt[v].load(std::memory_order_relaxed);
    }
    std::vector<int32_t> tmp(cnt[nv]);
    {
        std::vector<std::atomic<int64_t>> pos(nv);
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < nv; ++v) pos[v].store(cnt[v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < na; ++i)
            if (src[i] != dst[i]) tmp[pos[src[i]].fetch_add(1, std::memory_order_relaxed)] = dst[i];
    }
    std::vector<int32_t>().swap(src);
    std::vector<int32_t>().swap(dst);
    std::vector<int64_t> ndeg(nv + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < nv; ++v) {
        int32_t *b = tmp.data() + cnt[v], *e = tmp.data() + cnt[v + 1];
        std::sort(b, e);
        ndeg[v + 1] = std::unique(b, e) - b;
    }
    g->off.assign(nv + 1, 0);
    for (int64_t v = 0; v < nv; ++v) g->off[v + 1] = g->off[v] + ndeg[v + 1];
    g->col.resize(g->off[nv]);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < nv; ++v)
        std::memcpy(g->col.data() + g->off[v], tmp.data() + cnt[v], sizeof(int32_t) * (size_t)(g->off[v + 1] - g->off[v]));
    return g;
}

}  // namespace

extern "C" {

const char *dmolp_gen_last_error(void) { return g_err.c_str(); }

uint64_t dmolp_fnv1a(const void *data, int64_t n) {
    uint64_t h = 1469598103934665603ULL;
    const unsigned char *p = (const unsigned char *)data;
    for (int64_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

int dmolp_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int permute,
                   dmolp_csr **out) {
    try {
        if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) {
            g_err = "rmat: bad parameters";
            return 1;
        }
        const int64_t nv = int64_t(1) << scale;
        const int64_t ne = nv * edge_factor;
        const int64_t chunk = int64_t(1) << 16;
        const int64_t nchunks = (ne + chunk - 1) / chunk;
        std::vector<int32_t> src(2 * ne), dst(2 * ne);
        const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t ch = 0; ch < nchunks; ++ch) {
            Rng r(seed, (uint64_t)ch);
            const int64_t e0 = ch * chunk, e1 = std::min(ne, e0 + chunk);
            for (int64_t e = e0; e < e1; ++e) {
                int64_t u = 0, v = 0;
                for (int l = 0; l < scale; ++l) {
                    double x = r.uniform();
                    int bu = 0, bv = 0;
                    if (x < a) {
                    } else if (x < ab) {
                        bv = 1;
                    } else if (x < abc) {
                        bu = 1;
                    } else {
                        bu = 1;
                        bv = 1;
                    }
                    u = (u << 1) | bu;
                    v = (v << 1) | bv;
                }
                src[2 * e] = (int32_t)u;
                dst[2 * e] = (int32_t)v;
                src[2 * e + 1] = (int32_t)v;
                dst[2 * e + 1] = (int32_t)u;
            }
        }
        if (permute) {
            std::vector<int32_t> perm(nv);
            for (int64_t i = 0; i < nv; ++i) perm[i] = (int32_t)i;
            Rng r(seed ^ 0x5bd1e995ULL, 0xFFFFFFFFULL);
            for (int64_t i = nv - 1; i > 0; --i) std::swap(perm[i], perm[r.below((uint64_t)i + 1)]);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < 2 * ne; ++i) {
                src[i] = perm[src[i]];
                dst[i] = perm[dst[i]];
            }
        }
        *out = csr_from_arcs(nv, src, dst);
        return 0;
    } catch (const std::bad_alloc &) {
        g_err = "rmat: out of host memory";
        return 2;
    }
}

int dmolp_gen_knn(int64_t n, int dim, int knn, uint64_t seed, dmolp_csr **out) {
    try {
        if (n < 2 || (dim != 2 && dim != 3) || knn < 1 || knn >= n || n > (int64_t(1) << 31) - 1) {
            g_err = "knn: bad parameters";
            return 1;
        }
        std::vector<double> pts((size_t)n * dim);
        {
            const int64_t chunk = 4096;
#pragma omp parallel for schedule(static)
            for (int64_t ch = 0; ch < (n + chunk - 1) / chunk; ++ch) {
                Rng r(seed, (uint64_t)ch);
                for (int64_t i = ch * chunk; i < std::min(n, (ch + 1) * chunk); ++i)
                    for (int d = 0; d < dim; ++d) pts[(size_t)i * dim + d] = r.uniform();
            }
        }
        // uniform grid, about 2 points per cell
        int g = (int)std::max(1.0, std::floor(std::pow((double)n / 2.0, 1.0 / dim)));
        int64_t ncell = 1;
        for (int d = 0; d < dim; ++d) ncell *= g;
        auto cell_of = [&](int64_t i, int *c) {
            for (int d = 0; d < dim; ++d) c[d] = std::min(g - 1, (int)(pts[(size_t)i * dim + d] * g));
        };
        auto lin = [&](const int *c) {
            int64_t x = 0;
            for (int d = dim - 1; d >= 0; --d) x = x * g + c[d];
            return x;
        };
        std::vector<int64_t> cstart(ncell + 1, 0);
        std::vector<int32_t> order(n);
        {
            std::vector<int64_t> cid(n);
            for (int64_t i = 0; i < n; ++i) {
                int c[3];
                cell_of(i, c);
                cid[i] = lin(c);
                cstart[cid[i] + 1]++;
            }
            for (int64_t c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
            std::vector<int64_t> pos(cstart.begin(), cstart.end() - 1);
            for (int64_t i = 0; i < n; ++i) order[pos[cid[i]]++] = (int32_t)i;
        }
        std::vector<int32_t> src((size_t)n * knn * 2), dst((size_t)n * knn * 2);
        const double cw = 1.0 / g;
#pragma omp parallel
        {
            std::vector<std::pair<double, int32_t>> best;
            best.reserve(knn + 1);
#pragma omp for schedule(dynamic, 1024)
            for (int64_t i = 0; i < n; ++i) {
                best.clear();
                int c[3];
                cell_of(i, c);
                const double *pi = &pts[(size_t)i * dim];
                for (int ring = 0;; ++ring) {
                    // visit cells at Chebyshev distance exactly `ring`
                    int lo[3], hi[3];
                    for (int d = 0; d < dim; ++d) {
                        lo[d] = c[d] - ring;
                        hi[d] = c[d] + ring;
                    }
                    int cc[3];
                    bool any_cell = false;
                    for (cc[0] = std::max(0, lo[0]); cc[0] <= std::min(g - 1, hi[0]); ++cc[0])
                        for (cc[1] = std::max(0, lo[1]); cc[1] <= std::min(g - 1, hi[1]); ++cc[1])
                            for (cc[2] = (dim == 3 ? std::max(0, lo[2]) : 0); cc[2] <= (dim == 3 ? std::min(g - 1, hi[2]) : 0);
                                 ++cc[2]) {
                                bool on_shell = false;
                                for (int d = 0; d < dim; ++d)
                                    if (cc[d] == lo[d] || cc[d] == hi[d]) on_shell = true;
                                if (!on_shell) continue;
                                any_cell = true;
                                int64_t L = lin(cc);
                                for (int64_t s = cstart[L]; s < cstart[L + 1]; ++s) {
                                    int32_t j = order[s];
                                    if (j == i) continue;
                                    double d2 = 0;
                                    for (int d = 0; d < dim; ++d) {
                                        double t = pts[(size_t)j * dim + d] - pi[d];
                                        d2 += t * t;
                                    }
                                    std::pair<double, int32_t> cand(d2, j);
                                    if ((int)best.size() < knn) {
                                        best.push_back(cand);
                                        std::push_heap(best.begin(), best.end());
                                    } else if (cand < best.front()) {
                                        std::pop_heap(best.begin(), best.end());
                                        best.back() = cand;
                                        std::push_heap(best.begin(), best.end());
                                    }
                                }
                            }
                    // all points outside the visited block are farther than ring*cw from p
                    if ((int)best.size() == knn && best.front().first <= (ring * cw) * (ring * cw)) break;
                    if (!any_cell && ring > g) break;
                }
                for (int t = 0; t < knn; ++t) {
                    size_t o = ((size_t)i * knn + t) * 2;
                    src[o] = (int32_t)i;
                    dst[o] = best[t].second;
                    src[o + 1] = best[t].second;
                    dst[o + 1] = (int32_t)i;
                }
            }
        }
        *out = csr_from_arcs(n, src, dst);
        return 0;
    } catch (const std::bad_alloc &) {
        g_err = "knn: out of host memory";
        return 2;
    }
}

int dmolp_gen_ba(int64_t n, int m, uint64_t seed, dmolp_csr **out) {
    try {
        if (m < 1 || n <= m || n > (int64_t(1) << 31) - 1) {
            g_err = "ba: bad parameters";
            return 1;
        }
        Rng r(seed, 0);
        // endpoint list: a vertex appears once per incident edge, so uniform picks are degree-proportional
        std::vector<int32_t> ends;
        ends.reserve((size_t)2 * n * m);
        std::vector<int32_t> src, dst;
        src.reserve((size_t)2 * n * m);
        dst.reserve((size_t)2 * n * m);
        auto add = [&](int32_t u, int32_t v) {
            src.push_back(u);
            dst.push_back(v);
            src.push_back(v);
            dst.push_back(u);
            ends.push_back(u);
            ends.push_back(v);
        };
        // seed graph: a clique on m+1 vertices
        for (int32_t u = 0; u <= m; ++u)
            for (int32_t v = u + 1; v <= m; ++v) add(u, v);
        std::vector<int32_t> pick;
        for (int64_t u = m + 1; u < n; ++u) {
            pick.clear();
            while ((int)pick.size() < m) {
                int32_t v = ends[r.below(ends.size())];
                if (std::find(pick.begin(), pick.end(), v) == pick.end()) pick.push_back(v);
            }
            for (int32_t v : pick) add((int32_t)u, v);
        }
        *out = csr_from_arcs(n, src, dst);
        return 0;
    } catch (const std::bad_alloc &) {
        g_err = "ba: out of host memory";
        return 2;
    }
}

int dmolp_gen_band(int64_t n, int wmin, int wmax, uint64_t seed, dmolp_csr **out) {
    try {
        if (n < 3 || n > (int64_t(1) << 31) - 1 || wmin < 1 || wmax < wmin || 2 * (int64_t)wmax >= n) {
            g_err = "band: bad parameters";
            return 1;
        }
        // vertex i on a cycle of n, with a reach w_i uniform in [wmin, wmax]; i ~ j when their distance on
        // the cycle is at most max(w_i, w_j) (symmetric); rows come out sorted
        std::vector<int32_t> w((size_t)n);
        Rng r(seed, 0);
        for (int64_t i = 0; i < n; ++i) w[(size_t)i] = wmin + (int32_t)r.below((uint64_t)(wmax - wmin + 1));
        dmolp_csr *g = new dmolp_csr();
        g->nv = n;
        g->off.assign((size_t)n + 1, 0);
        // the candidates of i, ascending: distances up to wmax on both sides, as one or two id ranges
        auto visit = [&](int64_t i, auto f) {
            const int64_t lo = i - wmax, hi = i + wmax;
            auto range = [&](int64_t a, int64_t b) {  // ids a..b (inclusive), all in [0, n)
                for (int64_t j = a; j <= b; ++j) {
                    if (j == i) continue;
                    int64_t d = j > i ? j - i : i - j;
                    if (n - d < d) d = n - d;
                    if (d <= std::max(w[(size_t)i], w[(size_t)j])) f((int32_t)j);
                }
            };
            if (lo < 0) {
                range(0, hi);
                range(lo + n, n - 1);
            } else if (hi >= n) {
                range(0, hi - n);
                range(lo, n - 1);
            } else {
                range(lo, hi);
            }
        };
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < n; ++i) {
            int64_t c = 0;
            visit(i, [&](int32_t) { ++c; });
            g->off[(size_t)i + 1] = c;
        }
        for (int64_t i = 0; i < n; ++i) g->off[(size_t)i + 1] += g->off[(size_t)i];
        g->col.resize((size_t)g->off[(size_t)n]);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < n; ++i) {
            int32_t *dst = g->col.data() + g->off[(size_t)i];
            visit(i, [&](int32_t j) { *dst++ = j; });
        }
        *out = g;
        return 0;
    } catch (const std::bad_alloc &) {
        g_err = "band: out of host memory";
        return 2;
    }
}

int dmolp_csr_from_arrays(int64_t nv, int64_t narcs, const int64_t *off, const int32_t *col, dmolp_csr **out) {
    try {
        dmolp_csr *g = new dmolp_csr();
        g->nv = nv;
        g->off.assign(off, off + nv + 1);
        g->col.assign(col, col + narcs);
        *out = g;
        return 0;
    } catch (const std::bad_alloc &) {
        g_err = "csr: out of host memory";
        return 2;
    }
}

int64_t dmolp_csr_nv(const dmolp_csr *g) { return g ? g->nv : -1; }
int64_t dmolp_csr_narcs(const dmolp_csr *g) { return g ? (int64_t)g->col.size() : -1; }

int dmolp_csr_copy(const dmolp_csr *g, int64_t *off, int32_t *col) {
    if (!g) return 1;
    if (off) std::memcpy(off, g->off.data(), sizeof(int64_t) * g->off.size());
    if (col && !g->col.empty()) std::memcpy(col, g->col.data(), sizeof(int32_t) * g->col.size());
    return 0;
}

void dmolp_csr_free(dmolp_csr *g) { delete g; }

// Writes the reference's adjacency text (init.cpp:25-100): first line V, then line i+1 holds vertex i's
// neighbours separated by single spaces, no leading space, every line newline-terminated.
int dmolp_csr_write_adjtext(const dmolp_csr *g, const char *path) {
    FILE *f = fopen(path, "wb");
    if (!f) {
        g_err = std::string("cannot open ") + path;
        return 1;
    }
    fprintf(f, "%lld\n", (long long)g->nv);
    const int64_t block = 1 << 16;
    const int64_t nb = (g->nv + block - 1) / block;
    const int nt = omp_get_max_threads();
    for (int64_t b0 = 0; b0 < nb; b0 += nt) {
        std::vector<std::string> bufs(nt);
#pragma omp parallel for schedule(static, 1)
        for (int t = 0; t < nt; ++t) {
            int64_t b = b0 + t;
            if (b >= nb) continue;
            std::string &s = bufs[t];
            char tmp[16];
            for (int64_t v = b * block; v < std::min(g->nv, (b + 1) * block); ++v) {
                for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e) {
                    int len = snprintf(tmp, sizeof(tmp), e == g->off[v] ? "%d" : " %d", g->col[e]);
                    s.append(tmp, len);
                }
                s.push_back('\n');
            }
        }
        for (int t = 0; t < nt; ++t)
            if (!bufs[t].empty() && fwrite(bufs[t].data(), 1, bufs[t].size(), f) != bufs[t].size()) {
                fclose(f);
                g_err = "short write";
                return 1;
            }
    }
    fclose(f);
    return 0;
}

}  // extern "C"
