// Hub list of phase 1 (src/phase1/init.cpp:139-177) with the reference's exact sort order, computed on all
// host threads.
//
// find_hub_nodes sorts (vertex, degree) pairs by degree with std::sort, which is not stable: among equal
// degrees the order it leaves depends on every step of libstdc++'s introsort, and that order decides which of
// two equal-degree hubs seeding picks first.  This file restates that published algorithm step for step
// (median-of-three pivot moved to the front, unguarded Hoare partition, a depth limit of 2*floor(log2 n) with
// heapsort below it, ranges of at most 16 left to a final insertion pass) so that the permutation is the same,
// and runs it in parallel where the algorithm itself is independent:
//   * after a partition, the two sides are sorted without looking at each other: large right sides become
//     OpenMP tasks;
//   * the final insertion pass never moves an element left of a position p with max(a[0..p)) <= min(a[p..n)),
//     so the array is cut at such positions and the pieces are finished in parallel.
// The hub list needs only the top of that order (the number of hubs is known before sorting), so it sorts
// only the ranges that reach the top; find_first_seed's loop is evaluated from its closed form.
// tests/test_hubsort.py checks the permutation against std::sort itself on tie-heavy and adversarial inputs,
// the hub lists against the oracle and the first seed against the reference's loop.
#include <omp.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <memory>
#include <new>
#include <utility>
#include <vector>

#include "../../include/dmolp_b200.h"

namespace {

using Pair = std::pair<int32_t, int32_t>;  // (vertex, degree), ordered by degree only
constexpr int64_t kSmall = 16;             // ranges this short are left to the final insertion pass
constexpr int64_t kTaskMin = 1 << 15;      // right sides at least this long become tasks
constexpr int64_t kParallelMin = 1 << 18;  // shorter inputs are sorted on the calling thread

inline bool less(const Pair &a, const Pair &b) { return a.second < b.second; }

// ---- heapsort, used below the depth limit ----
void sift_up(Pair *a, int64_t hole, int64_t top, Pair v) {
    int64_t parent = (hole - 1) / 2;
    while (hole > top && less(a[parent], v)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

void sift_down(Pair *a, int64_t hole, int64_t len, Pair v) {
    const int64_t top = hole;
    int64_t child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (less(a[child], a[child - 1])) --child;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    sift_up(a, hole, top, v);
}

void heapsort(Pair *a, int64_t len) {
    if (len >= 2) {  // build the heap
        for (int64_t parent = (len - 2) / 2;; --parent) {
            sift_down(a, parent, len, a[parent]);
            if (parent == 0) break;
        }
    }
    for (int64_t last = len; last > 1;) {  // pop the maximum to the back
        --last;
        const Pair v = a[last];
        a[last] = a[0];
        sift_down(a, 0, last, v);
    }
}

// ---- quicksort steps ----
void median_to_front(Pair *res, Pair *x, Pair *y, Pair *z) {
    if (less(*x, *y)) {
        if (less(*y, *z)) std::swap(*res, *y);
        else if (less(*x, *z)) std::swap(*res, *z);
        else std::swap(*res, *x);
    } else if (less(*x, *z)) {
        std::swap(*res, *x);
    } else if (less(*y, *z)) {
        std::swap(*res, *z);
    } else {
        std::swap(*res, *y);
    }
}

// Hoare's partition pairs the k-th element from the left that is not below the pivot with the k-th element
// from the right that is not above it, swapping pairs until the two scans meet.  While the scanned regions
// are a block apart, that pairing is computed here from 64-element bitmasks (no data-dependent branches);
// the scalar loop then resumes right after the last swapped pair, exactly where it would have been.
constexpr int64_t kBlockLen = 64;

Pair *block_pairs(Pair *lo0, Pair *hi0, int32_t pv, Pair **hi_out) {
    Pair *lf = lo0, *rf = hi0;      // next unscanned position from the left; scanned region from the right
    Pair *last_l = nullptr, *last_r = nullptr;
    uint64_t lm = 0, rm = 0;        // pending offenders: bit i = lbase + i;  bit j = rtop - 1 - j
    Pair *lbase = lf, *rtop = rf;
    for (;;) {
        if (!lm) {
            if (rf - lf < 2 * kBlockLen) break;
            lbase = lf;
            for (int i = 0; i < kBlockLen; ++i) lm |= (uint64_t)(lf[i].second >= pv) << i;
            lf += kBlockLen;
        }
        if (!rm) {
            if (rf - lf < kBlockLen) break;
            rtop = rf;
            for (int j = 0; j < kBlockLen; ++j) rm |= (uint64_t)(rf[-1 - j].second <= pv) << j;
            rf -= kBlockLen;
        }
        while (lm && rm) {
            Pair *x = lbase + __builtin_ctzll(lm), *y = rtop - 1 - __builtin_ctzll(rm);
            std::swap(*x, *y);
            last_l = x;
            last_r = y;
            lm &= lm - 1;
            rm &= rm - 1;
        }
    }
    *hi_out = last_r ? last_r : hi0;
    return last_l ? last_l + 1 : lo0;
}

Pair *partition_around_front(Pair *first, Pair *last) {
    Pair *mid = first + (last - first) / 2;
    median_to_front(first, first + 1, mid, last - 1);
    const Pair *pivot = first;
    Pair *lo = first + 1, *hi = last;
    if (last - first > 4 * kBlockLen) lo = block_pairs(first + 1, last, first->second, &hi);
    for (;;) {
        while (less(*lo, *pivot)) ++lo;
        --hi;
        while (less(*pivot, *hi)) --hi;
        if (!(lo < hi)) return lo;
        std::swap(*lo, *hi);
        ++lo;
    }
}

// `spawn`: inside sort_by_degree's own parallel region, whose closing barrier waits for the tasks.  Anywhere
// else (in particular inside a caller's parallel loop, where a task would outlive the call) it stays false.
void introsort_loop(Pair *first, Pair *last, int64_t depth, bool spawn) {
    while (last - first > kSmall) {
        if (depth == 0) {
            heapsort(first, last - first);
            return;
        }
        --depth;
        Pair *cut = partition_around_front(first, last);
        if (spawn && last - cut >= kTaskMin) {
#pragma omp task firstprivate(cut, last, depth)
            introsort_loop(cut, last, depth, true);
        } else {
            introsort_loop(cut, last, depth, spawn);
        }
        last = cut;
    }
}

// ---- final insertion pass ----
void linear_insert(Pair *pos) {  // unguarded: some element to the left is not greater
    const Pair v = *pos;
    Pair *prev = pos - 1;
    while (less(v, *prev)) {
        *pos = *prev;
        pos = prev;
        --prev;
    }
    *pos = v;
}

void guarded_insertion(Pair *first, Pair *last) {
    if (first == last) return;
    for (Pair *i = first + 1; i != last; ++i) {
        if (less(*i, *first)) {
            const Pair v = *i;
            std::move_backward(first, i, i + 1);
            *first = v;
        } else {
            linear_insert(i);
        }
    }
}

int lg(int64_t n) {
    int b = 0;
    while (n > 1) {
        n >>= 1;
        ++b;
    }
    return b;
}

// std::sort's final insertion pass over a[0..n) once the loop has run on all of it.
void final_insertion(Pair *a, int64_t n, int T) {
    if (n <= kSmall) {
        guarded_insertion(a, a + n);
        return;
    }
    guarded_insertion(a, a + kSmall);
    if (T == 1) {
        for (Pair *i = a + kSmall; i != a + n; ++i) linear_insert(i);
        return;
    }
    // Cut points p with max(a[0..p)) <= min(a[p..n)): no element moves left across them, and a piece that
    // starts at one sorts the same way on its own (its insertions stop at p either way).  After the loop every
    // range is either sorted (heapsort) or at most kSmall long with all of it between its neighbours, so it
    // suffices that the kSmall elements before p are not above the kSmall elements from p on.
    auto safe = [&](int64_t p) {
        int32_t left = INT32_MIN, right = INT32_MAX;
        for (int64_t i = std::max<int64_t>(0, p - kSmall); i < p; ++i) left = std::max(left, a[i].second);
        for (int64_t i = p; i < std::min(n, p + kSmall); ++i) right = std::min(right, a[i].second);
        return left <= right;
    };
    const int64_t step = std::max<int64_t>(n / (8 * (int64_t)T), 4096);
    std::vector<int64_t> cuts{kSmall};
    for (int64_t p = kSmall + step; p < n; p += step) {
        int64_t q = p;
        while (q < n && !safe(q)) ++q;
        if (q < n && q > cuts.back()) cuts.push_back(q);
        p = std::max(p, q);
    }
    cuts.push_back(n);
    const int64_t pieces = (int64_t)cuts.size() - 1;
#pragma omp parallel for num_threads(T) schedule(dynamic, 1)
    for (int64_t s = 0; s < pieces; ++s) {
        if (s == 0) {  // continues the sorted first kSmall elements
            for (Pair *i = a + cuts[0]; i != a + cuts[1]; ++i) linear_insert(i);
        } else {       // never reads left of its start
            guarded_insertion(a + cuts[s], a + cuts[s + 1]);
        }
    }
}

int threads_for(int64_t n) { return n >= kParallelMin && !omp_in_parallel() ? std::max(1, omp_get_max_threads()) : 1; }

// Only the top of the order: the ranges of the loop that reach position t0 or beyond, none that end below
// it.  The ranges of introsort are independent (a range is partitioned by the same steps whatever happens
// beside it), and every range's left side holds no degree above its right side's, so skipping the ranges
// that end at or below t0 changes nothing at or above t0.  [first, last) holds t0 on entry; on return
// *leaf is the start of the last range that held t0 (a partition cut, or a heapsorted or short range).
void top_loop(Pair *first, Pair *last, int64_t depth, const Pair *t0, Pair **leaf, bool spawn) {
    while (last - first > kSmall) {
        if (depth == 0) {
            heapsort(first, last - first);
            break;
        }
        --depth;
        Pair *cut = partition_around_front(first, last);
        if (cut <= t0) {  // t0 is in the right side: the left side [first, cut) lies below t0
            first = cut;
            continue;
        }
        if (spawn && last - cut >= kTaskMin) {  // the right side lies above t0: needed whole
#pragma omp task firstprivate(cut, last, depth)
            introsort_loop(cut, last, depth, true);
        } else {
            introsort_loop(cut, last, depth, spawn);
        }
        last = cut;
    }
    *leaf = first;
}

}  // namespace

namespace dmolp {

// The permutation std::sort(a, a + n, by degree) leaves, computed in parallel for large n.
void sort_by_degree(Pair *a, int64_t n) {
    if (n <= 1) return;
    const int T = threads_for(n);
    if (T > 1) {
#pragma omp parallel num_threads(T)
#pragma omp single
        introsort_loop(a, a + n, 2 * (int64_t)lg(n), true);
    } else {
        introsort_loop(a, a + n, 2 * (int64_t)lg(n), false);
    }
    final_insertion(a, n, T);
}

// a[t0..n) as std::sort(a, a + n, by degree) leaves it; a[0..t0) holds the rest in some order.  From the
// start of the last range that held t0 (a point no element crosses: nothing left of it is above anything
// right of it) the final insertion pass runs as std::sort's does; when nothing was skipped it is the full one.
void top_by_degree(Pair *a, int64_t n, int64_t t0) {
    if (n <= 1 || t0 >= n) return;
    if (t0 <= 0) {
        sort_by_degree(a, n);
        return;
    }
    const int T = threads_for(n);
    Pair *leaf = a;
    if (T > 1) {
#pragma omp parallel num_threads(T)
#pragma omp single
        top_loop(a, a + n, 2 * (int64_t)lg(n), a + t0, &leaf, true);
    } else {
        top_loop(a, a + n, 2 * (int64_t)lg(n), a + t0, &leaf, false);
    }
    if (leaf == a) {
        final_insertion(a, n, T);
        return;
    }
    for (Pair *i = leaf; i != a + n; ++i) linear_insert(i);  // a[leaf-1] is not above anything right of it
}

// find_hub_nodes (init.cpp:139-177) on pairs in the reference's map order.  The reference sorts them all,
// accumulates the sorted degrees in a double, left to right (init.cpp:145-160), and takes vertices from the
// top down while (i + 1) / N is past the x-intercept of the Lorenz curve's last segment.  Every partial sum
// of non-negative integers below 2^53 is exact in a double, so the integer total and the largest degree give
// the same bits, and the number of hubs H follows from them before any sorting: only the top H places of
// std::sort's order are computed (top_by_degree), not the whole order.
std::vector<int> hubs_of_pairs(Pair *sd, int64_t n) {
    const int N = (int)n;
    std::vector<int> hubs;
    if (N < 2) return hubs;
    int64_t total_i = 0;
    int32_t dmax = INT32_MIN;
#pragma omp parallel for reduction(+ : total_i) reduction(max : dmax) schedule(static) \
    if (N >= kParallelMin && !omp_in_parallel())
    for (int i = 0; i < N; ++i) {
        total_i += sd[i].second;
        dmax = std::max(dmax, sd[i].second);
    }
    const double total = (double)total_i;
    const double y1 = (double)total_i / total, y0 = (double)(total_i - dmax) / total;
    const double inv_n = 1.0 / N;
    const double x1 = N * inv_n;
    const double x0 = (N - 1) * inv_n;
    const double slope = (y1 - y0) / (x1 - x0);
    const double x_int = x1 - y1 / slope;
    int H = 0;
    for (int i = N - 1; i >= 0; --i) {
        if ((i + 1) * inv_n > x_int) ++H;
        else break;
    }
    if (H == 0) return hubs;
    top_by_degree(sd, n, n - H);
    for (int i = N - 1; i >= N - H; --i) hubs.push_back(sd[i].first);
    return hubs;
}

// find_hub_nodes on pairs in the reference's map order.
std::vector<int> hubs_from_pairs(std::vector<Pair> sd) { return hubs_of_pairs(sd.data(), (int64_t)sd.size()); }

// find_hub_nodes on the raw degrees of one rank: the pairs (v, degree[v]) in the order the reference's
// degree map iterates, vertex V-1 down to 0, are written on all threads into storage that is not zeroed
// first (building the 32 MB of pairs of 4 M vertices on one thread was mostly first-touch page faults), then
// cut as above.
std::vector<int> hubs_from_degrees(const int32_t *degree, int64_t nv) {
    struct Release {
        void operator()(Pair *p) const { ::operator delete(p); }
    };
    std::unique_ptr<Pair, Release> buf(static_cast<Pair *>(::operator new((size_t)std::max<int64_t>(nv, 1) * sizeof(Pair))));
    Pair *sd = buf.get();
#pragma omp parallel for schedule(static) if (nv >= kParallelMin && !omp_in_parallel())
    for (int64_t i = 0; i < nv; ++i) new (sd + i) Pair((int32_t)(nv - 1 - i), degree[nv - 1 - i]);
    return hubs_of_pairs(sd, nv);  // Pair is trivially destructible: the storage is released as it is
}

// find_first_seed (init.cpp:179-187) over the same order, V-1 down to 0, from (-1, -1): the best pair is
// replaced by a larger degree, or by an equal degree whose vertex id is below the best DEGREE (the
// reference's tie test compares an id with a degree).  With D the largest degree and v1 the highest vertex of
// degree D, the loop holds v1 from there on, then every later (lower) vertex of degree D with id < D: it ends
// at the lowest vertex of degree D with id < D, or at v1 when there is none, and at (-1, -1) when D < 0 or
// there are no vertices.  Both come from two parallel passes.
std::pair<int, int> first_seed_of(const int32_t *degree, int64_t nv) {
    const bool par = nv >= kParallelMin && !omp_in_parallel();
    int32_t D = INT32_MIN;
#pragma omp parallel for reduction(max : D) schedule(static) if (par)
    for (int64_t v = 0; v < nv; ++v) D = std::max(D, degree[v]);
    if (nv == 0 || D < 0) return std::make_pair(-1, -1);
    int64_t v1 = -1, u = INT64_MAX;
#pragma omp parallel for reduction(max : v1) reduction(min : u) schedule(static) if (par)
    for (int64_t v = 0; v < nv; ++v)
        if (degree[v] == D) {
            v1 = std::max(v1, v);
            if (v < (int64_t)D) u = std::min(u, v);
        }
    return std::make_pair((int)(u != INT64_MAX ? u : v1), (int)D);
}

}  // namespace dmolp

extern "C" {

int dmolp_degree_order(int64_t n, int32_t *ids, int32_t *degrees) {
    if (n < 0 || (n > 0 && (!ids || !degrees))) return DMOLP_ERR_ARG;
    std::vector<Pair> a(n);
    for (int64_t i = 0; i < n; ++i) a[i] = Pair(ids[i], degrees[i]);
    dmolp::sort_by_degree(a.data(), n);
    for (int64_t i = 0; i < n; ++i) {
        ids[i] = a[i].first;
        degrees[i] = a[i].second;
    }
    return DMOLP_OK;
}

int dmolp_find_hubs(int64_t nv, const int32_t *raw_degree, int32_t *hubs, int64_t *nhubs, int32_t *first_seed,
                    int32_t *first_seed_degree) {
    if (nv < 0 || nv > 0x7fffffff || (nv > 0 && (!raw_degree || !hubs)) || !nhubs || !first_seed ||
        !first_seed_degree)
        return DMOLP_ERR_ARG;
    const std::vector<int> h = dmolp::hubs_from_degrees(raw_degree, nv);
    std::copy(h.begin(), h.end(), hubs);
    *nhubs = (int64_t)h.size();
    const std::pair<int, int> f = dmolp::first_seed_of(raw_degree, nv);
    *first_seed = f.first;
    *first_seed_degree = f.second;
    return DMOLP_OK;
}

int dmolp_find_hubs_pairs(int64_t n, const int32_t *ids, const int32_t *degrees, int32_t *hubs, int64_t *nhubs) {
    if (n < 0 || n > 0x7fffffff || (n > 0 && (!ids || !degrees || !hubs)) || !nhubs) return DMOLP_ERR_ARG;
    std::vector<Pair> a(n);
    for (int64_t i = 0; i < n; ++i) a[i] = Pair(ids[i], degrees[i]);
    const std::vector<int> h = dmolp::hubs_from_pairs(std::move(a));
    std::copy(h.begin(), h.end(), hubs);
    *nhubs = (int64_t)h.size();
    return DMOLP_OK;
}

}  // extern "C"
