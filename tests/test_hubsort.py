"""The hub sort of phase 1 (find_hub_nodes, src/phase1/init.cpp:139-177): the library's parallel restatement
of introsort must leave exactly the permutation this toolchain's std::sort leaves (the oracle calls std::sort
itself), ties included, on inputs that exercise every part of the algorithm; the hub lists must agree too."""
import sys

import numpy as np
import pytest

import oracle
from dmolp_b200 import cabi
from dmolp_b200._native import core


def lib_order(ids, deg):
    i = np.ascontiguousarray(ids, np.int32).copy()
    d = np.ascontiguousarray(deg, np.int32).copy()
    assert core().dmolp_degree_order(i.shape[0], i.ctypes.data, d.ctypes.data) == cabi.DMOLP_OK
    return i, d


def cases():
    rng = np.random.default_rng(11)
    out = []
    for n in (0, 1, 2, 3, 15, 16, 17, 33, 100, 1000, 5000):
        out.append(("few-keys-%d" % n, rng.integers(0, 4, n)))
        out.append(("wide-%d" % n, rng.integers(0, 1 << 20, n)))
    for n in (300_000, 1_200_000):  # the parallel path (tasks, cut points)
        out.append(("powerlaw-%d" % n, np.minimum((rng.pareto(1.2, n) * 3).astype(np.int64), 1 << 20)))
        out.append(("few-keys-%d" % n, rng.integers(0, 8, n)))
        out.append(("sorted-%d" % n, np.sort(rng.integers(0, 1000, n))))
        out.append(("reverse-%d" % n, np.sort(rng.integers(0, 1000, n))[::-1].copy()))
        out.append(("constant-%d" % n, np.full(n, 7)))
        saw = np.arange(n) % 977
        out.append(("sawtooth-%d" % n, saw))
        organ = np.concatenate([np.arange(n // 2), np.arange(n - n // 2)[::-1]])
        out.append(("organ-pipe-%d" % n, organ))
    return out


@pytest.mark.parametrize("name,deg", cases(), ids=[c[0] for c in cases()])
def test_degree_order_is_std_sort(name, deg):
    deg = np.asarray(deg, np.int32)
    ids = np.arange(deg.shape[0], dtype=np.int32)[::-1].copy()  # the reference's map order at one rank
    ri, rd = oracle.degree_order(ids, deg)
    li, ld = lib_order(ids, deg)
    assert np.array_equal(rd, ld) and np.array_equal(ri, li), name


def test_hub_lists_match_the_oracle():
    rng = np.random.default_rng(5)
    for n, hi in ((50_000, 30), (400_000, 200), (1_000_000, 12)):
        deg = np.minimum((rng.pareto(1.1, n) * 2).astype(np.int64), hi).astype(np.int32)  # many tied hubs
        ids = np.arange(n, dtype=np.int32)[::-1].copy()  # vertices V-1..0 with their degrees, as the map holds
        pair_deg = deg[::-1].copy()
        h = np.empty(n, np.int32)
        nh = cabi.c_int64()
        import ctypes

        assert core().dmolp_find_hubs_pairs(n, ids.ctypes.data, pair_deg.ctypes.data, h.ctypes.data,
                                            ctypes.byref(nh)) == cabi.DMOLP_OK
        assert np.array_equal(h[:nh.value], oracle.find_hubs(deg))


NESTED = r"""
#include <omp.h>
#include <cstdio>
#include <vector>
#include <random>
#include <algorithm>
#include <cstdint>
extern "C" int dmolp_degree_order(int64_t n, int32_t *ids, int32_t *degrees);
extern "C" int dmolp_find_hubs(int64_t nv, const int32_t *raw_degree, int32_t *hubs, int64_t *nhubs,
                               int32_t *first_seed, int32_t *first_seed_degree);
// hubs and first seed of a skewed degree array (sizes past the parallel threshold when called alone)
static std::vector<int32_t> hub_answer(const std::vector<int32_t> &deg) {
    std::vector<int32_t> h(deg.size() + 2);
    int64_t nh = 0;
    int32_t f = 0, fd = 0;
    if (dmolp_find_hubs((int64_t)deg.size(), deg.data(), h.data(), &nh, &f, &fd) != 0) return {};
    h.resize(nh);
    h.push_back(f);
    h.push_back(fd);
    return h;
}
int main() {
    int bad = 0;
    std::vector<std::vector<int32_t>> degs(12), inside(12);
    for (int g = 0; g < 12; ++g) {
        std::mt19937_64 rng(100 + g);
        degs[g].resize(300000 + rng() % 100000);
        for (auto &d : degs[g]) d = (int32_t)(std::min<uint64_t>(rng() % 1000, rng() % 1000) % (5 + g * 7));
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < 12; ++g) inside[g] = hub_answer(degs[g]);
    for (int g = 0; g < 12; ++g) bad += hub_answer(degs[g]) != inside[g] || inside[g].empty();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
    for (int g = 0; g < 48; ++g) {
        std::mt19937_64 rng(g);
        const int64_t n = 1000 + (int64_t)(rng() % 250000);
        std::vector<int32_t> ids(n), deg(n);
        for (int64_t i = 0; i < n; ++i) { ids[i] = (int32_t)(n - 1 - i); deg[i] = (int32_t)(rng() % 40); }
        std::vector<std::pair<int, int>> p(n);
        for (int64_t i = 0; i < n; ++i) p[i] = {ids[i], deg[i]};
        std::sort(p.begin(), p.end(), [](const std::pair<int, int> &x, const std::pair<int, int> &y) {
            return x.second < y.second; });
        dmolp_degree_order(n, ids.data(), deg.data());
        for (int64_t i = 0; i < n; ++i) bad += p[i].first != ids[i];
    }
    printf("%d\n", bad);
    return 0;
}
"""


def test_degree_order_inside_a_callers_parallel_loop(tmp_path):
    """The batched phase 1 computes many graphs' hubs from inside its own OpenMP loop: the sort must neither
    leave work behind (tasks outliving the call) nor differ from std::sort there, and the hub list and first
    seed found inside the loop must equal the ones found by a call on all threads."""
    import os
    import subprocess

    from dmolp_b200 import build

    src = tmp_path / "nested.cpp"
    src.write_text(NESTED)
    exe = tmp_path / "nested"
    lib = os.path.join(build.LIB)
    subprocess.run([build.CXX, "-O2", "-fopenmp", str(src), "-o", str(exe), "-L" + lib, "-ldmolp_b200",
                    "-Wl,-rpath," + lib], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=300)
    assert out.stdout.strip() == "0"


def literal_first_seed(deg):
    """find_first_seed (src/phase1/init.cpp:179-187) as the reference runs it at one rank: the degree map
    iterated from vertex V-1 down to 0, starting from (-1, -1), with its tie test comparing an id with the best
    degree."""
    best_v, best_d = -1, -1
    for v in range(len(deg) - 1, -1, -1):
        d = int(deg[v])
        if d > best_d or (d == best_d and v < best_d):
            best_v, best_d = v, d
    return best_v, best_d


def lib_find_hubs(deg):
    import ctypes

    deg = np.ascontiguousarray(deg, np.int32)
    n = deg.shape[0]
    h = np.empty(max(n, 1), np.int32)
    nh, f, fd = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
    assert core().dmolp_find_hubs(n, deg.ctypes.data, h.ctypes.data, ctypes.byref(nh), ctypes.byref(f),
                                  ctypes.byref(fd)) == cabi.DMOLP_OK
    return h[:nh.value].copy(), (f.value, fd.value)


def degree_cases():
    rng = np.random.default_rng(23)
    out = [("empty", np.zeros(0, np.int32)), ("one", np.array([5], np.int32)),
           ("zeros", np.zeros(1000, np.int32)), ("all-minus-one", np.full(50, -1, np.int32)),
           ("negative", np.full(100, -3, np.int32))]
    d = np.zeros(2000, np.int32)
    d[[5, 40, 1500, 1900]] = 100  # the largest degree at ids below it (5, 40) and above it: the loop ends at 5
    out.append(("tie-ids-below-degree", d))
    d = np.zeros(2000, np.int32)
    d[[300, 700]] = 50  # every id above the degree: the loop keeps the highest, 700
    out.append(("tie-ids-above-degree", d))
    d = np.ones(5000, np.int32)
    d[[4999, 3, 1]] = 7  # the first one met (4999) is replaced by 3, then by 1
    out.append(("tie-replaced-twice", d))
    for n in (50_000, 300_000, 1_200_000):  # 300 K and up: the parallel paths
        out.append(("powerlaw-%d" % n, np.minimum((rng.pareto(1.1, n) * 2).astype(np.int64), 200).astype(np.int32)))
        out.append(("few-keys-%d" % n, rng.integers(0, 6, n).astype(np.int32)))
    # structured orders (the hub count ranges from a few to every vertex; only the top is sorted)
    n = 300_000
    out.append(("sorted-%d" % n, np.sort(rng.integers(0, 1000, n)).astype(np.int32)))
    out.append(("reverse-%d" % n, np.sort(rng.integers(0, 1000, n))[::-1].astype(np.int32)))
    out.append(("constant-%d" % n, np.full(n, 7, np.int32)))
    out.append(("sawtooth-%d" % n, (np.arange(n) % 977).astype(np.int32)))
    out.append(("organ-pipe-%d" % n, np.concatenate([np.arange(n // 2), np.arange(n - n // 2)[::-1]]).astype(np.int32)))
    d = np.minimum((rng.pareto(1.1, n) * 2).astype(np.int64), 60).astype(np.int32)
    d[rng.integers(0, n, 40)] = 60  # many vertices tied at the largest degree, some of them hubs
    out.append(("tied-top-%d" % n, d))
    return out


@pytest.mark.parametrize("name,deg", degree_cases(), ids=[c[0] for c in degree_cases()])
def test_find_hubs_from_raw_degrees(name, deg):
    """dmolp_find_hubs (the host step of phase 1): the hub list equals the oracle's (std::sort over the map
    order) and the first seed equals the reference's loop, tie test included."""
    hubs, first = lib_find_hubs(deg)
    assert first == literal_first_seed(deg), name
    if deg.shape[0] and deg.min() >= 0:
        assert np.array_equal(hubs, oracle.find_hubs(deg)), name


THREADS = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from tests.test_hubsort import lib_find_hubs
rng = np.random.default_rng(31)
d = np.minimum((rng.pareto(1.1, 1_500_000) * 2).astype(np.int64), 300).astype(np.int32)
h, f = lib_find_hubs(d)
print(len(h), int((h.astype(np.int64) * np.arange(1, len(h) + 1)).sum()), f[0], f[1])
"""


def test_find_hubs_same_at_every_thread_count():
    """The pairs are written and the first seed reduced on however many threads OpenMP gives: the answer must
    not depend on it."""
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = set()
    for t in (1, 3, 16):
        env = dict(os.environ, OMP_NUM_THREADS=str(t))
        r = subprocess.run([sys.executable, "-c", THREADS, root], env=env, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.add(r.stdout.strip())
    assert len(outs) == 1, outs
