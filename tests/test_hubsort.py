"""The hub sort of phase 1 (find_hub_nodes, src/phase1/init.cpp:139-177): the library's parallel restatement
of introsort must leave exactly the permutation this toolchain's std::sort leaves (the oracle calls std::sort
itself), ties included, on inputs that exercise every part of the algorithm; the hub lists must agree too."""
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
int main() {
    int bad = 0;
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
    leave work behind (tasks outliving the call) nor differ from std::sort there."""
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
