"""The oracle (CPU restatement, oracle/dmolp_oracle.cpp) against the reference's own outputs.

The golden fixtures were produced by the reference sources themselves (tests/golden/make_golden.py), so this
file is what pins the oracle; the GPU tests then compare the CUDA path with the oracle and the fixtures.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
from conftest import f64_hex, golden_arrays, golden_graph, initial_labels_for


def _names(golden_cases):
    return sorted(golden_cases)


@pytest.fixture(scope="module")
def cases(golden_cases):
    return golden_cases


def test_graph_generators_unchanged(golden_cases):
    import make_golden

    for name, case in golden_cases.items():
        g = golden_graph(name)
        assert make_golden.graph_hash(g) == case["graph_hash"], name
        assert g.num_vertices == case["num_vertices"] and g.num_arcs == case["num_arcs"]


def test_hubs_match_reference(golden_cases):
    for name, case in golden_cases.items():
        g = golden_graph(name)
        hubs = oracle.find_hubs(g.raw_deg())
        assert "%016x" % oracle.fnv1a(hubs) == case["phase1"]["hubs_hash"], name


def test_phase1_matches_reference(golden_cases):
    checked = 0
    for name, case in golden_cases.items():
        if case["labels_from"] != "phase1":
            continue
        g = golden_graph(name)
        p1 = case["phase1"]
        o = oracle.phase1(g.offsets, g.indices, g.raw_deg(), case["k"], case["theta"])
        assert o.seeds.tolist() == p1["seeds"], name
        assert np.array_equal(o.labels, golden_arrays(name)["labels1"]), name
        assert o.res.initial_edge_cut == p1["initial_edge_cut"]
        assert f64_hex(o.res.initial_vertex_balance) == p1["initial_vertex_balance"]
        assert f64_hex(o.res.initial_edge_balance) == p1["initial_edge_balance"]
        assert o.vertex_counts.tolist() == p1["partition_vertex_counts"]
        assert o.edge_counts.tolist() == p1["partition_edge_counts"]
        checked += 1
    assert checked >= 3


def test_phase2_fixed_matches_reference(golden_cases):
    for name, case in golden_cases.items():
        run = case["runs"].get("fixed")
        if run is None:
            continue
        g = golden_graph(name)
        k = case["k"]
        lab0 = initial_labels_for(name, case, g)
        o = oracle.phase2(g.offsets, g.indices, lab0, k, "fixed", run["iters"])
        assert np.array_equal(o.labels, golden_arrays(name)["labels2_fixed"]), name
        assert o.res.edge_cut == run["result"]["edge_cut"]
        assert f64_hex(o.res.vertex_balance) == run["result"]["vertex_balance"]
        assert f64_hex(o.res.edge_balance) == run["result"]["edge_balance"]
        assert o.res.te_total == run["result"]["te_total"]
        for i, t in enumerate(run["trace"]):
            r = o.records[i]
            assert (r.window, r.changes, r.edge_cut) == (t["window"], t["changes"], t["edge_cut"]), (name, i)
            assert "%016x" % r.window_hash == t["window_hash"], (name, i)
            assert [f64_hex(x) for x in o.penalties[i]] == t["penalty"], (name, i)
            assert o.counts[i][:k].tolist() == t["vertex_counts"] and o.counts[i][k:].tolist() == t["edge_counts"]
            assert [r.te_prev, r.te_cand, r.te_sel, r.te_stats] == t["te"], (name, i)


def test_phase2_ref_mode_matches_reference(golden_cases):
    for name, case in golden_cases.items():
        run = case["runs"].get("ref")
        if run is None:
            continue
        g = golden_graph(name)
        lab0 = initial_labels_for(name, case, g)
        o = oracle.phase2(g.offsets, g.indices, lab0, case["k"], "ref")
        assert np.array_equal(o.labels, golden_arrays(name)["labels2_ref"]), name
        assert o.res.edge_cut == run["result"]["edge_cut"]
        assert f64_hex(o.res.vertex_balance) == run["result"]["vertex_balance"]
        assert f64_hex(o.res.edge_balance) == run["result"]["edge_balance"]
        # one LP call per iteration that reached the GPU step
        assert len(run["trace"]) == run["result"]["hook_calls"]
        assert o.res.iterations_run >= run["result"]["hook_calls"]


def test_lp_decide_tie_rule():
    """Equal penalised scores: the reference's shuffle tree keeps the label whose 5-bit reversed index is
    smallest (16 beats 8, 8 beats 24, ...)."""
    k = 32
    pen = np.zeros(k)
    assert oracle.lp_decide(0, [8, 16, 8, 16], pen, k) == 16
    assert oracle.lp_decide(0, [8, 24, 8, 24], pen, k) == 8
    assert oracle.lp_decide(3, [1, 2], pen, k) == 2      # 1 and 2 tie; reversed(2)=8 < reversed(1)=16
    # a penalty below -1 makes present labels score negative; an absent label (score 0) then has the maximum,
    # which beats the own label only when that one is unscored (>= 32): a move to the absent label 0
    pen2 = np.full(64, -2.0)
    assert oracle.lp_decide(40, [40, 40, 3], pen2, 64) == 0
    assert oracle.lp_decide(5, [5, 5, 7], pen2, 8) == 5  # own raw count 2 > 0
    # k > 32: labels >= 32 are ignored and a vertex labelled >= 32 always moves into [0, 32)
    pen3 = np.zeros(64)
    assert oracle.lp_decide(40, [40, 40, 40, 3], pen3, 64) == 3
    assert oracle.lp_decide(40, [40, 40, 40, 3], pen3, 64, cap="full") == 40


@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
def test_oracle_matches_live_reference_random_small_graphs():
    """Fresh random cases against the reference itself (only where its sources were built)."""
    from dmolp_b200 import graphs

    rng = np.random.default_rng(2024)
    with tempfile.TemporaryDirectory() as td:
        for trial in range(4):
            n = int(rng.integers(300, 1500))
            g = graphs.knn(n, int(rng.integers(2, 4)), int(rng.integers(4, 12)), int(rng.integers(1, 1000)))
            k = int(rng.integers(2, 12))
            theta = int(rng.integers(5, 200))
            txt = os.path.join(td, f"g{trial}.txt")
            graphs.write_adjtext(g, txt)
            r = oracle.run_reference(txt, k, theta, os.path.join(td, f"o{trial}"), mode="fixed", iters=12)
            if "unpinned" in r["phase1"]:
                continue
            o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, theta)
            assert np.array_equal(o1.labels, r["labels1"])
            o2 = oracle.phase2(g.offsets, g.indices, o1.labels, k, "fixed", 12)
            assert np.array_equal(o2.labels, r["labels2"])
            assert o2.res.edge_cut == r["result"]["edge_cut"]
