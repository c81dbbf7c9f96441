"""The plain path at its benchmark size: R-MAT scale 22, edge factor 16, seed 7 (4.19 M vertices, 128 M arcs).

Every LP iteration of the benchmarked runs (k = 32, and k = 16 and 64, 30 iterations each) is held to the
reference's own outputs on this graph (tests/golden/rmat22_full.json, written by make_golden_full.py from the
reference's phase-2 steps started from the oracle's phase-1 labels): per iteration the window's size and
order-independent checksum, the candidates, the changes, the edge cut, the part counts, the penalty bits and
the traversed-edge terms, then the final labels' hash, cut and balances.  The oracle also pins phase 1 and the
first iterations directly, and properties that hold at any size check the 30-iteration run once more: the
reported cut and part sizes equal a recount from the final labels and the full statistics pass, a rerun
repeats itself exactly, and under the reference's 32-label cap (k = 64) no vertex moves to a label >= 32."""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, f64_hex

pytestmark = pytest.mark.gpu

FULL = os.path.join(GOLDEN, "rmat22_full.json")


@pytest.fixture(scope="module")
def setup():
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import Partitioner

    g = graphs.rmat(22, 16, 0.57, 0.19, 0.19, seed=7)
    p = Partitioner(0)
    p.upload(g)
    src = np.repeat(np.arange(g.num_vertices, dtype=np.int32), np.diff(g.offsets))
    yield g, p, src
    p.close()


def recount(g, src, labels, k):
    """Edge cut, vertex counts and intra-part edges of a labelling, in numpy."""
    a, b = labels[src], labels[g.indices]
    same = a == b
    cut = int((~same).sum()) // 2
    vc = np.bincount(labels, minlength=k).astype(np.int64)
    ec = np.bincount(a[same], minlength=k).astype(np.int64) // 2
    return cut, vc, ec


def test_phase1_and_first_iterations_match_oracle(setup):
    g, p, _ = setup
    m1 = p.phase1(32, 10000)
    o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), 32, 10000)
    lab1 = p.labels()
    assert m1.seeds == o1.seeds.tolist() and m1.rounds == o1.res.rounds
    assert np.array_equal(lab1, o1.labels)
    assert m1.initial_edge_cut == o1.res.initial_edge_cut
    r = p.phase2(32, mode="fixed", iterations=2, records=False)
    o2 = oracle.phase2(g.offsets, g.indices, o1.labels, 32, "fixed", 2)
    assert np.array_equal(p.labels(), o2.labels)
    assert r.edge_cut == o2.res.edge_cut and r.traversed_edges == o2.res.te_total


def test_thirty_iterations_recount_and_repeat(setup):
    g, p, src = setup
    p.phase1(32, 10000)
    lab1 = p.labels()
    p.lib.dmolp_labels_save(p.ctx)
    r = p.phase2(32, mode="fixed", iterations=30, records=False)
    lab = p.labels()
    assert lab.min() >= 0 and lab.max() < 32
    cut, vc, ec = recount(g, src, lab, 32)
    assert r.edge_cut == cut
    mc, mvc, mec = p.metrics(32)  # the full statistics pass on the same labels
    assert mc == cut and np.array_equal(mvc, vc) and np.array_equal(mec, ec)
    assert int(vc.sum()) == g.num_vertices and int(ec.sum()) + cut == g.num_arcs // 2
    p._check(p.lib.dmolp_labels_restore(p.ctx))
    assert np.array_equal(p.labels(), lab1)
    r2 = p.phase2(32, mode="fixed", iterations=30, records=False)
    assert np.array_equal(p.labels(), lab) and r2.edge_cut == r.edge_cut
    assert r2.traversed_edges == r.traversed_edges


def test_label_cap_at_k64(setup):
    g, p, src = setup
    p.phase1(64, 10000)
    before = p.labels()
    r = p.phase2(64, mode="fixed", iterations=10, cap="ref", records=False)
    after = p.labels()
    moved = after != before
    assert moved.any()
    assert after[moved].max() < 32  # only the first min(k, 32) labels are scored (gpu_lp_boundary.cu:360)
    assert r.edge_cut == recount(g, src, after, 64)[0]


@pytest.mark.parametrize("k", [32, 16, 64])
def test_every_iteration_matches_reference(setup, k):
    g, p, _ = setup
    gold = json.load(open(FULL))[f"k{k}"]
    assert (gold["num_vertices"], gold["num_arcs"]) == (g.num_vertices, g.num_arcs)
    m1 = p.phase1(k, gold["theta"])
    assert "%016x" % oracle.fnv1a(p.labels()) == gold["labels1_hash"]
    assert m1.initial_edge_cut == gold["phase1_initial_edge_cut"] and m1.seeds == gold["phase1_seeds"]
    m = p.phase2(k, mode="fixed", iterations=gold["iters"])
    pen, cnt = p.history(k, gold["iters"])
    assert len(m.records) == len(gold["trace"]) == gold["iters"]
    for i, t in enumerate(gold["trace"]):
        r = m.records[i]
        assert (r.window, "%016x" % r.window_sum) == (t["window"], t["window_sum"]), (k, i + 1)
        assert (r.candidates, r.changes, r.edge_cut) == (t["candidates"], t["changes"], t["edge_cut"]), (k, i + 1)
        assert [r.te_prev, r.te_cand, r.te_sel, r.te_stats] == t["te"], (k, i + 1)
        assert [f64_hex(x) for x in pen[i]] == t["penalty"], (k, i + 1)
        assert cnt[i][:k].tolist() == t["vertex_counts"] and cnt[i][k:].tolist() == t["edge_counts"], (k, i + 1)
    assert "%016x" % oracle.fnv1a(p.labels()) == gold["labels2_hash"] == gold["trace"][-1]["labels_hash"]
    res = gold["result"]
    assert m.edge_cut == res["edge_cut"] and m.traversed_edges == res["te_total"]
    assert f64_hex(m.vertex_balance) == res["vertex_balance"] and f64_hex(m.edge_balance) == res["edge_balance"]
