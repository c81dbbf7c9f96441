"""The plain path at its benchmark size: R-MAT scale 22, edge factor 16, seed 7 (4.19 M vertices, 128 M arcs).

The oracle is affordable here for phase 1 and the first LP iterations, which must agree bit for bit.  For the
full 30-iteration run the test relies on properties that hold at any size: the edge cut and part sizes the
run reports equal a recount from its final labels, the statistics kept incrementally equal the full pass,
a rerun from the same start repeats itself exactly, and under the reference's 32-label cap (k = 64) no vertex
moves to a label of 32 or more."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


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
