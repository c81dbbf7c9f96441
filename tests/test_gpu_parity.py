"""CUDA path (through the C-ABI) against the reference's golden outputs and the oracle.  Bit-exact: labels,
part sizes, edge cut, per-iteration windows/changes/cuts, penalty bits, traversed-edge counts."""
import numpy as np
import pytest

import oracle
from conftest import f64_hex, golden_arrays, golden_graph, initial_labels_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def part():
    from dmolp_b200.partitioner import Partitioner

    p = Partitioner(0)
    yield p
    p.close()


def test_phase1_matches_reference(golden_cases, part):
    for name, case in golden_cases.items():
        g = golden_graph(name)
        part.upload(g)
        m = part.phase1(case["k"], case["theta"])
        o = oracle.phase1(g.offsets, g.indices, g.raw_deg(), case["k"], case["theta"])
        # always equal to the oracle (including seed completion where the reference is undefined)
        assert m.seeds == o.seeds.tolist(), name
        assert np.array_equal(part.labels(), o.labels), name
        assert m.initial_edge_cut == o.res.initial_edge_cut
        assert m.num_seeds_found == o.res.num_seeds and m.rounds == o.res.rounds
        assert m.traversed_edges == o.res.te
        if case["labels_from"] == "phase1":  # and to the reference itself where it is defined
            p1 = case["phase1"]
            assert np.array_equal(part.labels(), golden_arrays(name)["labels1"]), name
            assert m.seeds == p1["seeds"]
            assert f64_hex(m.initial_vertex_balance) == p1["initial_vertex_balance"]
            assert f64_hex(m.initial_edge_balance) == p1["initial_edge_balance"]
            assert m.partition_vertex_counts == p1["partition_vertex_counts"]
            assert m.partition_edge_counts == p1["partition_edge_counts"]


@pytest.mark.parametrize("mode", ["fixed", "ref"])
def test_phase2_matches_reference(golden_cases, part, mode):
    n = 0
    for name, case in golden_cases.items():
        run = case["runs"].get(mode)
        if run is None:
            continue
        g = golden_graph(name)
        k = case["k"]
        part.upload(g)
        part.set_labels(initial_labels_for(name, case, g))
        m = part.phase2(k, mode=mode, iterations=run["iters"])
        assert np.array_equal(part.labels(), golden_arrays(name)[f"labels2_{mode}"]), (name, mode)
        assert m.edge_cut == run["result"]["edge_cut"], name
        assert f64_hex(m.vertex_balance) == run["result"]["vertex_balance"], name
        assert f64_hex(m.edge_balance) == run["result"]["edge_balance"], name
        if mode == "fixed":
            assert m.traversed_edges == run["result"]["te_total"], name
            pen, cnt = part.history(k, m.iterations_run)
            for i, t in enumerate(run["trace"]):
                r = m.records[i]
                assert (r.window, r.changes, r.edge_cut) == (t["window"], t["changes"], t["edge_cut"]), (name, i)
                assert [r.te_prev, r.te_cand, r.te_sel, r.te_stats] == t["te"], (name, i)
                assert r.candidates == t["candidates"], (name, i)
                assert [f64_hex(x) for x in pen[i]] == t["penalty"], (name, i)
                assert cnt[i][:k].tolist() == t["vertex_counts"], (name, i)
                assert cnt[i][k:].tolist() == t["edge_counts"], (name, i)
        else:
            o = oracle.phase2(g.offsets, g.indices, initial_labels_for(name, case, g), k, "ref")
            assert m.iterations_run == o.res.iterations_run and m.stop_reason == o.res.stop_reason, name
        n += 1
    assert n >= 5


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_cases_against_oracle(part, seed):
    """Random graphs, k, labels and both label caps; the uncapped mode has no reference, only the oracle."""
    from dmolp_b200 import graphs

    rng = np.random.default_rng(seed)
    for trial in range(3):
        kind = trial % 3
        if kind == 0:
            g = graphs.knn(int(rng.integers(500, 5000)), int(rng.integers(2, 4)), int(rng.integers(4, 14)),
                           int(rng.integers(1, 10_000)))
        elif kind == 1:
            g = graphs.barabasi_albert(int(rng.integers(500, 5000)), int(rng.integers(2, 8)), int(rng.integers(1, 999)))
        else:
            g = graphs.rmat(int(rng.integers(9, 13)), int(rng.integers(4, 16)), seed=int(rng.integers(1, 999)))
        k = int(rng.choice([2, 3, 7, 16, 31, 32, 33, 48, 64, 100]))
        theta = int(rng.integers(1, 300))
        cap = "full" if rng.random() < 0.4 else "ref"
        part.upload(g)
        m1 = part.phase1(k, theta)
        o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, theta)
        assert np.array_equal(part.labels(), o1.labels)
        assert m1.seeds == o1.seeds.tolist()
        lab0 = o1.labels if rng.random() < 0.5 else rng.integers(0, k, g.num_vertices).astype(np.int32)
        part.set_labels(lab0)
        iters = int(rng.integers(1, 25))
        m2 = part.phase2(k, mode="fixed", iterations=iters, cap=cap)
        o2 = oracle.phase2(g.offsets, g.indices, lab0, k, "fixed", iters, cap=cap)
        assert np.array_equal(part.labels(), o2.labels), (seed, trial, k, cap)
        # per iteration: the window's order-independent checksum, its size and the changes
        assert [(r.window, r.window_sum, r.changes) for r in m2.records] == \
               [(r.window, r.window_sum, r.changes) for r in o2.records], (seed, trial)
        assert m2.edge_cut == o2.res.edge_cut
        assert m2.traversed_edges == o2.res.te_total
        assert f64_hex(m2.vertex_balance) == f64_hex(o2.res.vertex_balance)


def test_metrics_pass(part):
    from dmolp_b200 import graphs

    g = graphs.knn(4000, 3, 10, 77)
    part.upload(g)
    rng = np.random.default_rng(5)
    lab = rng.integers(0, 13, g.num_vertices).astype(np.int32)
    part.set_labels(lab)
    cut, vc, ec = part.metrics(13)
    src = np.repeat(np.arange(g.num_vertices), np.diff(g.offsets))
    diff = lab[src] != lab[g.indices]
    assert cut == int(diff.sum()) // 2
    assert vc.tolist() == np.bincount(lab, minlength=13).tolist()
    same = ~diff
    assert ec.tolist() == (np.bincount(lab[src][same], minlength=13) // 2).tolist()


def test_bad_labels_are_an_error_not_a_fault(part):
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import DmolpError

    g = graphs.knn(500, 2, 6, 3)
    part.upload(g)
    lab = np.zeros(g.num_vertices, np.int32)
    lab[17] = -1  # the reference aborts on a -1 label (phase2.cpp:239-244)
    part.set_labels(lab)
    with pytest.raises(DmolpError) as e:
        part.phase2(4, mode="fixed", iterations=3)
    assert e.value.code == 5
    with pytest.raises(DmolpError):
        part.metrics(4)
    lab[17] = 9  # >= k
    part.set_labels(lab)
    with pytest.raises(DmolpError):
        part.phase2(4, mode="ref")


def test_edge_cases(part):
    from dmolp_b200 import graphs

    # no arcs at all: every vertex isolated; phase 1 dumps the non-seeds into the smallest part
    g = graphs.Graph(np.zeros(11, np.int64), np.zeros(0, np.int32))
    part.upload(g)
    m = part.phase1(3, 5)
    o = oracle.phase1(g.offsets, g.indices, g.raw_deg(), 3, 5)
    assert np.array_equal(part.labels(), o.labels)
    r = part.phase2(3, mode="ref")
    assert r.edge_cut == 0 and r.stop_reason == 1
    # k = 1 and k > V
    g = graphs.knn(50, 2, 4, 1)
    part.upload(g)
    for k in (1, 64):
        part.phase1(k, 10)
        o = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, 10)
        assert np.array_equal(part.labels(), o.labels)
        lab = part.labels()
        part.phase2(k, mode="fixed", iterations=5)
        o2 = oracle.phase2(g.offsets, g.indices, lab, k, "fixed", 5)
        assert np.array_equal(part.labels(), o2.labels)
    # empty graph
    g = graphs.Graph(np.zeros(1, np.int64), np.zeros(0, np.int32))
    part.upload(g)
    part.phase1(2, 1)
    assert part.phase2(2, mode="ref").edge_cut == 0


def test_window_select_and_lp_apply_match_oracle(golden_cases, part):
    """The single-step entry points (the reference's expandBoundaryNodes and runBoundaryLPOnGPU_*) replay
    the golden fixed-mode run iteration by iteration."""
    name = "knn3d_2k"
    case = golden_cases[name]
    g = golden_graph(name)
    k = case["k"]
    part.upload(g)
    lab = initial_labels_for(name, case, g).copy()
    part.set_labels(lab)
    window = np.arange(g.num_vertices, dtype=np.int32)
    trace = case["runs"]["fixed"]["trace"]
    for i, t in enumerate(trace):
        pen = np.array([np.uint64(int(h, 16)).view(np.float64) for h in t["penalty"]])
        RE = np.array([np.uint64(int(h, 16)).view(np.float64) for h in t["RE"]])
        window = part.window_select(k, i + 1, RE, window)
        assert len(window) == t["window"]
        assert "%016x" % oracle.fnv1a(window) == t["window_hash"]
        nodes, labs = part.lp_apply(k, pen, window)
        assert len(nodes) == t["changes"]
    assert np.array_equal(part.labels(), golden_arrays(name)["labels2_fixed"])


@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")
def test_reference_gpu_kernel_agrees(part):
    """The reference's own CUDA path (boundaryLPKernel_unified built unmodified for sm_100a, driven by its
    run_phase2 loop) against the oracle and this library, on the same graphs and phase-1 labels."""
    import os
    import tempfile

    from dmolp_b200 import graphs

    rng = np.random.default_rng(77)
    with tempfile.TemporaryDirectory() as td:
        for trial in range(3):
            n = int(rng.integers(800, 4000))
            g = graphs.knn(n, int(rng.integers(2, 4)), int(rng.integers(6, 13)), int(rng.integers(1, 1000)))
            k = int(rng.integers(2, 40))
            o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, 100)
            txt = os.path.join(td, f"g{trial}.txt")
            graphs.write_adjtext(g, txt)
            lab = os.path.join(td, f"l{trial}.bin")
            o1.labels.astype(np.int32).tofile(lab)
            r = oracle.run_reference(txt, k, 100, os.path.join(td, f"o{trial}"), mode="fixed", iters=10, gpu=True,
                                     labels_in=lab, seed_dump=False, timeout=600)
            o2 = oracle.phase2(g.offsets, g.indices, o1.labels, k, "fixed", 10)
            assert np.array_equal(r["labels2"], o2.labels), trial
            assert r["result"]["edge_cut"] == o2.res.edge_cut
            part.upload(g)
            part.set_labels(o1.labels)
            m = part.phase2(k, mode="fixed", iterations=10)
            assert np.array_equal(part.labels(), r["labels2"]), trial
            assert m.edge_cut == r["result"]["edge_cut"]


def test_symmetry_detection_selects_the_statistics_path(part):
    """An upload whose arcs all have reverses updates cut and balance from the movers; one missing reverse
    switches the loop to the full statistics pass (one more launch per iteration: two more over iterations 2
    and 3)."""
    from dmolp_b200 import graphs

    g = graphs.knn(2000, 3, 10, seed=3)

    def launches_for(gr):
        """Kernel launches of LP iterations 2 and 3: a 3-iteration run minus a 1-iteration run, each the
        first run after a fresh upload (so the one-time set-up of a run cancels out)."""
        def run(iters):
            part.upload(gr)
            part.set_labels(np.zeros(gr.num_vertices, np.int32))
            a = part.kernel_launches()
            part.phase2(1, mode="fixed", iterations=iters, records=False)
            return part.kernel_launches() - a
        return run(3) - run(1)

    def drop_arc(gr, x, y):  # the graph without arc (x, y); (y, x) stays
        row = gr.indices[gr.offsets[x]:gr.offsets[x + 1]]
        keep = np.ones(gr.num_arcs, bool)
        keep[gr.offsets[x] + int(np.nonzero(row == y)[0][0])] = False
        off = np.zeros(gr.num_vertices + 1, np.int64)
        src = np.repeat(np.arange(gr.num_vertices), np.diff(gr.offsets))
        off[1:] = np.cumsum(np.diff(gr.offsets) - np.bincount(src[~keep], minlength=gr.num_vertices))
        return graphs.Graph(off, gr.indices[keep])

    sym = launches_for(g)
    u = 7
    v = int(g.indices[g.offsets[u]])
    # the missing reverse on either side: the endpoint that searches and the one that is only counted
    assert launches_for(drop_arc(g, v, u)) == sym + 2
    assert launches_for(drop_arc(g, u, v)) == sym + 2
    assert launches_for(g) == sym
    # a skewed graph: an arc between a hub and a leaf, dropped from the hub's row and from the leaf's
    r = graphs.rmat(12, 8, seed=5)
    deg = np.diff(r.offsets)
    hub = int(np.argmax(deg))
    leaf = int(r.indices[r.offsets[hub]:r.offsets[hub + 1]][np.argmin(deg[r.indices[r.offsets[hub]:r.offsets[hub + 1]]])])
    rs = launches_for(r)
    assert launches_for(drop_arc(r, hub, leaf)) == rs + 2
    assert launches_for(drop_arc(r, leaf, hub)) == rs + 2
