"""Batched phase 2: every instance of a batch must end exactly where the oracle's single-graph phase 2 ends
on the same graph and initial labels (labels, cut, part counts, iterations, stop reason, traversed edges),
for every launch shape; host-side pieces (instance mix, union CSR) run on the CPU."""
import numpy as np
import pytest

import oracle
from dmolp_b200 import graphs
from dmolp_b200.batch import Instance, random_instances, union


def part_counts(g, labels, k):
    vc = np.bincount(labels, minlength=k).astype(np.int64)
    src = np.repeat(np.arange(g.num_vertices), np.diff(g.offsets))
    same = labels[src] == labels[g.indices]
    ec = np.bincount(labels[src][same], minlength=k).astype(np.int64) // 2
    return vc, ec


def small_batch(seed=5):
    """Mixed small instances plus edge cases: isolated vertices, one vertex, k = 1, k = 64, a path."""
    inst = random_instances(14, seed=seed, vmin=200, vmax=3000, threads=4)
    inst.append(Instance(graphs.from_edges(7, [(0, 1), (1, 2), (4, 5)]), 3, "isolated"))
    inst.append(Instance(graphs.from_edges(1, []), 1, "single"))
    inst.append(Instance(graphs.knn(500, 3, 10, seed=3), 1, "k1"))
    inst.append(Instance(graphs.knn(3000, 3, 12, seed=4), 64, "k64"))
    inst.append(Instance(graphs.from_edges(40, [(i, i + 1) for i in range(39)]), 4, "path"))
    return inst


def initial_labels(inst):
    out = []
    for it in inst:
        g = it.graph
        if it.k <= g.num_vertices and g.num_arcs > 0:
            out.append(oracle.phase1(g.offsets, g.indices, g.raw_deg(), it.k, 100).labels)
        else:
            out.append((np.arange(g.num_vertices) % it.k).astype(np.int32))
    return out


def test_instance_mix_is_deterministic_and_in_range():
    a = random_instances(8, seed=3, vmin=1000, vmax=5000, threads=2)
    b = random_instances(8, seed=3, vmin=1000, vmax=5000, threads=2)
    for x, y in zip(a, b):
        assert x.k == y.k and x.family == y.family
        assert np.array_equal(x.graph.indices, y.graph.indices)
        assert 1000 <= x.graph.num_vertices <= 5000 and 2 <= x.k <= 64
    assert {x.family[:3] for x in a} == {"knn", "ba"}


def test_union_layout():
    inst = small_batch()
    vstart, off, col, parts = union(inst)
    assert vstart[0] == 0 and vstart[-1] == off.size - 1 and off[-1] == col.size
    for i, it in enumerate(inst):
        g = it.graph
        seg = off[vstart[i]:vstart[i + 1] + 1]
        assert np.array_equal(seg - seg[0], g.offsets)
        assert np.array_equal(col[seg[0]:seg[-1]], g.indices)
        assert parts[i] == it.k


@pytest.fixture(scope="module")
def batch():
    from dmolp_b200.batch import Batch

    b = Batch(0)
    inst = small_batch()
    b.upload(inst)
    yield b, inst, initial_labels(inst)
    b.close()


def check_against_oracle(b, inst, lab0, res, mode, iters, cap):
    final = b.split(b.labels())
    for i, it in enumerate(inst):
        g = it.graph
        o = oracle.phase2(g.offsets, g.indices, lab0[i], it.k, mode, iters, cap)
        r = res[i]
        assert r["status"] == 0, i
        assert np.array_equal(final[i], o.labels), (i, it.family, mode, cap)
        assert r["edge_cut"] == o.res.edge_cut, i
        assert r["iterations_run"] == o.res.iterations_run, i
        assert r["stop_reason"] == o.res.stop_reason, i
        assert r["traversed_edges"] == o.res.te_total, i
        vc, ec = b.counts(i)
        evc, eec = part_counts(g, o.labels, it.k)
        assert np.array_equal(vc, evc) and np.array_equal(ec, eec), i
        assert r["vertex_balance"] == o.res.vertex_balance and r["edge_balance"] == o.res.edge_balance, i


@pytest.mark.gpu
@pytest.mark.parametrize("mode,iters,cap", [("ref", 0, "ref"), ("fixed", 12, "ref"), ("fixed", 9, "full"),
                                            ("ref", 0, "full")])
def test_batch_matches_oracle(batch, mode, iters, cap):
    b, inst, lab0 = batch
    b.set_labels(lab0)
    res, ms = b.run(mode, iters, cap)
    assert ms > 0
    check_against_oracle(b, inst, lab0, res, mode, iters, cap)


@pytest.mark.gpu
def test_every_launch_shape_gives_the_same_result(batch):
    b, inst, lab0 = batch
    ref = None
    for nt in (256, 512, 1024):
        for td in (8, 16):
            b.set_labels(lab0)
            res, _ = b.run("ref", 0, "ref", tuning=dict(block_threads=nt, thread_row_max=td, blocks_per_sm=1))
            lab = b.labels()
            if ref is None:
                ref = (lab, [r["edge_cut"] for r in res])
            assert np.array_equal(lab, ref[0]), (nt, td)
            assert [r["edge_cut"] for r in res] == ref[1]


@pytest.mark.gpu
def test_autotune_restores_labels_and_keeps_results(batch, tmp_path):
    b, inst, lab0 = batch
    b.set_labels(lab0)
    t = b.autotune("ref", 0, "ref", cache=str(tmp_path / "tune.json"))
    assert t["block_threads"] in (256, 512, 1024) and t["thread_row_max"] in (8, 16) and not t["cached"]
    assert np.array_equal(b.labels(), np.concatenate(lab0))
    t2 = b.autotune("ref", 0, "ref", cache=str(tmp_path / "tune.json"))
    assert t2["cached"] and t2["block_threads"] == t["block_threads"]
    res, _ = b.run("ref", 0, "ref")
    check_against_oracle(b, inst, lab0, res, "ref", 0, "ref")


@pytest.mark.gpu
def test_unsorted_and_directed_instances_recount():
    """Rows that are not sorted, or arcs without their reverse: the batch recounts cut and balance each
    iteration instead of updating them from the movers; results still match the oracle."""
    from dmolp_b200.batch import Batch
    from dmolp_b200.partitioner import DmolpError

    rng = np.random.default_rng(2)
    g = graphs.knn(800, 3, 10, seed=9)
    col = g.indices.copy()
    for v in range(g.num_vertices):  # same graph, rows shuffled
        rng.shuffle(col[g.offsets[v]:g.offsets[v + 1]])
    shuffled = graphs.Graph(g.offsets, col)
    n = 300
    rows = [np.unique(rng.integers(0, n, size=rng.integers(1, 9))).astype(np.int32) for _ in range(n)]
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum([len(r) for r in rows])
    directed = graphs.Graph(off, np.concatenate(rows).astype(np.int32))
    inst = [Instance(shuffled, 6, "shuffled"), Instance(directed, 3, "directed")]
    lab0 = [oracle.phase1(g.offsets, g.indices, g.raw_deg(), 6, 60).labels, (np.arange(n) % 3).astype(np.int32)]
    b = Batch(0)
    b.upload(inst)
    b.set_labels(lab0)
    try:
        o1 = oracle.phase2(directed.offsets, directed.indices, lab0[1], 3, "fixed", 6, "ref")
    except RuntimeError:
        o1 = None  # an odd cut-arc count: the reference aborts
    if o1 is None:
        with pytest.raises(DmolpError) as ei:
            b.run("fixed", 6, "ref")
        assert "instance 1" in str(ei.value)
        res = None
    else:
        res, _ = b.run("fixed", 6, "ref")
        assert np.array_equal(b.split(b.labels())[1], o1.labels)
        assert res[1]["edge_cut"] == o1.res.edge_cut
    o0 = oracle.phase2(shuffled.offsets, shuffled.indices, lab0[0], 6, "fixed", 6, "ref")
    assert np.array_equal(b.split(b.labels())[0], o0.labels)
    if res is not None:
        assert res[0]["edge_cut"] == o0.res.edge_cut and res[0]["traversed_edges"] == o0.res.te_total
    b.close()


@pytest.mark.gpu
def test_bad_labels_leave_instance_and_report():
    from dmolp_b200.batch import Batch
    from dmolp_b200.partitioner import DmolpError

    inst = [Instance(graphs.knn(600, 3, 10, seed=7), 4, "a"), Instance(graphs.knn(700, 2, 9, seed=8), 6, "b")]
    lab = initial_labels(inst)
    bad = lab[1].copy()
    bad[5] = 6  # outside [0, 6)
    b = Batch(0)
    b.upload(inst)
    b.set_labels([lab[0], bad])
    with pytest.raises(DmolpError) as ei:
        b.run("fixed", 5, "ref")
    assert ei.value.code == 5 and "instance 1" in str(ei.value)
    out = b.split(b.labels())
    assert np.array_equal(out[1], bad)
    o = oracle.phase2(inst[0].graph.offsets, inst[0].graph.indices, lab[0], 4, "fixed", 5, "ref")
    assert np.array_equal(out[0], o.labels)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("theta", [1, 7, 100])
def test_batched_phase1_matches_single_graph_path(batch, theta):
    """Phase 1 of every graph in one launch: seeds, labels, rounds and traversed edges as dmolp_phase1
    gives them for each graph alone (which the oracle and the reference pin)."""
    from dmolp_b200.partitioner import Partitioner

    b, inst, _ = batch
    res, seeds, ms = b.phase1(theta, seeds=True)
    assert ms > 0
    got = b.split(b.labels())
    p = Partitioner(0)
    for i, it in enumerate(inst):
        g = it.graph
        if g.num_vertices == 0:
            continue
        p.upload(g)
        m = p.phase1(it.k, theta)
        assert np.array_equal(got[i], p.labels()), (i, it.family, theta)
        assert seeds[i, :it.k].tolist() == m.seeds, i
        assert res[i]["num_seeds_found"] == m.num_seeds_found and res[i]["rounds"] == m.rounds, i
        assert res[i]["traversed_edges"] == m.traversed_edges, i
    p.close()
    # a masked run leaves the other graphs' labels alone
    before = b.labels()
    b.set_labels(np.zeros(b.num_vertices, np.int32))
    only = np.arange(len(inst)) % 2 == 0
    b.phase1(theta, only=only)
    masked = b.split(b.labels())
    for i in range(len(inst)):
        ref = before[b.vstart[i]:b.vstart[i + 1]] if only[i] else np.zeros(inst[i].graph.num_vertices, np.int32)
        assert np.array_equal(masked[i], ref), i
    b.phase1(theta)
    # phase 1 then phase 2, both batched: each graph as the oracle's whole path
    b.run("ref")
    fin = b.split(b.labels())
    for i, it in enumerate(inst[:6]):
        g = it.graph
        o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), it.k, theta)
        o2 = oracle.phase2(g.offsets, g.indices, o1.labels, it.k, "ref", 0)
        assert np.array_equal(fin[i], o2.labels), i
