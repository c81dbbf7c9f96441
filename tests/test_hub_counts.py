"""Hub decisions (rows longer than 4096 arcs) on graphs that have hubs, against the oracle.

On a symmetric graph with strictly increasing rows the loop counts every hub's row once at the start of a
run and then keeps those label counts current from the movers' arcs; on any other graph (here: one arc
pair listed twice) it recounts the selected hubs' rows every iteration.  Both must give the oracle's labels, cut and traversed-edge counts over many
iterations, for both label caps, with self-loops on hubs (a hub that moves changes its own count) and hubs
adjacent to each other."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def hub_graph(seed=0, n=20000, hubs=(11, 4000, 9000, 15000, 19999), loops=(4000, 19999)):
    """k-nearest-neighbour base graph plus hub vertices joined to 4200-9000 random vertices each (and to one
    another), symmetric, rows strictly increasing, self-loops on `loops`."""
    from dmolp_b200 import graphs

    base = graphs.knn(n, 3, 8, seed=seed + 1)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(base.offsets))
    e = [np.stack([src, base.indices.astype(np.int64)], 1)]
    rng = np.random.default_rng(seed)
    for h in hubs:
        nb = rng.choice(n, size=int(rng.integers(4200, 9000)), replace=False)
        e.append(np.stack([np.full(nb.size, h), nb], 1))
    hs = np.array(hubs, dtype=np.int64)
    e.append(np.stack(np.meshgrid(hs, hs), -1).reshape(-1, 2))
    e = np.concatenate(e)
    e = e[e[:, 0] != e[:, 1]]
    both = np.concatenate([e, e[:, ::-1], np.stack([np.array(loops), np.array(loops)], 1)])
    both = np.unique(both, axis=0)
    off = np.zeros(n + 1, dtype=np.int64)
    np.add.at(off, both[:, 0] + 1, 1)
    g = graphs.Graph(np.cumsum(off), both[:, 1].astype(np.int32))
    assert (np.diff(g.offsets)[list(hubs)] > 4096).all()
    return g


def duplicate_arc(g, x, y):
    """The graph with arc (x, y) and its reverse each listed twice: rows no longer strictly increasing, so
    the loop takes its recounting path (and the cut-arc count stays even)."""
    from dmolp_b200 import graphs

    src = np.repeat(np.arange(g.num_vertices, dtype=np.int64), np.diff(g.offsets))
    e = np.concatenate([np.stack([src, g.indices.astype(np.int64)], 1), [[x, y], [y, x]]])
    e = e[np.lexsort((e[:, 1], e[:, 0]))]
    off = np.zeros(g.num_vertices + 1, np.int64)
    np.add.at(off, e[:, 0] + 1, 1)
    return graphs.Graph(np.cumsum(off), e[:, 1].astype(np.int32))


@pytest.fixture(scope="module")
def part():
    from dmolp_b200.partitioner import Partitioner

    p = Partitioner(0)
    yield p
    p.close()


@pytest.mark.parametrize("k,cap,start", [(8, "ref", "phase1"), (40, "full", "random"), (64, "ref", "random"),
                                         (32, "ref", "random")])
def test_hub_decisions_match_oracle(part, k, cap, start):
    g = hub_graph()
    part.upload(g)
    if start == "phase1":
        lab0 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, 200).labels
    else:
        lab0 = np.random.default_rng(k).integers(0, k, g.num_vertices).astype(np.int32)
    for recount in (False, True):
        gr = duplicate_arc(g, 9000, int(g.indices[g.offsets[9000] + 5])) if recount else g
        part.upload(gr)
        part.set_labels(lab0)
        m = part.phase2(k, mode="fixed", iterations=20, cap=cap)
        o = oracle.phase2(gr.offsets, gr.indices, lab0, k, "fixed", 20, cap=cap)
        assert np.array_equal(part.labels(), o.labels), (k, cap, recount)
        assert m.edge_cut == o.res.edge_cut and m.traversed_edges == o.res.te_total
        # a second run from the same start recounts the hubs at its start and repeats the first
        part.set_labels(lab0)
        m2 = part.phase2(k, mode="fixed", iterations=20, cap=cap)
        assert np.array_equal(part.labels(), o.labels) and m2.edge_cut == m.edge_cut


def test_hub_decisions_reference_stopping_rules(part):
    g = hub_graph(seed=3)
    part.upload(g)
    lab0 = np.random.default_rng(5).integers(0, 16, g.num_vertices).astype(np.int32)
    part.set_labels(lab0)
    m = part.phase2(16, mode="ref")
    o = oracle.phase2(g.offsets, g.indices, lab0, 16, "ref")
    assert np.array_equal(part.labels(), o.labels)
    assert m.edge_cut == o.res.edge_cut and m.iterations_run == o.res.iterations_run


def test_graph_without_hubs_after_one_with_hubs(part):
    """The per-graph arena is reused: a hub-free graph uploaded after a graph with hubs must not see the
    earlier graph's hub-window counts."""
    from dmolp_b200 import graphs

    g = hub_graph(seed=4)
    part.upload(g)
    part.set_labels(np.random.default_rng(1).integers(0, 8, g.num_vertices).astype(np.int32))
    part.phase2(8, mode="fixed", iterations=12)
    h = graphs.knn(30000, 3, 10, seed=9)
    assert np.diff(h.offsets).max() <= 4096
    part.upload(h)
    lab0 = np.random.default_rng(2).integers(0, 8, h.num_vertices).astype(np.int32)
    part.set_labels(lab0)
    m = part.phase2(8, mode="fixed", iterations=12)
    o = oracle.phase2(h.offsets, h.indices, lab0, 8, "fixed", 12)
    assert np.array_equal(part.labels(), o.labels) and m.edge_cut == o.res.edge_cut
