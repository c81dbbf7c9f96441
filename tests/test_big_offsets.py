"""Beyond 32-bit arc offsets (the int64-offset configuration the reference's int32 row_ptr cannot hold,
include/graph_types.h:128-130): a band graph of 65,536 vertices with about 2.6e9 arcs, every vertex a hub
(rows of 24 K to 48 K arcs, offsets past 2^31).  Phase 1 and two LP iterations of the CUDA path are held bit
for bit to the oracle, which takes int64 offsets: labels, seeds, cut, traversed edges, and per iteration the
window's size and checksum and the changes.  Needs ~11 GB of host memory for the arcs and ~35 GB on the
device."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_graph_beyond_32bit_offsets_matches_oracle():
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import Partitioner

    g = graphs.band(65536, 12000, 24000, seed=5)
    assert g.num_arcs > 2**31 and int(g.offsets[-1]) == g.num_arcs
    k, theta, iters = 16, 2000, 2
    with Partitioner(0) as p:
        p.upload(g)
        m1 = p.phase1(k, theta)
        lab1 = p.labels()
        m2 = p.phase2(k, mode="fixed", iterations=iters)
        lab2 = p.labels()
    o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, theta)
    assert m1.seeds == o1.seeds.tolist() and m1.rounds == o1.res.rounds
    assert np.array_equal(lab1, o1.labels)
    assert m1.initial_edge_cut == o1.res.initial_edge_cut
    o2 = oracle.phase2(g.offsets, g.indices, o1.labels, k, "fixed", iters)
    assert [(r.window, r.window_sum, r.changes, r.edge_cut) for r in m2.records] == \
           [(r.window, r.window_sum, r.changes, r.edge_cut) for r in o2.records]
    assert np.array_equal(lab2, o2.labels)
    assert m2.edge_cut == o2.res.edge_cut and m2.traversed_edges == o2.res.te_total
