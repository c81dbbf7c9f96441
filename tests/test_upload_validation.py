"""dmolp_graph_upload validates the host arrays before it touches the resident graph: offsets that go
backwards or past the arc count, ids outside [0, nv) and negative raw degrees are errors, and the previous
graph stays resident; rows that are not strictly increasing are accepted (they only switch the LP loop to
the full statistics pass) and partition like the oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def part():
    from dmolp_b200.partitioner import Partitioner

    p = Partitioner(0)
    yield p
    p.close()


def upload_raw(part, off, col, raw=None):
    import ctypes

    off = np.ascontiguousarray(off, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    rawp = None
    if raw is not None:
        raw = np.ascontiguousarray(raw, np.int32)
        rawp = ctypes.c_void_p(raw.ctypes.data)
    part._check(part.lib.dmolp_graph_upload(part.ctx, off.size - 1, col.size, ctypes.c_void_p(off.ctypes.data),
                                            ctypes.c_void_p(col.ctypes.data), rawp))


def test_bad_uploads_are_errors_and_keep_the_graph(part):
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import DmolpError

    g = graphs.knn(3000, 3, 8, seed=5)
    part.upload(g)
    before = part.graph_arrays()
    bad = [
        ([0, 2, 3, 4], [1, 2, 0, 7], None),            # id 7 >= nv = 3
        ([0, 2, 3, 4], [1, -1, 0, 1], None),           # negative id
        ([0, 3, 1, 4], [1, 2, 0, 1], None),            # offsets go backwards
        ([0, 9, 2, 4], [1, 2, 0, 1], None),            # a row past the arc count (and back)
        ([0, 2, 3, 4], [1, 2, 0, 1], [2, -1, 1]),      # negative raw degree
    ]
    for off, col, raw in bad:
        with pytest.raises(DmolpError):
            upload_raw(part, off, col, raw)
        after = part.graph_arrays()
        assert np.array_equal(before.offsets, after.offsets) and np.array_equal(before.indices, after.indices)


def test_unsorted_rows_partition_like_the_oracle(part):
    from dmolp_b200 import graphs

    g = graphs.knn(4000, 3, 10, seed=6)
    rng = np.random.default_rng(3)
    col = g.indices.copy()
    for v in range(0, g.num_vertices, 7):  # shuffle some rows: still symmetric, no longer sorted
        s, e = g.offsets[v], g.offsets[v + 1]
        col[s:e] = rng.permutation(col[s:e])
    part.upload(graphs.Graph(g.offsets, col))
    h = part.graph_arrays()
    assert np.array_equal(h.indices, col)
    lab0 = rng.integers(0, 8, g.num_vertices).astype(np.int32)
    part.set_labels(lab0)
    m = part.phase2(8, mode="fixed", iterations=12)
    o = oracle.phase2(g.offsets, col, lab0, 8, "fixed", 12)
    assert np.array_equal(part.labels(), o.labels) and m.edge_cut == o.res.edge_cut
