"""The LP loop's symmetry test and the device-side upload check it relies on.

A graph counts as symmetric when its rows are strictly increasing and every arc's reverse is present; the
loop then updates cut and balance from the movers alone (the reference recounts every iteration,
src/phase2/phase2.cpp:214-253, and the results are the same either way).  The default test forms two keyed
multiset sums in one streaming pass; the exact test looks every reverse arc up.  Both must agree on
symmetric graphs and on graphs that miss symmetry by one arc, including edits that keep every degree; a
graph found asymmetric partitions like the oracle through the full recount (or, where the reference aborts
on an odd cut-arc count, is reported as an error).  The upload's order test
works on 16-byte groups of arcs with row-start bits: rows whose first id is below the previous row's last
id are in order, and one descent anywhere (the first group, across a group boundary, in the arcs past the
last whole group) is found."""
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


def both(part, g):
    out = []
    for exact in (False, True):
        part.set_symmetry_test(exact)
        part.upload(g)
        out.append(part.symmetric())
    part.set_symmetry_test(False)
    return out


def edit_rows(g, edits):
    """Rows replaced by edits {v: new sorted row}; returns a new Graph."""
    from dmolp_b200 import graphs

    rows = [g.indices[g.offsets[v]:g.offsets[v + 1]] for v in range(g.num_vertices)]
    for v, r in edits.items():
        rows[v] = np.asarray(r, np.int32)
    off = np.zeros(g.num_vertices + 1, np.int64)
    off[1:] = np.cumsum([len(r) for r in rows])
    return graphs.Graph(off, np.concatenate(rows).astype(np.int32))


def graph_cases():
    from dmolp_b200 import graphs

    return {
        "rmat14": graphs.rmat(14, 8, seed=11),
        "knn": graphs.knn(5000, 3, 9, seed=2),
        "ba": graphs.barabasi_albert(4000, 4, seed=8),
        "star": graphs.Graph(np.array([0, 5000] + list(range(5001, 10001)), np.int64),
                             np.array(list(range(1, 5001)) + [0] * 5000, np.int32)),
    }


@pytest.mark.parametrize("name", ["rmat14", "knn", "ba", "star"])
def test_symmetric_graphs_pass_both_tests(part, name):
    g = graph_cases()[name]
    assert both(part, g) == [True, True]


@pytest.mark.parametrize("kind", ["drop", "redirect", "degree_preserving", "add"])
def test_one_arc_off_fails_both_tests(part, kind):
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import DmolpError

    g = graphs.knn(4000, 3, 8, seed=4)
    rng = np.random.default_rng(7)
    row = lambda v: list(g.indices[g.offsets[v]:g.offsets[v + 1]])  # noqa: E731
    u = int(rng.integers(0, g.num_vertices))
    v = int(row(u)[0])
    w = next(int(x) for x in rng.permutation(g.num_vertices) if x != u and x not in row(u))
    if kind == "drop":  # (u, v) gone, (v, u) kept
        edits = {u: [x for x in row(u) if x != v]}
    elif kind == "redirect":  # (u, v) becomes (u, w)
        edits = {u: sorted([x for x in row(u) if x != v] + [w])}
    elif kind == "degree_preserving":  # (u, v), (w, z) -> (u, w), (w, v): every degree kept, two pairs differ
        z = int(row(w)[0])
        edits = {u: sorted([x for x in row(u) if x != v] + [w]),
                 w: sorted([x for x in row(w) if x != z] + [v]) if v not in row(w) else row(w)}
    else:  # one extra arc (u, w)
        edits = {u: sorted(row(u) + [w])}
    h = edit_rows(g, edits)
    assert both(part, h) == [False, False]
    lab0 = rng.integers(0, 8, h.num_vertices).astype(np.int32)
    part.upload(h)
    part.set_labels(lab0)
    try:
        o = oracle.phase2(h.offsets, h.indices, lab0, 8, "fixed", 10)
    except RuntimeError:  # an odd cut-arc count along the way: the reference aborts, the library reports it
        o = None
    if o is None:
        with pytest.raises(DmolpError):
            part.phase2(8, mode="fixed", iterations=10)
    else:
        m = part.phase2(8, mode="fixed", iterations=10)
        assert np.array_equal(part.labels(), o.labels) and m.edge_cut == o.res.edge_cut


def test_asymmetric_graph_partitions_like_the_oracle(part):
    """Arcs a -> b without their reverse, b with an empty row and a's label: a never leaves b's label (its
    only neighbour), so the cut-arc count stays even and the reference runs; the library takes the full
    recount and ends where the oracle does."""
    from dmolp_b200 import graphs

    g = graphs.knn(4000, 3, 8, seed=4)
    n = g.num_vertices
    extra = 3
    rows = [g.indices[g.offsets[v]:g.offsets[v + 1]] for v in range(n)]
    rows += [np.array([n + 2 * i + 1], np.int32) if j == 0 else np.array([], np.int32)
             for i in range(extra) for j in range(2)]
    off = np.zeros(n + 2 * extra + 1, np.int64)
    off[1:] = np.cumsum([len(r) for r in rows])
    h = graphs.Graph(off, np.concatenate(rows).astype(np.int32))
    assert both(part, h) == [False, False]
    rng = np.random.default_rng(11)
    lab0 = rng.integers(0, 8, h.num_vertices).astype(np.int32)
    for i in range(extra):
        lab0[n + 2 * i] = lab0[n + 2 * i + 1]
    part.upload(h)
    part.set_labels(lab0)
    o = oracle.phase2(h.offsets, h.indices, lab0, 8, "fixed", 10)
    m = part.phase2(8, mode="fixed", iterations=10)
    assert np.array_equal(part.labels(), o.labels) and m.edge_cut == o.res.edge_cut
    assert m.traversed_edges == o.res.te_total


def test_symmetric_with_self_loops(part):
    from dmolp_b200 import graphs

    g = graphs.knn(3000, 3, 6, seed=1)
    edits = {}
    for v in range(0, g.num_vertices, 5):
        r = list(g.indices[g.offsets[v]:g.offsets[v + 1]])
        edits[v] = sorted(r + [v])
    assert both(part, edit_rows(g, edits)) == [True, True]


@pytest.mark.parametrize("narcs_mod", [0, 1, 2, 3])
def test_order_check_on_arc_groups(part, narcs_mod):
    """Rows 0..n-1 of a symmetric graph laid out so that rows start below the previous row's end; then one
    descent placed at every position class of the 16-byte groups, and past the last whole group."""
    from dmolp_b200 import graphs

    rng = np.random.default_rng(narcs_mod)
    n = 64
    # complete graph minus a few arcs on n vertices, symmetric, sorted rows: row v starts at 0 or 1 (below
    # the previous row's last id), so every row start is a descent that must not count
    adj = np.ones((n, n), bool)
    np.fill_diagonal(adj, False)
    for _ in range(40):
        a, b = rng.integers(0, n, 2)
        adj[a, b] = adj[b, a] = False
    # trim arcs so that narcs % 4 == narcs_mod, symmetrically (drop pairs), keeping some rows non-empty
    def build(adj):
        rows = [np.flatnonzero(adj[v]).astype(np.int32) for v in range(n)]
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum([len(r) for r in rows])
        return graphs.Graph(off, np.concatenate(rows))
    g = build(adj)
    # add self-loops (one arc each, symmetric by themselves) until the residue matches
    v = 0
    while g.num_arcs % 4 != narcs_mod:
        adj[v, v] = True
        v += 1
        g = build(adj)
    assert both(part, g) == [True, True]
    # one descent at each of several arc positions inside a row (swap two neighbours of that row)
    for j in [1, 2, 3, 4, 5, 7, 8, g.num_arcs - 1, g.num_arcs - 2, g.num_arcs - 3]:
        u = int(np.searchsorted(g.offsets, j, side="right") - 1)
        s = int(g.offsets[u])
        if j == s:  # a row start: nothing to swap with inside the row
            continue
        col = g.indices.copy()
        col[j - 1], col[j] = col[j], col[j - 1]
        h = graphs.Graph(g.offsets, col)
        assert both(part, h) == [False, False], j
        part.upload(h)
        np.testing.assert_array_equal(part.graph_arrays().indices, col)
