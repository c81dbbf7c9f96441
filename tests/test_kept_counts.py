"""The invariants behind the LP loop's kept counts, restated on the host in numpy.

On a symmetric graph with rows free of duplicates, a vertex's neighbour-label counts change only through
its neighbours' moves: a mover v from label a to c moves one count of every neighbour u from a to c (the
arc (u, v) is in u's row exactly once).  The device keeps the counts of labels < 32 as 16-bit halves of
32-bit words and applies a move with one 32-bit add of the difference of the two halves' units; that is
exact while the count that leaves is >= 1 and the one that enters stays below 2^16.  The hub-window count
of a vertex (how many hubs of the previous window list it) moves by one whenever such a hub enters or
leaves the window."""
import numpy as np

from dmolp_b200 import graphs


def recount(g, labels, eff):
    src = np.repeat(np.arange(g.num_vertices), np.diff(g.offsets))
    cnt = np.zeros((g.num_vertices, 32), np.int64)
    lab = labels[g.indices]
    ok = lab < eff
    np.add.at(cnt, (src[ok], lab[ok]), 1)
    return cnt


def pack(cnt):
    c = cnt.astype(np.uint32)
    return c[:, 0::2] | (c[:, 1::2] << np.uint32(16))


def unpack(words):
    w = words.astype(np.uint64)
    out = np.zeros((words.shape[0], 32), np.int64)
    out[:, 0::2] = (w & 0xFFFF).astype(np.int64)
    out[:, 1::2] = (w >> 16).astype(np.int64)
    return out


def test_counts_follow_the_moves_exactly():
    g = graphs.knn(3000, 3, 12, seed=4)
    rng = np.random.default_rng(1)
    k, eff = 40, 32  # labels >= eff are not counted, as under the reference's 32-label cap
    labels = rng.integers(0, k, g.num_vertices)
    words = pack(recount(g, labels, eff))
    for _ in range(6):
        movers = rng.choice(g.num_vertices, size=400, replace=False)
        new = rng.integers(0, k, movers.size)
        keep = new != labels[movers]
        movers, new = movers[keep], new[keep]
        for v, c in zip(movers, new):  # Jacobi: every update uses the old labels
            a = labels[v]
            for u in g.indices[g.offsets[v]:g.offsets[v + 1]]:
                ia, ic = a < eff, c < eff
                da = np.uint32(1) << np.uint32((a & 1) * 16)
                dc = np.uint32(1) << np.uint32((c & 1) * 16)
                if ia and ic and (a >> 1) == (c >> 1):
                    words[u, a >> 1] = np.uint32((int(words[u, a >> 1]) + int(dc) - int(da)) % (1 << 32))
                else:
                    if ia:
                        words[u, a >> 1] = np.uint32((int(words[u, a >> 1]) - int(da)) % (1 << 32))
                    if ic:
                        words[u, c >> 1] = np.uint32((int(words[u, c >> 1]) + int(dc)) % (1 << 32))
        labels[movers] = new
        assert np.array_equal(unpack(words), recount(g, labels, eff))


def test_hub_window_counts_follow_the_window():
    g = graphs.rmat(12, 16, seed=3)
    deg = np.diff(g.offsets)
    hubs = np.nonzero(deg > np.quantile(deg, 0.98))[0]
    rng = np.random.default_rng(2)
    inside = np.zeros(hubs.size, bool)
    hubwin = np.zeros(g.num_vertices, np.int64)
    for _ in range(8):
        now = rng.random(hubs.size) < 0.6  # the hubs in this iteration's previous window
        for i in np.nonzero(now != inside)[0]:
            h = hubs[i]
            hubwin[g.indices[g.offsets[h]:g.offsets[h + 1]]] += 1 if now[i] else -1
        inside = now
        want = np.zeros(g.num_vertices, np.int64)
        for h in hubs[inside]:
            want[g.indices[g.offsets[h]:g.offsets[h + 1]]] += 1
        assert np.array_equal(hubwin, want)
        # a vertex is a candidate through the hubs exactly when a window hub lists it
        assert np.array_equal(hubwin > 0, want > 0)
