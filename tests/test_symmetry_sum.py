"""The multiset symmetry sum of the LP loop's default symmetry test, restated in numpy (the kernel is
k_symhash; its GPU tests are in test_symmetry.py).  Over every arc (u, v), u != v, of the pair
p = (min, max): S += s * mix(p ^ key) mod 2^64, s = +1 when u < v and -1 when u > v, mix the SplitMix64
finaliser.  A graph whose every arc has its reverse with the same multiplicity sums to zero for every key;
graphs one arc, one redirection or one degree-preserving swap away from symmetric do not."""
import numpy as np

from dmolp_b200 import graphs

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def mix(z):
    z = z.astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def sym_sum(g, key):
    src = np.repeat(np.arange(g.num_vertices, dtype=np.uint64), np.diff(g.offsets))
    dst = g.indices.astype(np.uint64)
    keep = src != dst
    u, v = src[keep], dst[keep]
    lo, hi = np.minimum(u, v), np.maximum(u, v)
    f = mix((lo << np.uint64(32) | hi) ^ np.uint64(key))
    with np.errstate(over="ignore"):
        signed = np.where(u < v, f, (np.uint64(0) - f))
        return int(np.sum(signed, dtype=np.uint64))


def edit(g, u, drop=(), add=()):
    rows = [list(g.indices[g.offsets[x]:g.offsets[x + 1]]) for x in range(g.num_vertices)]
    rows[u] = sorted([x for x in rows[u] if x not in drop] + list(add))
    off = np.zeros(g.num_vertices + 1, np.int64)
    off[1:] = np.cumsum([len(r) for r in rows])
    return graphs.Graph(off, np.concatenate([np.asarray(r, np.int32) for r in rows]))


def test_symmetric_graphs_sum_to_zero_for_any_key():
    for g in (graphs.knn(3000, 3, 8, seed=1), graphs.barabasi_albert(2000, 4, seed=2), graphs.rmat(11, 8, seed=3)):
        for key in (0, 1, 0x9E3779B97F4A7C15, 0xDEADBEEFCAFEF00D):
            assert sym_sum(g, key) == 0


def test_graphs_one_edit_from_symmetric_do_not():
    g = graphs.knn(3000, 3, 8, seed=4)
    rng = np.random.default_rng(5)
    row = lambda x: list(g.indices[g.offsets[x]:g.offsets[x + 1]])  # noqa: E731
    for _ in range(20):
        u = int(rng.integers(0, g.num_vertices))
        v = row(u)[0]
        w = next(int(x) for x in rng.permutation(g.num_vertices) if x != u and x not in row(u))
        variants = [edit(g, u, drop=[v]), edit(g, u, drop=[v], add=[w]), edit(g, u, add=[w])]
        z = int(row(w)[0])
        if v not in row(w) and z != u:  # (u, v), (w, z) -> (u, w), (w, v): every degree kept
            h = edit(g, u, drop=[v], add=[w])
            variants.append(edit(h, w, drop=[z], add=[v]))
        for h in variants:
            for key in (0x1234, 0xABCDEF987654321):
                assert sym_sum(h, key) != 0
