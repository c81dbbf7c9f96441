"""Learned initial partition: the CPU oracle's gradients against finite differences, its decoder's balance;
on the GPU the project's feature, forward, backward (tensor-core GEMMs), loss and decoder kernels against
the oracle, and the proposal end to end."""
import numpy as np
import pytest

from dmolp_b200 import graphs
from dmolp_b200.batch import Instance
from oracle import mpnn as M


def fd_check(off, col, X, P, R, idx, eps=1e-6):
    Z, cache = M.forward(off, col, X, P, exact=True)
    g = M.backward(off, col, cache, R, P, exact=True)
    worst = 0.0
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += eps
        Pm[i] -= eps
        fp = (M.forward(off, col, X, Pp, exact=True)[0] * R).sum()
        fm = (M.forward(off, col, X, Pm, exact=True)[0] * R).sum()
        fd = (fp - fm) / (2 * eps)
        worst = max(worst, abs(fd - g[i]) / max(1e-8, abs(fd) + abs(g[i])))
    return worst


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    for seed, n in ((3, 60), (4, 90)):
        g = graphs.knn(n, 2, 5, seed=seed)
        P = rng.standard_normal(M.num_params()) * 0.3
        X = rng.standard_normal((n, 16))
        R = rng.standard_normal((n, 16))
        idx = rng.choice(M.num_params(), 60, replace=False)
        assert fd_check(g.offsets, g.indices, X, P, R, idx) < 1e-5


def test_oracle_contrastive_gradient():
    rng = np.random.default_rng(1)
    g = graphs.knn(80, 2, 6, seed=2)
    Z = rng.standard_normal((80, 16)).astype(np.float32) * 0.3
    t = rng.integers(0, 4, 80).astype(np.int32)
    _, dZ = M.contrastive(g.offsets, g.indices, Z, t)
    eps = 1e-3
    for _ in range(30):
        v, c = int(rng.integers(80)), int(rng.integers(16))
        Zp, Zm = Z.astype(np.float64).copy(), Z.astype(np.float64).copy()
        Zp[v, c] += eps
        Zm[v, c] -= eps
        fd = (M.contrastive(g.offsets, g.indices, Zp, t)[0] - M.contrastive(g.offsets, g.indices, Zm, t)[0]) / (2 * eps)
        assert abs(fd - dZ[v, c]) < 2e-3 * max(1.0, abs(fd))


@pytest.mark.parametrize("k", [1, 2, 3, 7, 32, 64])
def test_oracle_rcb_is_balanced(k):
    rng = np.random.default_rng(k)
    n = 1000
    Z = rng.standard_normal((n, 16)).astype(np.float32)
    lab = M.rcb(Z, k)
    c = np.bincount(lab, minlength=k)
    assert lab.min() >= 0 and lab.max() < k
    assert c.max() - c.min() <= 6  # floor splits lose at most one vertex per level


def small_instances():
    return [Instance(graphs.knn(700, 3, 10, seed=5), 6, "knn3d"), Instance(graphs.barabasi_albert(500, 4, seed=6), 9, "ba"),
            Instance(graphs.knn(900, 2, 8, seed=7), 17, "knn2d"), Instance(graphs.from_edges(5, [(0, 1)]), 8, "tiny")]


@pytest.fixture(scope="module")
def setup():
    from dmolp_b200.batch import Batch
    from dmolp_b200.learned import Proposal

    inst = small_instances()
    b = Batch(0)
    b.upload(inst)
    m = Proposal(0)
    m.prepare_training(b)
    yield b, m, inst
    m.close()
    b.close()


def oracle_union(inst):
    from dmolp_b200.batch import union

    vstart, off, col, parts = union(inst)
    gcol = col.copy()
    for i in range(len(inst)):
        a, z = off[vstart[i]], off[vstart[i + 1]]
        gcol[a:z] += vstart[i]
    return vstart, off, gcol.astype(np.int32)


@pytest.mark.gpu
def test_features_match_oracle(setup):
    b, m, inst = setup
    X = m.features(b)
    for i, it in enumerate(inst):
        g = it.graph
        ref = M.features(g.offsets, g.indices, it.k)
        got = X[b.vstart[i]:b.vstart[i + 1]]
        np.testing.assert_allclose(got, ref, rtol=2e-4, atol=2e-4, err_msg=it.family)


@pytest.mark.gpu
def test_forward_and_backward_match_oracle(setup):
    b, m, inst = setup
    vstart, off, col = oracle_union(inst)
    rng = np.random.default_rng(3)
    P = (rng.standard_normal(M.num_params()) * 0.2).astype(np.float32)
    m.set_params(P)
    X = rng.standard_normal((b.num_vertices, 16)).astype(np.float32)
    m.set_features(b, X)
    Z = m.forward(b)
    Zr, cache = M.forward(off, col, X, P)
    err = np.linalg.norm(Z - Zr) / np.linalg.norm(Zr)
    assert err < 5e-3, err
    R = rng.standard_normal(Z.shape).astype(np.float32)
    g = m.backward(b, R)
    gr = M.backward(off, col, cache, R, P)
    o = 0
    for K, N in M.LAYERS:
        for part, size in (("W", K * N), ("b", N)):
            a, r = g[o:o + size], gr[o:o + size]
            rel = np.linalg.norm(a - r) / max(1e-12, np.linalg.norm(r))
            assert rel < 2e-2, (K, N, part, rel)
            o += size


@pytest.mark.gpu
def test_train_step_loss_matches_oracle_and_decreases(setup):
    b, m, inst = setup
    vstart, off, col = oracle_union(inst)
    rng = np.random.default_rng(4)
    P = (rng.standard_normal(M.num_params()) * 0.2).astype(np.float32)
    m.set_params(P)
    X = m.features(b)
    tgt = np.concatenate([(np.arange(it.graph.num_vertices) * it.k // max(1, it.graph.num_vertices)).astype(np.int32)
                          for it in inst])
    Zr, _ = M.forward(off, col, X, P)
    lr_, _ = M.contrastive(off, col, M.coords(X, Zr), tgt)
    l0 = m.train_step(b, tgt, 1e-3)
    assert abs(l0 - lr_) <= 1e-2 * max(1.0, abs(lr_)), (l0, lr_)
    losses = [m.train_step(b, tgt, 1e-3) for _ in range(30)]
    assert losses[-1] < l0


@pytest.mark.gpu
def test_decoder_matches_oracle(setup):
    """Principal axes + recursive bisection against the oracle's (float64 axes by another summation order:
    a few vertices at a split may land on the other side)."""
    b, m, inst = setup
    rng = np.random.default_rng(5)
    X = rng.standard_normal((b.num_vertices, 16)).astype(np.float32)
    X[:, 3] *= 4.0  # a dominant axis
    m.set_features(b, X)
    Z = (rng.standard_normal((b.num_vertices, 16)) * 0.1).astype(np.float32)
    st = m.decode(b, Z)
    lab = b.split(b.labels())
    for i, it in enumerate(inst):
        if it.graph.num_vertices < it.k:
            assert st[i] == 1
            continue
        assert st[i] == 0
        sl = slice(b.vstart[i], b.vstart[i + 1])
        ref = M.decode(X[sl], Z[sl], it.k)
        agree = np.mean(lab[i] == ref)
        assert agree > 0.97, (it.family, agree)
        c = np.bincount(lab[i], minlength=it.k)
        assert c.max() - c.min() <= 6


@pytest.mark.gpu
def test_propose_then_lp(setup):
    b, m, inst = setup
    m.set_params(np.zeros(M.num_params(), np.float32))  # gate 0: every usable proposal is accepted
    st = m.propose(b)
    assert list(st) == [0, 0, 0, 1]
    lab = b.split(b.labels())
    for i, it in enumerate(inst[:3]):
        c = np.bincount(lab[i], minlength=it.k)
        assert c.min() > 0 and c.max() - c.min() <= 6


@pytest.mark.gpu
def test_gate_scores_and_training(setup):
    """The gate is the per-graph mean of output 8; its cross-entropy training step lowers the loss."""
    b, m, inst = setup
    rng = np.random.default_rng(8)
    P = (rng.standard_normal(M.num_params()) * 0.2).astype(np.float32)
    m.set_params(P)
    m.features(b, copy=False)
    Z = m.forward(b)
    sc = m.gate(b)
    for i in range(len(inst)):
        sl = slice(b.vstart[i], b.vstart[i + 1])
        assert abs(sc[i] - float(Z[sl, 8].astype(np.float64).mean())) < 1e-5 * max(1.0, abs(sc[i]))
    y = np.array([1, 0, 1, 0], np.float32)
    l0 = m.train_gate(b, y, 1e-2)
    for _ in range(40):
        last = m.train_gate(b, y, 1e-2)
    assert last < l0


@pytest.mark.gpu
def test_trained_network_gains_over_untrained_and_tracks_plain():
    """What training buys, on held-out graphs of the training distribution: the shipped weights' gate keeps
    phase-1 seeding where the proposal would end worse, so the edge cut after phase 2 stays at the plain
    method's (within 2 %), while the untrained network (which accepts every proposal) ends higher."""
    import os

    from dmolp_b200.batch import random_instances
    from dmolp_b200.learned import WEIGHTS, Proposal
    from dmolp_b200.train_proposal import evaluate, plain_eval

    assert os.path.exists(WEIGHTS)
    ev = random_instances(64, seed=777, vmin=1000, vmax=100_000)
    plain = plain_eval(ev, 1000)
    trained = evaluate(Proposal(0, WEIGHTS), ev, plain, 1000)
    untrained = evaluate(Proposal(0), ev, plain, 1000)
    pc = float(np.sum(plain["cut"]))
    tr, un = float(np.sum(trained["cut"])) / pc, float(np.sum(untrained["cut"])) / pc
    print("cut ratios vs plain: trained", tr, "untrained", un, "fallbacks", trained["fallbacks"])
    assert tr < un
    assert tr <= 1.02
    # the proposal's own starts are balanced: every accepted graph's initial parts differ by a few vertices
    assert untrained["fallbacks"] <= sum(1 for it in ev if it.graph.num_vertices < it.k)
