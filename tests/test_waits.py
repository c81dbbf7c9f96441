"""Bounded waits end, report, and leave the context usable.

The window selections are cooperative launches whose blocks meet at grid barriers; the tensor-core GEMM of
the learned proposal waits on its MMAs' completion barrier.  Every such wait gives up after a number of
polls (host-settable; the defaults are never reached).  With the limit set to one poll the wait runs out:
the call returns DMOLP_ERR_CUDA naming the barrier, every block has left the kernel, and the same context
then runs the same call bit-exact with the default limit.  No GPU fault is involved: a barrier that gives up
only makes the blocks leave early."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [16, 100])  # the degree-bin selection (k <= 64) and the radix selection
def test_selection_barrier_gives_up_and_context_recovers(k):
    from dmolp_b200 import cabi, graphs
    from dmolp_b200.partitioner import DmolpError, Partitioner

    g = graphs.rmat(14, 8, seed=3)
    with Partitioner(0) as p:
        p.upload(g)
        p.phase1(k, 100)
        lab = p.labels()
        ref = p.phase2(k, mode="fixed", iterations=6, records=False)
        ref_labels = p.labels()
        p.set_labels(lab)
        assert p.lib.dmolp_set_wait_limit(p.ctx, 1) == cabi.DMOLP_OK
        with pytest.raises(DmolpError) as e:
            p.phase2(k, mode="fixed", iterations=6, records=False)
        assert e.value.code == cabi.DMOLP_ERR_CUDA and "gave up" in str(e.value)
        assert p.lib.dmolp_set_wait_limit(p.ctx, 0) == cabi.DMOLP_OK
        p.set_labels(lab)
        again = p.phase2(k, mode="fixed", iterations=6, records=False)
        assert np.array_equal(p.labels(), ref_labels)
        assert again.edge_cut == ref.edge_cut and again.traversed_edges == ref.traversed_edges


def test_gemm_wait_gives_up_and_network_recovers():
    from dmolp_b200 import cabi, graphs
    from dmolp_b200.batch import Batch, Instance
    from dmolp_b200.learned import Proposal
    from dmolp_b200.partitioner import DmolpError

    inst = [Instance(graphs.knn(600, 3, 8, seed=9), 5, "knn3d"), Instance(graphs.barabasi_albert(400, 3, seed=2), 7, "ba")]
    b = Batch(0)
    m = Proposal(0)
    try:
        b.upload(inst)
        rng = np.random.default_rng(1)
        m.set_params((rng.standard_normal(m.n) * 0.2).astype(np.float32))
        m.set_features(b, rng.standard_normal((b.num_vertices, 16)).astype(np.float32))
        ref = m.forward(b)
        assert m.lib.dmolp_mpnn_set_wait_limit(m.h, 1) == cabi.DMOLP_OK
        with pytest.raises(DmolpError) as e:
            m.forward(b)
        assert e.value.code == cabi.DMOLP_ERR_CUDA and "timed out" in str(e.value)
        assert m.lib.dmolp_mpnn_set_wait_limit(m.h, 0) == cabi.DMOLP_OK
        assert np.array_equal(m.forward(b), ref)
    finally:
        m.close()
        b.close()
