"""dmolp_metrics_noalloc: the cut/balance reduction for callers that cannot let a library allocate device
memory (their GPU memory belongs to another allocator).  The caller's CSR and labels are device buffers --
allocated here with torch, by the test, as such a caller would own them -- and the results must equal those of
dmolp_metrics, the entry point that works on the library's own resident copy.  Two calls in a row with
different label sets and k check that the shared scratch array is cleared between calls.  A neighbour id
outside [0, nv) in the caller's CSR is skipped and flagged by the kernel (an error status, never a read out of
range), and the caller's current device is the same after every call."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_metrics_noalloc_matches_dmolp_metrics():
    import torch

    from dmolp_b200 import cabi, graphs
    from dmolp_b200.partitioner import Partitioner

    g = graphs.rmat(14, 8, seed=21)
    dev = torch.device("cuda", 0)
    off_d = torch.from_numpy(g.offsets).to(dev)
    col_d = torch.from_numpy(g.indices).to(dev)
    rng = np.random.default_rng(8)
    with Partitioner(0) as p:
        p.upload(g)
        for k in (40, 7):  # second call uses fewer parts: stale counts from the first would show
            lab = rng.integers(0, k, g.num_vertices).astype(np.int32)
            p.set_labels(lab)
            cut_ref, vc_ref, ec_ref = p.metrics(k)
            lab_d = torch.from_numpy(lab).to(dev)
            torch.cuda.synchronize()
            cut = ctypes.c_int64(-1)
            vc = np.full(k, -1, np.int64)
            ec = np.full(k, -1, np.int64)
            rc = p.lib.dmolp_metrics_noalloc(0, g.num_vertices, ctypes.c_void_p(off_d.data_ptr()),
                                             ctypes.c_void_p(col_d.data_ptr()), ctypes.c_void_p(lab_d.data_ptr()), k,
                                             None, ctypes.byref(cut), vc.ctypes.data_as(ctypes.c_void_p),
                                             ec.ctypes.data_as(ctypes.c_void_p))
            assert rc == cabi.DMOLP_OK, p.lib.dmolp_last_error()
            assert cut.value == cut_ref
            assert np.array_equal(vc, vc_ref) and np.array_equal(ec, ec_ref)
        # a neighbour id outside [0, nv): DMOLP_ERR_ARG from the kernel's own check, then a good call again
        bad = g.indices.copy()
        bad[len(bad) // 2] = g.num_vertices + 3
        col_bad = torch.from_numpy(bad).to(dev)
        torch.cuda.synchronize()
        rc = p.lib.dmolp_metrics_noalloc(0, g.num_vertices, ctypes.c_void_p(off_d.data_ptr()),
                                         ctypes.c_void_p(col_bad.data_ptr()), ctypes.c_void_p(lab_d.data_ptr()), k,
                                         None, ctypes.byref(cut), None, None)
        assert rc == cabi.DMOLP_ERR_ARG and b"neighbour id" in p.lib.dmolp_last_error()
        assert p.lib.dmolp_current_device() == 0
        rc = p.lib.dmolp_metrics_noalloc(0, g.num_vertices, ctypes.c_void_p(off_d.data_ptr()),
                                         ctypes.c_void_p(col_d.data_ptr()), ctypes.c_void_p(lab_d.data_ptr()), k,
                                         None, ctypes.byref(cut), None, None)
        assert rc == cabi.DMOLP_OK and cut.value == cut_ref
        # a null id array with vertices: rejected on the host
        rc = p.lib.dmolp_metrics_noalloc(0, g.num_vertices, ctypes.c_void_p(off_d.data_ptr()), None,
                                         ctypes.c_void_p(lab_d.data_ptr()), k, None, ctypes.byref(cut), None, None)
        assert rc == cabi.DMOLP_ERR_ARG
        # beyond the scratch array's size: a clear error, no device work
        rc = p.lib.dmolp_metrics_noalloc(0, g.num_vertices, ctypes.c_void_p(off_d.data_ptr()),
                                         ctypes.c_void_p(col_d.data_ptr()), ctypes.c_void_p(lab_d.data_ptr()), 1025,
                                         None, ctypes.byref(cut), None, None)
        assert rc == cabi.DMOLP_ERR_ARG
        assert b"1024" in p.lib.dmolp_last_error()
