"""CPU-side checks of the native libraries: they load, export every symbol the public header declares, refuse
to run without a GPU, and the host-only pieces (text loader, generators) behave as the reference's."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "dmolp_b200.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dmolp_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from dmolp_b200 import _native, cabi

    path = _native.core_path()
    assert os.path.exists(path), "run __graft_entry__.build() first"
    lib = ctypes.CDLL(path)
    declared = header_functions()
    assert set(cabi.EXPORTS) == set(declared)
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dmolp_\w+)", out))
    assert set(declared) <= exported


@pytest.mark.gpu
def test_library_is_built_for_sm100a():
    """The runtime reports the loaded device code as sm_100 (the library carries sm_100a code only)."""
    from dmolp_b200 import _native, cabi

    v = ctypes.c_int(0)
    lib = _native.core()
    assert lib.dmolp_device_code_version(0, ctypes.byref(v)) == cabi.DMOLP_OK, lib.dmolp_last_error()
    assert v.value == 100


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_no_gpu_is_an_error_not_a_fallback():
    from dmolp_b200 import cabi
    from dmolp_b200.partitioner import DmolpError, Partitioner

    with pytest.raises(DmolpError) as e:
        Partitioner(0)
    assert e.value.code == cabi.DMOLP_ERR_NO_GPU


TRICKY_TEXTS = {
    "plain": "4\n1 2\n0 2\n0 1 3\n2\n",
    "dups_selfloop": "3\n1 1 2 0\n0 0\n1 0\n",
    "leading_space": "3\n 1\n0\n\n",           # fast_atoi turns the leading space into a neighbour 0
    "separators": "3\n1,2\n0\t2\r\n0  1 \n",
    "unterminated_last": "3\n1\n0\n1",           # the reference drops the last line
    "empty_lines": "5\n\n\n3\n2\n\n",
}


@pytest.mark.parametrize("name", sorted(TRICKY_TEXTS))
def test_text_loader_matches_reference_loader(name):
    from dmolp_b200.partitioner import load_adjtext

    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.txt")
        open(p, "w").write(TRICKY_TEXTS[name])
        off, col, raw = oracle.load_adjtext(p)
        g = load_adjtext(p)
        assert np.array_equal(g.offsets, off) and np.array_equal(g.indices, col)
        assert np.array_equal(g.raw_degree, raw)
        if oracle.reference_available():  # the reference's own CSR (built by its phase 1)
            try:
                r = oracle.run_reference(p, 1, 1, os.path.join(td, "o"), phase1_only=True)
                assert np.array_equal(r["row_ptr"], off.astype(np.int32))
                assert np.array_equal(r["col_idx"], col)
            except RuntimeError:
                pass


def test_text_loader_rejects_out_of_range_ids():
    from dmolp_b200.partitioner import DmolpError, load_adjtext

    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.txt")
        open(p, "w").write("2\n1\n5\n")
        with pytest.raises(DmolpError):
            load_adjtext(p)


def test_text_loader_round_trip_generated_graph():
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import load_adjtext

    g = graphs.rmat(12, 8, seed=3)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.txt")
        graphs.write_adjtext(g, p)
        h = load_adjtext(p)
    assert np.array_equal(g.offsets, h.offsets) and np.array_equal(g.indices, h.indices)
    assert np.array_equal(h.raw_degree, g.degree())


def test_generators_are_deterministic_and_symmetric():
    from dmolp_b200 import graphs

    for make in (lambda: graphs.rmat(11, 8, seed=5), lambda: graphs.knn(3000, 3, 9, 4),
                 lambda: graphs.barabasi_albert(2000, 3, 9)):
        a, b = make(), make()
        assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.indices, b.indices)
        src = np.repeat(np.arange(a.num_vertices), np.diff(a.offsets))
        fwd = set(zip(src.tolist(), a.indices.tolist()))
        assert all((v, u) in fwd for (u, v) in fwd)
        assert not any(u == v for (u, v) in fwd)
