"""ORACLE / TEST INFRASTRUCTURE ONLY.

Python access to the checker: the CPU restatement (libdmolp_oracle.so, built from dmolp_oracle.cpp) and the
reference harness (oracle/_ref/ref_harness, built from the reference's own sources when they are present).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this package.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint64, c_void_p
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")


class Phase1Result(ctypes.Structure):
    _fields_ = [("initial_edge_cut", c_int64), ("initial_vertex_balance", c_double),
                ("initial_edge_balance", c_double), ("num_seeds", c_int32), ("first_seed", c_int32),
                ("first_seed_degree", c_int32), ("rounds", c_int32), ("num_hubs", c_int64), ("te", c_uint64)]


class IterRecord(ctypes.Structure):
    _fields_ = [("iteration", c_int32), ("window", c_int32), ("candidates", c_int32), ("changes", c_int32),
                ("edge_cut", c_int64), ("window_hash", c_uint64), ("labels_hash", c_uint64),
                ("te_prev", c_uint64), ("te_cand", c_uint64), ("te_sel", c_uint64), ("te_stats", c_uint64),
                ("window_sum", c_uint64)]


class Phase2Result(ctypes.Structure):
    _fields_ = [("edge_cut", c_int64), ("vertex_balance", c_double), ("edge_balance", c_double),
                ("iterations_run", c_int32), ("stop_reason", c_int32), ("te_total", c_uint64),
                ("total_vertices", c_int64), ("total_edges", c_int64)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libdmolp_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} not built (make -C oracle)")
        L = ctypes.CDLL(path)
        L.oracle_last_error.restype = c_char_p
        L.oracle_load_adjtext.argtypes = [c_char_p, POINTER(c_int64), POINTER(c_int64), c_void_p, c_void_p, c_void_p]
        L.oracle_find_hubs.argtypes = [c_int64, c_void_p, c_void_p, POINTER(c_int64)]
        L.oracle_degree_order.argtypes = [c_int64, c_void_p, c_void_p]
        L.oracle_phase1.argtypes = [c_int64, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                    c_void_p, POINTER(Phase1Result)]
        L.oracle_phase2.argtypes = [c_int64, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_void_p,
                                    c_void_p, c_void_p, POINTER(Phase2Result)]
        L.oracle_lp_decide.argtypes = [c_int32, c_void_p, c_int64, c_void_p, c_int, c_int]
        L.oracle_lp_decide.restype = c_int32
        L.oracle_fnv1a.argtypes = [c_void_p, ctypes.c_size_t]
        L.oracle_fnv1a.restype = c_uint64
        L.oracle_set_sum.argtypes = [c_void_p, c_int64]
        L.oracle_set_sum.restype = c_uint64
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}: {lib().oracle_last_error().decode()}")


def load_adjtext(path: str):
    """(offsets int64, indices int32, raw_degree int32) as the reference loads and builds them."""
    nv, na = c_int64(), c_int64()
    _check(lib().oracle_load_adjtext(os.fsencode(path), ctypes.byref(nv), ctypes.byref(na), None, None, None))
    off = np.empty(nv.value + 1, np.int64)
    col = np.empty(na.value, np.int32)
    raw = np.empty(nv.value, np.int32)
    _check(lib().oracle_load_adjtext(os.fsencode(path), ctypes.byref(nv), ctypes.byref(na), _p(off), _p(col), _p(raw)))
    return off, col, raw


def degree_order(ids: np.ndarray, degrees: np.ndarray):
    """(ids, degrees) in the order std::sort by degree leaves them (find_hub_nodes' sort, init.cpp:142)."""
    i = np.ascontiguousarray(ids, np.int32).copy()
    d = np.ascontiguousarray(degrees, np.int32).copy()
    _check(lib().oracle_degree_order(i.shape[0], _p(i), _p(d)))
    return i, d


def find_hubs(raw_degree: np.ndarray) -> np.ndarray:
    raw = np.ascontiguousarray(raw_degree, np.int32)
    n = c_int64()
    _check(lib().oracle_find_hubs(raw.shape[0], _p(raw), None, ctypes.byref(n)))
    out = np.empty(n.value, np.int32)
    _check(lib().oracle_find_hubs(raw.shape[0], _p(raw), _p(out), ctypes.byref(n)))
    return out


@dataclass
class Phase1:
    labels: np.ndarray
    seeds: np.ndarray
    vertex_counts: np.ndarray
    edge_counts: np.ndarray
    res: Phase1Result


def phase1(off, col, raw, k: int, theta: int) -> Phase1:
    off = np.ascontiguousarray(off, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    raw = np.ascontiguousarray(raw, np.int32)
    nv = off.shape[0] - 1
    labels = np.empty(nv, np.int32)
    seeds = np.empty(k, np.int32)
    vc = np.empty(k, np.int64)
    ec = np.empty(k, np.int64)
    r = Phase1Result()
    _check(lib().oracle_phase1(nv, _p(off), _p(col), _p(raw), k, theta, _p(labels), _p(seeds), _p(vc), _p(ec),
                               ctypes.byref(r)))
    return Phase1(labels, seeds, vc, ec, r)


@dataclass
class Phase2:
    labels: np.ndarray
    records: list
    counts: np.ndarray  # [iters, 2k]
    penalties: np.ndarray  # [iters, k]
    res: Phase2Result


def phase2(off, col, labels, k: int, mode: str = "fixed", iters: int = 20, cap: str = "ref") -> Phase2:
    off = np.ascontiguousarray(off, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    lab = np.array(labels, dtype=np.int32, copy=True)
    nv = off.shape[0] - 1
    m = 0 if mode == "ref" else 1
    n_rec = 500 if m == 0 else iters
    recs = (IterRecord * max(1, n_rec))()
    counts = np.zeros((max(1, n_rec), 2 * k), np.int64)
    pens = np.zeros((max(1, n_rec), k), np.float64)
    r = Phase2Result()
    _check(lib().oracle_phase2(nv, _p(off), _p(col), k, _p(lab), m, iters, 0 if cap == "ref" else 1,
                               ctypes.cast(recs, c_void_p), _p(counts), _p(pens), ctypes.byref(r)))
    n = r.iterations_run
    return Phase2(lab, [recs[i] for i in range(n)], counts[:n], pens[:n], r)


def lp_decide(own: int, nbr_labels, penalty, k: int, cap: str = "ref") -> int:
    nl = np.ascontiguousarray(nbr_labels, np.int32)
    pen = np.ascontiguousarray(penalty, np.float64)
    return int(lib().oracle_lp_decide(own, _p(nl), nl.shape[0], _p(pen), k, 0 if cap == "ref" else 1))


def reference_available() -> bool:
    return os.path.exists(REF_HARNESS)


def run_reference(graph_txt: str, k: int, theta: int, out_dir: str, mode: str = "fixed", iters: int = 20,
                  gpu: bool = False, threads: int = 1, labels_in: str | None = None, seed_dump: bool = True,
                  phase1_only: bool = False, timeout: float | None = None) -> dict:
    """Run the reference sources (oracle/_ref/ref_harness) and return its parsed outputs."""
    if not reference_available():
        raise RuntimeError("reference harness not built")
    cmd = [REF_HARNESS, graph_txt, str(k), str(theta), "--out", out_dir, "--mode", mode, "--iters", str(iters),
           "--threads", str(threads)]
    if gpu:
        cmd.append("--gpu")
    if labels_in:
        cmd += ["--labels-in", labels_in]
    if not seed_dump:
        cmd.append("--no-seed-dump")
    if phase1_only:
        cmd.append("--phase1-only")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"reference harness failed ({p.returncode}): {p.stderr[-2000:]}")
    return read_reference(out_dir)


def read_reference(out_dir: str) -> dict:
    out = {"phase1": json.load(open(os.path.join(out_dir, "phase1.json")))}
    for name in ("labels1", "labels2", "row_ptr", "col_idx"):
        f = os.path.join(out_dir, name + ".bin")
        if os.path.exists(f):
            out[name] = np.fromfile(f, dtype=np.int32)
    f = os.path.join(out_dir, "result.json")
    if os.path.exists(f):
        out["result"] = json.load(open(f))
    f = os.path.join(out_dir, "trace.jsonl")
    if os.path.exists(f):
        out["trace"] = [json.loads(l) for l in open(f) if l.strip()]
    return out


def f64_bits(x: float) -> str:
    return "%016x" % np.float64(x).view(np.uint64)


def fnv1a(a: np.ndarray) -> int:
    """64-bit FNV-1a over the array's bytes (the hash the reference harness writes)."""
    a = np.ascontiguousarray(a)
    if a.nbytes >= 4096 and os.path.exists(os.path.join(HERE, "libdmolp_oracle.so")):
        return int(lib().oracle_fnv1a(_p(a), a.nbytes))
    h = 1469598103934665603
    for b in a.view(np.uint8).tobytes():
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def set_sum(ids: np.ndarray) -> int:
    """Order-independent checksum of a vertex set: sum mod 2^64 of SplitMix64(id) (the reference harness's
    window_sum and the CUDA path's per-iteration window checksum)."""
    v = np.ascontiguousarray(ids, np.int32)
    return int(lib().oracle_set_sum(_p(v), v.shape[0]))
