"""Python host API over libdmolp_b200.so (include/dmolp_b200.h).

Mirrors the reference's partitioning interface at one rank:

    run_phase1(graph_file, num_parts, theta)  ->  Phase1Metrics   (src/phase1/phase1.cpp:18)
    run_phase2(num_partitions)                ->  PartitioningMetrics (src/phase2/phase2.cpp:256)

with the same metric definitions.  Differences: a fixed-iteration mode (exactly `iterations` iterations,
no stopping rule), an uncapped label mode (all k labels scored instead of the first 32), seed completion
when the reference's seed rule finds fewer than k seeds, and errors returned as exceptions where the
reference calls MPI_Abort.  There is no CPU fallback: every call runs the
CUDA library, and a missing library or GPU raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import byref, c_int64, c_void_p
from dataclasses import dataclass, field

import numpy as np

from . import _native, cabi
from .graphs import Graph


class DmolpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dmolp error {code}: {msg}")
        self.code = code


def _p(a: np.ndarray) -> c_void_p:
    return a.ctypes.data_as(c_void_p)


@dataclass
class Phase1Metrics:  # include/graph_types.h:276-309
    initial_edge_cut: int
    initial_vertex_balance: float
    initial_edge_balance: float
    total_vertices: int
    total_edges: int
    partition_vertex_counts: list
    partition_edge_counts: list
    seeds: list
    num_seeds_found: int
    rounds: int
    num_hubs: int
    traversed_edges: int
    gpu_ms: float
    stage_ms: dict = field(default_factory=dict)  # hubs / seeds / expand (wall clock)


@dataclass
class PartitioningMetrics:  # include/graph_types.h:312-346
    edge_cut: int
    vertex_balance: float
    edge_balance: float
    num_partitions: int
    total_vertices: int
    total_edges: int
    iterations_run: int
    stop_reason: int
    traversed_edges: int
    gpu_ms: float
    records: list = field(default_factory=list)


STOP_REASONS = {0: "iteration limit", 1: "empty window", 2: "no changes", 3: "converged", 4: "error"}


def load_adjtext(path: str) -> Graph:
    """Parse the reference's adjacency text with the native loader (rows sorted, de-duplicated)."""
    lib = _native.core()
    h = c_void_p()
    if lib.dmolp_adjtext_load(os.fsencode(path), byref(h)) != 0:
        raise DmolpError(cabi.DMOLP_ERR_ARG, lib.dmolp_adjtext_error().decode())
    try:
        nv = lib.dmolp_host_graph_nv(h)
        na = lib.dmolp_host_graph_narcs(h)
        off = np.ctypeslib.as_array(ctypes.cast(lib.dmolp_host_graph_offsets(h), ctypes.POINTER(ctypes.c_int64)),
                                    shape=(nv + 1,)).copy()
        col = (np.ctypeslib.as_array(ctypes.cast(lib.dmolp_host_graph_indices(h), ctypes.POINTER(ctypes.c_int32)),
                                     shape=(na,)).copy() if na else np.zeros(0, np.int32))
        raw = (np.ctypeslib.as_array(ctypes.cast(lib.dmolp_host_graph_raw_degree(h), ctypes.POINTER(ctypes.c_int32)),
                                     shape=(nv,)).copy() if nv else np.zeros(0, np.int32))
    finally:
        lib.dmolp_host_graph_free(h)
    return Graph(off, col, raw, name=os.path.basename(path))


class Partitioner:
    """One CUDA device, one resident graph."""

    def __init__(self, device: int = 0):
        self.lib = _native.core()
        self.ctx = c_void_p()
        self._check(self.lib.dmolp_create(device, byref(self.ctx)))
        self.graph: Graph | None = None
        self.num_vertices = 0
        self.raw_total: int | None = None  # sum of raw degrees of a device-parsed graph

    def _check(self, rc: int) -> None:
        if rc != cabi.DMOLP_OK:
            raise DmolpError(rc, self.lib.dmolp_last_error().decode())

    def close(self) -> None:
        if self.ctx:
            self.lib.dmolp_destroy(self.ctx)
            self.ctx = c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- graph and labels ----
    def upload(self, g: Graph) -> None:
        off = np.ascontiguousarray(g.offsets, np.int64)
        col = np.ascontiguousarray(g.indices, np.int32)
        raw = None if g.raw_degree is None else np.ascontiguousarray(g.raw_degree, np.int32)
        self._check(self.lib.dmolp_graph_upload(self.ctx, g.num_vertices, g.num_arcs, _p(off), _p(col),
                                                None if raw is None else _p(raw)))
        self.graph = g
        self.num_vertices = g.num_vertices
        self.raw_total = None

    def upload_adjtext(self, source) -> dict:
        """Parse the reference's adjacency text on the device into the resident graph.  `source` is a file
        path (read through the pinned staging ring), the text itself (bytes), or the text already on the
        device (a uint8 CUDA tensor).  Returns sizes and times."""
        info = cabi.IngestInfo()
        if hasattr(source, "data_ptr"):  # a uint8 CUDA tensor on this context's device
            self._check(self.lib.dmolp_graph_upload_adjtext_device(self.ctx, c_void_p(source.data_ptr()),
                                                                   source.numel(), byref(info)))
        elif isinstance(source, (bytes, bytearray, memoryview)):
            data = bytes(source)
            self._check(self.lib.dmolp_graph_upload_adjtext(self.ctx, data, len(data), byref(info)))
        else:
            self._check(self.lib.dmolp_graph_load_adjtext(self.ctx, os.fsencode(source), byref(info)))
        self.graph = None
        self.num_vertices = int(info.num_vertices)
        self.raw_total = int(info.num_tokens)
        return {f: getattr(info, f) for f, _ in cabi.IngestInfo._fields_}

    def graph_arrays(self) -> Graph:
        """The resident graph copied back to the host (offsets, indices, raw degree)."""
        nv, na = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.dmolp_graph_size(self.ctx, byref(nv), byref(na)))
        off = np.empty(nv.value + 1, np.int64)
        col = np.empty(na.value, np.int32)
        raw = np.empty(nv.value, np.int32)
        self._check(self.lib.dmolp_graph_get(self.ctx, _p(off), _p(col), _p(raw)))
        return Graph(off, col, raw)

    def labels(self) -> np.ndarray:
        out = np.empty(self.num_vertices, np.int32)
        self._check(self.lib.dmolp_labels_get(self.ctx, _p(out)))
        return out

    def set_labels(self, labels) -> None:
        lab = np.ascontiguousarray(labels, np.int32)
        if lab.shape[0] != self.num_vertices:
            raise ValueError("labels length != number of vertices")
        self._check(self.lib.dmolp_labels_set(self.ctx, _p(lab)))

    def symmetric(self) -> bool:
        """Whether the resident graph is symmetric with strictly increasing rows (the LP loop then updates cut
        and balance from the movers alone); runs the symmetry test now if the loop has not yet."""
        out = ctypes.c_int()
        self._check(self.lib.dmolp_graph_symmetric(self.ctx, byref(out)))
        return bool(out.value)

    def set_symmetry_test(self, exact: bool) -> None:
        """exact=False (default): keyed multiset sums in one pass; exact=True: every reverse arc looked up."""
        self._check(self.lib.dmolp_set_symmetry_test(self.ctx, 1 if exact else 0))

    def kernel_launches(self) -> int:
        return int(self.lib.dmolp_kernel_launches(self.ctx))

    # ---- phase 1 ----
    def phase1(self, k: int, theta: int) -> Phase1Metrics:
        seeds = np.empty(k, np.int32)
        vc = np.empty(k, np.int64)
        ec = np.empty(k, np.int64)
        info = cabi.Phase1Info()
        self._check(self.lib.dmolp_phase1(self.ctx, k, theta, _p(seeds), _p(vc), _p(ec), byref(info)))
        g = self.graph
        return Phase1Metrics(
            initial_edge_cut=info.initial_edge_cut, initial_vertex_balance=info.initial_vertex_balance,
            initial_edge_balance=info.initial_edge_balance, total_vertices=self.num_vertices,
            total_edges=(int(g.raw_deg().astype(np.int64).sum() // 2) if g is not None
                         else (self.raw_total or 0) // 2),
            partition_vertex_counts=vc.tolist(), partition_edge_counts=ec.tolist(), seeds=seeds.tolist(),
            num_seeds_found=info.num_seeds_found, rounds=info.rounds, num_hubs=info.num_hubs,
            traversed_edges=info.traversed_edges, gpu_ms=info.gpu_ms,
            stage_ms={"hubs": info.hubs_ms, "seeds": info.seeds_ms, "expand": info.expand_ms})

    # ---- phase 2 ----
    def phase2(self, k: int, mode: str = "ref", iterations: int = 20, cap: str = "ref",
               records: bool = True) -> PartitioningMetrics:
        cfg = cabi.LpConfig(cabi.MODE_REF if mode == "ref" else cabi.MODE_FIXED, iterations,
                            cabi.CAP_REF if cap == "ref" else cabi.CAP_FULL, 0)
        res = cabi.LpResult()
        nrec = 500
        recs = (cabi.LpRecord * nrec)() if records else None
        self._check(self.lib.dmolp_lp_run(self.ctx, k, byref(cfg), byref(res),
                                          ctypes.cast(recs, c_void_p) if records else None, nrec if records else 0))
        rl = [recs[i] for i in range(res.iterations_run)] if records else []
        return PartitioningMetrics(
            edge_cut=res.edge_cut, vertex_balance=res.vertex_balance, edge_balance=res.edge_balance,
            num_partitions=k, total_vertices=res.total_vertices, total_edges=res.total_edges,
            iterations_run=res.iterations_run, stop_reason=res.stop_reason, traversed_edges=res.traversed_edges,
            gpu_ms=res.gpu_ms, records=rl)

    def history(self, k: int, iters: int):
        pen = np.zeros((iters, k), np.float64)
        cnt = np.zeros((iters, 2 * k), np.int64)
        self._check(self.lib.dmolp_lp_history(self.ctx, k, iters, _p(pen), _p(cnt)))
        return pen, cnt

    def metrics(self, k: int):
        cut = c_int64()
        vc = np.empty(k, np.int64)
        ec = np.empty(k, np.int64)
        self._check(self.lib.dmolp_metrics(self.ctx, k, byref(cut), _p(vc), _p(ec)))
        return cut.value, vc, ec

    # ---- single steps (the reference's expandBoundaryNodes / runBoundaryLPOnGPU_*) ----
    def window_select(self, k: int, iteration: int, RE, prev) -> np.ndarray:
        re = np.ascontiguousarray(RE, np.float64)
        pv = np.ascontiguousarray(prev, np.int32)
        out = np.empty(max(1, self.num_vertices), np.int32)
        n = c_int64()
        self._check(self.lib.dmolp_window_select(self.ctx, k, iteration, _p(re), _p(pv), pv.shape[0], _p(out),
                                                 byref(n)))
        return out[:n.value].copy()

    def lp_apply(self, k: int, penalty, window, cap: str = "ref"):
        pen = np.ascontiguousarray(penalty, np.float64)
        w = np.ascontiguousarray(window, np.int32)
        nodes = np.empty(max(1, w.shape[0]), np.int32)
        labs = np.empty(max(1, w.shape[0]), np.int32)
        n = c_int64()
        self._check(self.lib.dmolp_lp_apply(self.ctx, k, cabi.CAP_REF if cap == "ref" else cabi.CAP_FULL, _p(pen),
                                            _p(w), w.shape[0], _p(nodes), _p(labs), byref(n)))
        return nodes[:n.value].copy(), labs[:n.value].copy()


def run_phase1(graph_file: str, num_parts: int, theta: int, device: int = 0):
    """The reference's run_phase1 (src/phase1/phase1.cpp:18) at one rank: returns (metrics, partitioner); the
    partitioner keeps the graph and the phase-1 labels resident for run_phase2."""
    p = Partitioner(device)
    p.upload_adjtext(graph_file)  # parsed on the device into the resident graph
    return p.phase1(num_parts, theta), p


def run_phase2(p: Partitioner, num_partitions: int, mode: str = "ref", iterations: int = 20,
               cap: str = "ref") -> PartitioningMetrics:
    """The reference's run_phase2 (src/phase2/phase2.cpp:256) on the partitioner's resident labels."""
    return p.phase2(num_partitions, mode=mode, iterations=iterations, cap=cap)
