"""Seeded synthetic graphs (C++ generators in csrc/graphgen.cpp) as numpy CSR arrays.

A graph is undirected and stored as a CSR with int64 offsets, int32 neighbour ids, rows sorted and
de-duplicated, no self-loops.  ``raw_degree`` is the per-vertex token count of the adjacency text the
reference reads; for generated graphs it equals the CSR degree.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

from . import _native


@dataclass
class Graph:
    offsets: np.ndarray  # int64 [V+1]
    indices: np.ndarray  # int32 [arcs]
    raw_degree: np.ndarray | None = None  # int32 [V]
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def num_vertices(self) -> int:
        return int(self.offsets.shape[0] - 1)

    @property
    def num_arcs(self) -> int:
        return int(self.indices.shape[0])

    def degree(self) -> np.ndarray:
        return np.diff(self.offsets).astype(np.int32)

    def raw_deg(self) -> np.ndarray:
        return self.raw_degree if self.raw_degree is not None else self.degree()


def _take(ptr) -> Graph:
    lib = _native.gen()
    nv = lib.dmolp_csr_nv(ptr)
    na = lib.dmolp_csr_narcs(ptr)
    off = np.empty(nv + 1, dtype=np.int64)
    col = np.empty(na, dtype=np.int32)
    lib.dmolp_csr_copy(ptr, off.ctypes.data_as(ctypes.c_void_p), col.ctypes.data_as(ctypes.c_void_p))
    lib.dmolp_csr_free(ptr)
    return Graph(off, col)


def _call(fn, *args) -> Graph:
    lib = _native.gen()
    out = ctypes.c_void_p()
    rc = fn(*args, ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(lib.dmolp_gen_last_error().decode())
    return _take(out)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 7,
         permute: bool = True) -> Graph:
    """Symmetrised R-MAT (self-loops and duplicates removed)."""
    g = _call(_native.gen().dmolp_gen_rmat, scale, edge_factor, a, b, c, seed, int(permute))
    g.name = f"rmat-s{scale}-ef{edge_factor}-seed{seed}"
    g.meta = dict(kind="rmat", scale=scale, edge_factor=edge_factor, a=a, b=b, c=c, seed=seed, permute=permute)
    return g


def knn(n: int, dim: int = 3, k: int = 12, seed: int = 1) -> Graph:
    """Symmetrised k-nearest-neighbour graph of n points uniform in [0,1)^dim."""
    g = _call(_native.gen().dmolp_gen_knn, n, dim, k, seed)
    g.name = f"knn{dim}d-n{n}-k{k}-seed{seed}"
    g.meta = dict(kind="knn", n=n, dim=dim, k=k, seed=seed)
    return g


def barabasi_albert(n: int, m: int, seed: int = 1) -> Graph:
    """Preferential attachment: each new vertex joins m distinct earlier vertices."""
    g = _call(_native.gen().dmolp_gen_ba, n, m, seed)
    g.name = f"ba-n{n}-m{m}-seed{seed}"
    g.meta = dict(kind="ba", n=n, m=m, seed=seed)
    return g


def band(n: int, wmin: int, wmax: int, seed: int = 1) -> Graph:
    """Band graph on a cycle: i ~ j when their cycle distance is at most max(w_i, w_j), w uniform in
    [wmin, wmax] (dense rows; large parameters give more than 2^31 arcs)."""
    g = _call(_native.gen().dmolp_gen_band, n, wmin, wmax, seed)
    g.name = f"band-n{n}-w{wmin}-{wmax}-seed{seed}"
    g.meta = dict(kind="band", n=n, wmin=wmin, wmax=wmax, seed=seed)
    return g


def from_edges(n: int, edges) -> Graph:
    """Undirected graph from an edge list (pairs); symmetrised, de-duplicated, self-loops dropped."""
    e = np.asarray(list(edges), dtype=np.int64).reshape(-1, 2)
    e = e[e[:, 0] != e[:, 1]]
    both = np.concatenate([e, e[:, ::-1]]) if len(e) else np.zeros((0, 2), np.int64)
    both = np.unique(both, axis=0)
    off = np.zeros(n + 1, dtype=np.int64)
    if len(both):
        np.add.at(off, both[:, 0] + 1, 1)
    off = np.cumsum(off)
    return Graph(off, both[:, 1].astype(np.int32) if len(both) else np.zeros(0, np.int32))


def fnv1a(a: np.ndarray) -> int:
    """64-bit FNV-1a over the array's bytes (the label fingerprint the parity fixtures record)."""
    a = np.ascontiguousarray(a)
    return int(_native.gen().dmolp_fnv1a(a.ctypes.data_as(ctypes.c_void_p), a.nbytes))


def write_adjtext(g: Graph, path: str) -> None:
    """Write the reference's adjacency text format (first line V; line i+1 = neighbours of i)."""
    lib = _native.gen()
    ptr = ctypes.c_void_p()
    off = np.ascontiguousarray(g.offsets, dtype=np.int64)
    col = np.ascontiguousarray(g.indices, dtype=np.int32)
    rc = lib.dmolp_csr_from_arrays(g.num_vertices, g.num_arcs, off.ctypes.data_as(ctypes.c_void_p),
                                   col.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ptr))
    if rc != 0:
        raise RuntimeError(lib.dmolp_gen_last_error().decode())
    try:
        rc = lib.dmolp_csr_write_adjtext(ptr, os.fsencode(path))
        if rc != 0:
            raise RuntimeError(lib.dmolp_gen_last_error().decode())
    finally:
        lib.dmolp_csr_free(ptr)
