"""Batched phase 2 over libdmolp_b200.so (include/dmolp_b200.h, dmolp_batch_*).

A batch is a list of independent graphs, each with its own part count k <= 64, partitioned together by one
persistent kernel launch (replayed from a captured CUDA graph).  Each instance follows run_phase2
(src/phase2/phase2.cpp:256-449) exactly as the single-graph path does.  The launch shape (threads per CTA,
the thread-row limit of the degree buckets, CTAs per SM) comes from the built-in autotuner; tuned shapes
are cached per GPU and batch signature in a JSON file.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
from concurrent.futures import ThreadPoolExecutor
from ctypes import byref, c_double, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _native, cabi, graphs
from .graphs import Graph
from .partitioner import DmolpError

MODES = {"ref": cabi.MODE_REF, "fixed": cabi.MODE_FIXED}
CAPS = {"ref": cabi.CAP_REF, "full": cabi.CAP_FULL}


def _p(a: np.ndarray) -> c_void_p:
    return a.ctypes.data_as(c_void_p)


@dataclass
class Instance:
    graph: Graph
    k: int
    family: str = ""


def random_instances(n: int, seed: int = 11, vmin: int = 1000, vmax: int = 200_000, threads: int | None = None
                     ) -> list[Instance]:
    """The batched workload's instance mix: vertex counts log-uniform in [vmin, vmax]; half random geometric
    k-NN graphs (2-D or 3-D points, k_nn uniform in 8..14), half preferential-attachment graphs (m uniform in
    4..8); part counts uniform in 2..64.  Deterministic in `seed`; generated in parallel on the host."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        nv = int(round(np.exp(rng.uniform(np.log(vmin), np.log(vmax)))))
        k = int(rng.integers(2, 65))
        gseed = int(rng.integers(1, 2**31 - 1))
        if i % 2 == 0:
            dim = int(rng.integers(2, 4))
            knn = int(rng.integers(8, 15))
            specs.append(("knn%dd" % dim, nv, k, gseed, dim, knn))
        else:
            m = int(rng.integers(4, 9))
            specs.append(("ba", nv, k, gseed, m, 0))

    def make(sp):
        fam, nv, k, gseed, a, b = sp
        g = graphs.knn(nv, a, b, seed=gseed) if fam.startswith("knn") else graphs.barabasi_albert(nv, a, seed=gseed)
        return Instance(g, k, fam)

    with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 4) as ex:
        return list(ex.map(make, specs))


def union(instances: list[Instance]) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(vstart[n+1], offsets[V+1], local indices[A], parts[n]) of the batch's union CSR."""
    nvs = np.array([it.graph.num_vertices for it in instances], np.int64)
    vstart = np.zeros(len(instances) + 1, np.int64)
    np.cumsum(nvs, out=vstart[1:])
    nas = np.array([it.graph.num_arcs for it in instances], np.int64)
    astart = np.zeros(len(instances) + 1, np.int64)
    np.cumsum(nas, out=astart[1:])
    off = np.empty(int(vstart[-1]) + 1, np.int64)
    col = np.empty(int(astart[-1]), np.int32)
    for i, it in enumerate(instances):
        g = it.graph
        off[vstart[i]:vstart[i + 1]] = g.offsets[:-1] + astart[i]
        col[astart[i]:astart[i + 1]] = g.indices
    off[-1] = astart[-1]
    parts = np.array([it.k for it in instances], np.int32)
    return vstart, off, col, parts


class Batch:
    """A batch resident on one GPU."""

    def __init__(self, device: int = 0):
        self.lib = _native.core()
        self.device = device
        h = c_void_p()
        self._check(self.lib.dmolp_batch_create(device, byref(h)))
        self.h = h
        self.vstart = None
        self.parts = None
        self.tuning = None

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise DmolpError(rc, self.lib.dmolp_last_error().decode())

    def close(self) -> None:
        if self.h:
            self.lib.dmolp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- data ----
    def upload(self, instances: list[Instance] | None = None, arrays=None) -> None:
        vstart, off, col, parts = arrays if arrays is not None else union(instances)
        self._check(self.lib.dmolp_batch_upload(self.h, len(parts), _p(vstart), _p(off), _p(col), _p(parts)))
        self.vstart, self.parts = vstart, parts
        self.signature = hashlib.sha1(np.concatenate([vstart, parts.astype(np.int64),
                                                      off[vstart[1:]]]).tobytes()).hexdigest()[:16]

    @property
    def num_instances(self) -> int:
        return len(self.parts)

    @property
    def num_vertices(self) -> int:
        return int(self.vstart[-1])

    def set_labels(self, labels) -> None:
        lab = np.ascontiguousarray(np.concatenate(labels) if isinstance(labels, (list, tuple)) else labels,
                                   dtype=np.int32)
        assert lab.size == self.num_vertices
        self._check(self.lib.dmolp_batch_labels_set(self.h, _p(lab)))

    def labels(self) -> np.ndarray:
        out = np.empty(self.num_vertices, np.int32)
        self._check(self.lib.dmolp_batch_labels_get(self.h, _p(out)))
        return out

    def split(self, union_array: np.ndarray) -> list[np.ndarray]:
        return [union_array[self.vstart[i]:self.vstart[i + 1]] for i in range(self.num_instances)]

    def save_labels(self) -> None:
        self._check(self.lib.dmolp_batch_labels_save(self.h))

    def restore_labels(self) -> None:
        self._check(self.lib.dmolp_batch_labels_restore(self.h))

    def device_labels(self) -> int:
        p = c_void_p()
        self._check(self.lib.dmolp_batch_device_labels(self.h, byref(p)))
        return p.value

    def stream(self) -> int:
        return self.lib.dmolp_batch_stream(self.h)

    # ---- runs ----
    @staticmethod
    def _cfg(mode: str, iterations: int, cap: str) -> cabi.LpConfig:
        return cabi.LpConfig(MODES[mode], iterations, CAPS[cap], 0)

    def run(self, mode: str = "ref", iterations: int = 0, cap: str = "ref", tuning: dict | None = None,
            results: bool = True):
        """Phase 2 on every instance.  Returns (list of per-instance dicts or None, device ms)."""
        cfg = self._cfg(mode, iterations, cap)
        shape = tuning or self.tuning  # an explicit shape, else the tuned (or cached) one, else the default
        t = cabi.BatchTuning(**shape) if shape else None
        res = (cabi.BatchResult * self.num_instances)() if results else None
        ms = c_double()
        rc = self.lib.dmolp_batch_lp_run(self.h, byref(cfg), byref(t) if t else None, res, byref(ms))
        self._check(rc)
        if res is None:
            return None, ms.value
        out = [{f: getattr(r, f) for f, _ in cabi.BatchResult._fields_} for r in res]
        return out, ms.value

    def phase1(self, theta: int, seeds: bool = False, only=None):
        """Phase 1 (BFS / hub seeding) for every graph (or those with only[i] true), labels into the batch.
        Returns (per-graph dicts, seeds [n, 64] or None, device ms)."""
        res = (cabi.BatchP1Result * self.num_instances)()
        sd = np.empty((self.num_instances, cabi.BATCH_MAX_K), np.int32) if seeds else None
        mask = None if only is None else np.ascontiguousarray(np.asarray(only, bool), np.uint8)
        ms = c_double()
        self._check(self.lib.dmolp_batch_phase1(self.h, theta, None if mask is None else _p(mask),
                                                _p(sd) if seeds else None, res, byref(ms)))
        out = [{f: getattr(r, f) for f, _ in cabi.BatchP1Result._fields_} for r in res]
        return out, sd, ms.value

    def counts(self, i: int) -> tuple[np.ndarray, np.ndarray]:
        k = int(self.parts[i])
        vc = np.zeros(k, np.int64)
        ec = np.zeros(k, np.int64)
        self._check(self.lib.dmolp_batch_counts(self.h, i, _p(vc), _p(ec)))
        return vc, ec

    def autotune(self, mode: str = "ref", iterations: int = 0, cap: str = "ref", cache: str | None = None) -> dict:
        """Time every launch shape on this batch (labels restored) and keep the fastest.  With `cache`, a
        JSON file keyed by GPU name and batch signature, a shape tuned before is reused without timing."""
        key = None
        if cache:
            import torch

            key = "%s|%s|%s|%d|%s" % (torch.cuda.get_device_name(self.device), self.signature, mode, iterations, cap)
            try:
                db = json.load(open(cache))
            except (OSError, ValueError):
                db = {}
            if key in db:
                self.tuning = db[key]["tuning"]
                return dict(self.tuning, cached=True, ms=db[key]["ms"])
        cfg = self._cfg(mode, iterations, cap)
        best = cabi.BatchTuning()
        ms = c_double()
        self._check(self.lib.dmolp_batch_autotune(self.h, byref(cfg), byref(best), byref(ms)))
        self.tuning = {f: getattr(best, f) for f, _ in cabi.BatchTuning._fields_}
        if cache:
            try:
                db = json.load(open(cache))
            except (OSError, ValueError):
                db = {}
            db[key] = {"tuning": self.tuning, "ms": ms.value}
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            json.dump(db, open(cache, "w"), indent=1, sort_keys=True)
        return dict(self.tuning, cached=False, ms=ms.value)
