"""Learned initial partition over libdmolp_b200.so (include/dmolp_b200.h, dmolp_mpnn_* / dmolp_batch_propose).

A 3-layer mean-aggregation message-passing network (BF16 weights, FP32 accumulation on the tensor cores,
the project's own forward and backward kernels) runs over every vertex of a batch of graphs.  Its first 8
outputs are a residual on the 8 random-walk features (proposal coordinates, cut into k balanced labels per
graph by recursive inertial bisection); its output 8, averaged over a graph, is a learned gate that says
whether the proposal will end at an edge cut no higher than phase 1's.  The proposal replaces phase 1
(BFS / hub seeding) as the start of phase 2 where the gate accepts it; elsewhere phase 1 is the fallback.
The gate is trained on runs of the plain method (phase 1 + phase 2): which start ended lower.
"""
from __future__ import annotations

import os
import time
from ctypes import byref, c_double, c_float, c_void_p

import numpy as np

from . import _native
from .batch import Batch, Instance, random_instances, union
from .partitioner import DmolpError, Partitioner

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "proposal.npy")


def _p(a: np.ndarray) -> c_void_p:
    return a.ctypes.data_as(c_void_p)


class Proposal:
    """The network on one GPU: parameters, optimiser state and a workspace sized for the largest batch."""

    def __init__(self, device: int = 0, params: np.ndarray | str | None = None):
        self.lib = _native.core()
        self.device = device
        h = c_void_p()
        self._check(self.lib.dmolp_mpnn_create(device, byref(h)))
        self.h = h
        self.n = int(self.lib.dmolp_mpnn_num_params())
        if isinstance(params, str):
            params = np.load(params)
        if params is not None:
            self.set_params(params)

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise DmolpError(rc, self.lib.dmolp_last_error().decode())

    def close(self) -> None:
        if self.h:
            self.lib.dmolp_mpnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters ----
    def params(self) -> np.ndarray:
        out = np.empty(self.n, np.float32)
        self._check(self.lib.dmolp_mpnn_get_params(self.h, _p(out)))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n
        self._check(self.lib.dmolp_mpnn_set_params(self.h, _p(p)))

    def save(self, path: str = WEIGHTS) -> None:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.save(path, self.params())

    # ---- passes ----
    def prepare_training(self, b: Batch) -> None:
        self._check(self.lib.dmolp_mpnn_prepare_training(self.h, b.h))

    def features(self, b: Batch, copy: bool = True) -> np.ndarray | None:
        out = np.empty((b.num_vertices, 16), np.float32) if copy else None
        self._check(self.lib.dmolp_mpnn_features(self.h, b.h, _p(out) if copy else None))
        return out

    def set_features(self, b: Batch, X: np.ndarray) -> None:
        X = np.ascontiguousarray(X, np.float32)
        self._check(self.lib.dmolp_mpnn_set_features(self.h, b.h, _p(X)))

    def forward(self, b: Batch, copy: bool = True) -> np.ndarray | None:
        out = np.empty((b.num_vertices, 16), np.float32) if copy else None
        self._check(self.lib.dmolp_mpnn_forward(self.h, b.h, _p(out) if copy else None))
        return out

    def backward(self, b: Batch, dZ: np.ndarray) -> np.ndarray:
        dZ = np.ascontiguousarray(dZ, np.float32)
        g = np.empty(self.n, np.float32)
        self._check(self.lib.dmolp_mpnn_backward(self.h, b.h, _p(dZ), _p(g)))
        return g

    def train_step(self, b: Batch, target: np.ndarray, lr: float) -> float:
        t = np.ascontiguousarray(target, np.int32)
        loss = c_double()
        self._check(self.lib.dmolp_mpnn_train_step(self.h, b.h, _p(t), c_float(lr), byref(loss)))
        return loss.value

    def gate(self, b: Batch) -> np.ndarray:
        out = np.empty(b.num_instances, np.float64)
        self._check(self.lib.dmolp_mpnn_gate(self.h, b.h, _p(out)))
        return out

    def train_gate(self, b: Batch, y: np.ndarray, lr: float) -> float:
        t = np.ascontiguousarray(y, np.float32)
        loss = c_double()
        self._check(self.lib.dmolp_mpnn_train_gate(self.h, b.h, _p(t), c_float(lr), byref(loss)))
        return loss.value

    def decode(self, b: Batch, Z: np.ndarray | None = None) -> np.ndarray:
        st = np.empty(b.num_instances, np.int32)
        z = None if Z is None else np.ascontiguousarray(Z, np.float32)
        self._check(self.lib.dmolp_mpnn_decode(self.h, b.h, None if z is None else _p(z), _p(st)))
        return st

    def propose(self, b: Batch) -> np.ndarray:
        """Labels of every graph of the batch from the network (into the batch); returns per-graph status
        (0 = proposal used, 1 = proposal not usable, 2 = the gate prefers phase 1)."""
        st = np.empty(b.num_instances, np.int32)
        self._check(self.lib.dmolp_batch_propose(b.h, self.h, _p(st)))
        return st


def phase1_labels(instances: list[Instance], theta: int, device: int = 0, which=None) -> list[np.ndarray]:
    """The plain seeding (phase 1 of the single-graph path, one graph after another) for the given
    instances."""
    p = Partitioner(device)
    out = []
    for i, it in enumerate(instances):
        if which is not None and not which[i]:
            out.append(None)
            continue
        p.upload(it.graph)
        p.phase1(it.k, theta)
        out.append(p.labels())
    p.close()
    return out


def propose_with_fallback(model: Proposal, b: Batch, instances: list[Instance] | None = None, theta: int = 1000,
                          device: int = 0) -> tuple[np.ndarray, float]:
    """Learned labels for every graph of the batch, phase-1 seeding (batched, one launch) for the graphs the
    proposal flags.  Returns (status per graph, seconds spent in the fallback)."""
    st = model.propose(b)
    t = 0.0
    if st.any():
        t0 = time.perf_counter()
        b.phase1(theta, only=st != 0)
        t = time.perf_counter() - t0
    return st, t


def plain_targets(instances: list[Instance], theta: int = 1000, device: int = 0) -> list[np.ndarray]:
    """Final partitions of the plain method (phase 1, then phase 2 with the reference's stopping rules),
    computed for many graphs at once with the batched phase 2 (identical per graph to the single-graph
    path)."""
    lab1 = phase1_labels(instances, theta, device)
    b = Batch(device)
    b.upload(instances)
    b.set_labels(lab1)
    b.run("ref")
    out = b.split(b.labels())
    b.close()
    return [x.copy() for x in out]


def train_gate(model: Proposal, sets: list[tuple[list[Instance], np.ndarray]], epochs: int, lr: float = 1e-3,
               device: int = 0, log=None) -> list[float]:
    """Adam on the gate's binary cross-entropy over training minibatches (graphs, 0/1 targets)."""
    prepared = []
    for inst, y in sets:
        b = Batch(device)
        b.upload(inst)
        model.prepare_training(b)
        X = model.features(b)
        prepared.append((b, X, np.asarray(y, np.float32)))
    losses = []
    for ep in range(epochs):
        tot = 0.0
        for b, X, y in prepared:
            model.set_features(b, X)
            tot += model.train_gate(b, y, lr)
        losses.append(tot / len(prepared))
        if log:
            log(ep, losses[-1])
    for b, _, _ in prepared:
        b.close()
    return losses


def train(model: Proposal, sets: list[tuple[list[Instance], list[np.ndarray]]], epochs: int, lr: float = 1e-3,
          device: int = 0, log=None) -> list[float]:
    """Adam on the edge-contrastive loss over training minibatches (each a list of graphs and their target
    partitions); features are computed once per minibatch."""
    prepared = []
    for inst, tgt in sets:
        b = Batch(device)
        b.upload(inst)
        model.prepare_training(b)
        X = model.features(b)
        prepared.append((b, X, np.concatenate(tgt).astype(np.int32)))
    losses = []
    for ep in range(epochs):
        tot = 0.0
        for b, X, t in prepared:
            model.set_features(b, X)
            tot += model.train_step(b, t, lr)
        losses.append(tot / len(prepared))
        if log:
            log(ep, losses[-1])
    for b, _, _ in prepared:
        b.close()
    return losses


def evaluate_large(model: Proposal, g, k: int, theta: int, device: int = 0) -> dict:
    """One large graph, k parts: the plain method (phase 1, then phase 2 with the reference's stopping rules,
    on the single-graph path) against the learned start -- the proposal where the gate accepts it, phase 1
    where it declines -- and against the proposal itself with the gate ignored.  Per start: edge cut, vertex
    and edge balance, iterations to converge, wall time of the start and of phase 2."""
    import torch

    def run_from(p: Partitioner, labels: np.ndarray | None) -> dict:
        if labels is not None:
            p.set_labels(labels)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m = p.phase2(k, mode="ref", records=False)
        return {"edge_cut": int(m.edge_cut), "vertex_balance": m.vertex_balance, "edge_balance": m.edge_balance,
                "iterations": int(m.iterations_run), "phase2_s": time.perf_counter() - t0}

    p = Partitioner(device)
    p.upload(g)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    p.phase1(k, theta)
    plain_start_s = time.perf_counter() - t0
    lab1 = p.labels()
    plain = run_from(p, None)
    plain["start_s"] = plain_start_s
    b = Batch(device)
    b.upload([Instance(g, k, "eval")])
    model.propose(b)  # workspace set-up for this size (not timed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = model.propose(b)
    gate = float(model.gate(b)[0])
    prop_s = time.perf_counter() - t0
    out = {"num_vertices": g.num_vertices, "num_arcs": g.num_arcs, "k": k, "theta": theta, "plain": plain,
           "gate_score": gate, "gate_accepts": bool(st[0] == 0)}
    forced_st = st if st[0] == 0 else model.decode(b)  # the proposal with the gate ignored
    if forced_st[0] == 0:
        forced = run_from(p, b.labels())
        forced["start_s"] = prop_s
        out["proposal_gate_ignored"] = forced
    out["learned"] = out.get("proposal_gate_ignored") if st[0] == 0 else dict(plain, start_s=plain_start_s + prop_s)
    b.close()
    p.set_labels(lab1)
    p.close()
    return out
