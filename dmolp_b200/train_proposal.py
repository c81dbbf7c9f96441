"""Train the learned initial partition on runs of the plain method, then compare it with the plain method
on held-out graphs.

    python -m dmolp_b200.train_proposal --train 10240 --vmax 200000 --epochs 30 --lr 0.003 --pos-repeat 5 \
        --eval 256 --out dmolp_b200/weights/proposal.npy --report report.json

(the command that made the shipped weights, dmolp_b200/weights/proposal.npy, and its record
proposal_training.json beside them).

Training graphs and held-out graphs come from the batched workload's distribution (vertex counts
log-uniform in [vmin, vmax], half k-NN 2-D/3-D, half preferential attachment, k uniform in 2..64) with
different seeds.  Per training graph the plain method (phase 1 = BFS / hub seeding, then phase 2 with the
reference's stopping rules) and the proposal followed by the same phase 2 are both run; the gate's target is
1 where the proposal ended at an edge cut no higher than the plain method's.  Evaluation, per held-out
graph: the plain method, the proposal with the trained gate (phase 1 where the gate declines), and the
proposal without it (the untrained gate accepts every graph) -- edge cut, vertex balance, iterations to
converge -- plus the wall time of each start.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .batch import Batch, random_instances
from .learned import WEIGHTS, Proposal, phase1_labels, propose_with_fallback, train_gate


def evaluate(model: Proposal, inst, plain, theta: int, device: int = 0) -> dict:
    """Phase 2 from the model's proposal (phase 1 where it falls back) against the plain results."""
    b = Batch(device)
    b.upload(inst)
    t0 = time.perf_counter()
    st, fb_s = propose_with_fallback(model, b, inst, theta, device)
    start_s = time.perf_counter() - t0
    init = b.split(b.labels())
    init = [x.copy() for x in init]
    res, ms = b.run("ref")
    b.close()
    out = {"fallbacks": int((st != 0).sum()), "start_wall_s": start_s, "fallback_wall_s": fb_s, "lp_ms": ms,
           "cut": [r["edge_cut"] for r in res], "vertex_balance": [r["vertex_balance"] for r in res],
           "iterations": [r["iterations_run"] for r in res]}
    out["initial_cut"] = [int(cut_of(it.graph, l)) for it, l in zip(inst, init)]
    return out


def chunked_targets(inst, theta: int, chunk: int = 1024, device: int = 0) -> tuple[np.ndarray, dict]:
    """The gate's targets for many graphs, chunk by chunk (a batch per chunk): per graph the plain method
    (batched phase 1, identical per graph to the single-graph phase 1, then phase 2 with the reference's
    stopping rules) and the untrained proposal (accepted for every graph) followed by the same phase 2;
    target 1 where the proposal ended at an edge cut no higher than the plain method's."""
    y = np.zeros(len(inst), np.float32)
    model = Proposal(device)
    stats = {"plain_cut": 0, "proposal_cut": 0, "chunks": 0}
    for c0 in range(0, len(inst), chunk):
        part = inst[c0:c0 + chunk]
        b = Batch(device)
        b.upload(part)
        b.phase1(theta)
        plain, _ = b.run("ref")
        st = model.propose(b)
        if st.any():
            b.phase1(theta, only=st != 0)
        prop, _ = b.run("ref")
        b.close()
        pc = np.array([r["edge_cut"] for r in plain])
        qc = np.array([r["edge_cut"] for r in prop])
        y[c0:c0 + len(part)] = (qc <= pc).astype(np.float32)
        stats["plain_cut"] += int(pc.sum())
        stats["proposal_cut"] += int(qc.sum())
        stats["chunks"] += 1
    model.close()
    return y, stats


def cut_of(g, lab) -> int:
    src = np.repeat(np.arange(g.num_vertices), np.diff(g.offsets))
    return int((lab[src] != lab[g.indices]).sum() // 2)


def plain_eval(inst, theta: int, device: int = 0) -> dict:
    t0 = time.perf_counter()
    lab1 = phase1_labels(inst, theta, device)
    p1_s = time.perf_counter() - t0
    b = Batch(device)
    b.upload(inst)
    b.set_labels(lab1)
    res, ms = b.run("ref")
    b.close()
    return {"phase1_wall_s": p1_s, "lp_ms": ms, "cut": [r["edge_cut"] for r in res],
            "vertex_balance": [r["vertex_balance"] for r in res], "iterations": [r["iterations_run"] for r in res],
            "initial_cut": [cut_of(it.graph, l) for it, l in zip(inst, lab1)]}


def summary(plain: dict, other: dict) -> dict:
    pc, oc = np.array(plain["cut"], float), np.array(other["cut"], float)
    return {"cut_ratio_total": float(oc.sum() / max(1.0, pc.sum())),
            "cut_ratio_median": float(np.median(oc / np.maximum(pc, 1))),
            "graphs_better_or_equal": int((oc <= pc).sum()),
            "vertex_balance_mean": float(np.mean(other["vertex_balance"])),
            "vertex_balance_max": float(np.max(other["vertex_balance"])),
            "iterations_mean": float(np.mean(other["iterations"])),
            "initial_cut_ratio_total": float(np.sum(other["initial_cut"]) / max(1, np.sum(plain["initial_cut"])))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2048, help="training graphs")
    ap.add_argument("--eval", type=int, default=256, help="held-out graphs")
    ap.add_argument("--vmin", type=int, default=1000)
    ap.add_argument("--vmax", type=int, default=200_000)
    ap.add_argument("--minibatch", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--theta", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=101)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    ap.add_argument("--chunk", type=int, default=1024, help="graphs per batch when computing the targets")
    ap.add_argument("--pos-repeat", type=int, default=1,
                    help="each graph whose target is 1 appears this many times in the training minibatches")
    a = ap.parse_args()
    rep = {"args": vars(a)}
    t0 = time.time()
    tr = random_instances(a.train, seed=a.seed, vmin=a.vmin, vmax=a.vmax)
    rep["generate_s"] = time.time() - t0
    t0 = time.time()
    y, rep["target_stats"] = chunked_targets(tr, a.theta, a.chunk)
    rep["targets_s"] = time.time() - t0
    rep["train_targets_positive"] = float(y.mean())
    idx = np.arange(len(tr))
    if a.pos_repeat > 1:  # balance the classes by repeating the (rarer) positive graphs
        idx = np.concatenate([idx] + [np.nonzero(y > 0.5)[0]] * (a.pos_repeat - 1))
        np.random.default_rng(a.seed).shuffle(idx)
    rep["train_samples"] = int(len(idx))
    sets = [([tr[j] for j in idx[i:i + a.minibatch]], y[idx[i:i + a.minibatch]])
            for i in range(0, len(idx), a.minibatch)]
    model = Proposal(0)
    t0 = time.time()
    losses = train_gate(model, sets, a.epochs, a.lr, log=lambda ep, l: print(f"epoch {ep} loss {l:.5f}", flush=True))
    rep["train_s"] = time.time() - t0
    rep["losses"] = losses
    model.save(a.out)
    del tr, sets
    if a.eval > 0:
        ev = random_instances(a.eval, seed=a.seed + 1, vmin=a.vmin, vmax=a.vmax)
        plain = plain_eval(ev, a.theta)
        learned = evaluate(model, ev, plain, a.theta)
        untrained = evaluate(Proposal(0), ev, plain, a.theta)
        rep["eval"] = {"graphs": a.eval, "plain": {k: v for k, v in plain.items() if not isinstance(v, list)},
                       "learned": summary(plain, learned), "untrained": summary(plain, untrained),
                       "plain_summary": summary(plain, plain),
                       "learned_start_wall_s": learned["start_wall_s"], "learned_fallbacks": learned["fallbacks"],
                       "learned_fallback_wall_s": learned["fallback_wall_s"],
                       "untrained_start_wall_s": untrained["start_wall_s"],
                       "learned_lp_ms": learned["lp_ms"], "untrained_lp_ms": untrained["lp_ms"]}
        print(json.dumps(rep["eval"], indent=1))
    if a.report:
        json.dump(rep, open(a.report, "w"), indent=1)


if __name__ == "__main__":
    main()
