#!/usr/bin/env python
"""Benchmark of the DMOLP partitioning hot path on B200: label-propagation traversed edges per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload rmat22] [--impl ours|reference]

A step is one phase-2 run (the fixed number of LP iterations of the workload) from the phase-1 partition,
on a graph resident in HBM.  Traversed edges (TE) per iteration = sum of degrees over the previous window,
over the candidates and over the selected window, plus all arcs for the statistics pass; the same count
the oracle and the reference harness report.

One JSON line on stdout (rank 0).  With --gpus N (launched under torchrun) every rank runs the same
workload on its own GPU: the path does not shard a single graph, so N GPUs are N independent replicas.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # R-MAT scale 22, edge factor 16, (.57,.19,.19,.05), seed 7, k = 32, 30 LP iterations
    "rmat22": dict(kind="rmat", scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7, k=32, theta=10000,
                   iters=30),
    "rmat22-k16": dict(kind="rmat", scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7, k=16, theta=10000,
                       iters=30),
    "rmat22-k64": dict(kind="rmat", scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7, k=64, theta=10000,
                       iters=30),
    # R-MAT scale 26, edge factor 24 (67.1 M vertices, ~3.2 B arcs), k = 64, 40 LP iterations
    "rmat26": dict(kind="rmat", scale=26, edge_factor=24, a=0.57, b=0.19, c=0.19, seed=7, k=64, theta=10000,
                   iters=40),
    # 3-D k-NN (k=12), 55,476 points, k = 8, 20 LP iterations
    "knn-c0": dict(kind="knn", n=55476, dim=3, knn=12, seed=1, k=8, theta=1000, iters=20),
    # 2048 graphs, V log-uniform in [1K, 200K], half k-NN 2-D/3-D (k_nn 8..14), half preferential attachment
    # (m 4..8), k uniform in 2..64; phase 2 with the reference's stopping rules from phase-1 partitions
    "batch2048": dict(kind="batch", n=2048, seed=11, vmin=1000, vmax=200_000, theta=1000),
    # the same mix, 256 graphs (profiling and quick checks)
    "batch256": dict(kind="batch", n=256, seed=11, vmin=1000, vmax=200_000, theta=1000),
    # the rmat22 graph as the reference's adjacency text, parsed into the resident CSR
    "ingest-rmat22": dict(kind="ingest", graph=dict(kind="rmat", scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19,
                                                    seed=7)),
    # the learned proposal against the plain method on R-MAT scale 24 and a 3-D geometric 2 M-vertex graph, k = 32
    "learned-eval": dict(kind="learned"),
}


def rank_seed(seed: int, rank: int) -> int:
    """Each rank of a multi-GPU run partitions its own batch of graphs (weak scaling, no collective on the
    data path): the instance generator's seed per rank."""
    return seed + 1000 * rank


def max_over_ranks(dist, values: list[float]) -> list[float]:
    """Element-wise maximum of per-rank timings (the job's time is its slowest rank's); identity without a
    process group.  The tensor lives where the backend wants it (GPU for NCCL, host for gloo)."""
    if not dist:
        return list(values)
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def describe(w: dict) -> str:
    if w["kind"] == "batch":
        return (f"{w['n']} graphs, V log-uniform in [{w['vmin']}, {w['vmax']}], half 2-D/3-D k-NN (k_nn 8-14), "
                f"half preferential attachment (m 4-8), k uniform in 2..64, seed {w['seed']}, phase-1 theta "
                f"{w['theta']}, phase 2 with the reference's stopping rules")
    if w["kind"] == "rmat":
        return (f"R-MAT scale {w['scale']} edge factor {w['edge_factor']} ({w['a']},{w['b']},{w['c']}) seed "
                f"{w['seed']}, symmetrised, k={w['k']}, theta={w['theta']}, {w['iters']} LP iterations")
    return f"3-D kNN n={w['n']} knn={w['knn']} seed {w['seed']}, k={w['k']}, {w['iters']} LP iterations"


def make_graph(w: dict):
    from dmolp_b200 import graphs

    if w["kind"] == "ingest":
        return make_graph(w["graph"])
    if w["kind"] == "rmat":
        return graphs.rmat(w["scale"], w["edge_factor"], w["a"], w["b"], w["c"], seed=w["seed"])
    return graphs.knn(w["n"], w["dim"], w["knn"], w["seed"])


def measured_peaks() -> tuple[float, str]:
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200", "-i",
                 str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


def golden_parity(w: dict, labels1: np.ndarray, labels: np.ndarray, result) -> dict | None:
    """The timed run against the reference's own outputs for this workload (tests/golden/rmat22_full.json,
    written by tests/golden/make_golden_full.py from the reference's phase-2 steps): phase-1 labels, final
    labels, edge cut and traversed edges.  None when no fixture covers the workload."""
    from dmolp_b200 import graphs

    if not (w["kind"] == "rmat" and w["scale"] == 22 and w["edge_factor"] == 16 and w["seed"] == 7):
        return None
    try:
        gold = json.load(open(os.path.join(ROOT, "tests", "golden", "rmat22_full.json")))[f"k{w['k']}"]
    except (OSError, KeyError):
        return None
    if gold["iters"] != w["iters"] or gold["theta"] != w["theta"]:
        return None
    checks = {"phase1_labels": "%016x" % graphs.fnv1a(labels1) == gold["labels1_hash"],
              "labels": "%016x" % graphs.fnv1a(labels) == gold["labels2_hash"],
              "edge_cut": int(result.edge_cut) == int(gold["result"]["edge_cut"]),
              "traversed_edges": int(result.traversed_edges) == int(gold["result"]["te_total"])}
    return {"ok": all(checks.values()), "checks": checks,
            "against": f"reference phase-2 run, tests/golden/rmat22_full.json k{w['k']}"}


def traffic_from_profiles(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/ncu_traffic.json)."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
        return d.get(workload, {}).get(kernel)
    except Exception:
        return None


# ------------------------------------------------------------------------------------------- our arm
def run_ours(args, w, rank: int, world: int, local_rank: int, dist) -> dict | None:
    import torch

    from dmolp_b200.partitioner import Partitioner

    torch.cuda.set_device(local_rank)
    g = make_graph(w)
    p = Partitioner(local_rank)
    p.upload(g)
    m1 = p.phase1(w["k"], w["theta"])
    labels1 = p.labels()
    p.lib.dmolp_labels_save(p.ctx)
    stream = torch.cuda.ExternalStream(p.lib.dmolp_stream(p.ctx), device=torch.device("cuda", local_rank))

    def step():
        p._check(p.lib.dmolp_labels_restore(p.ctx))
        return p.phase2(w["k"], mode="fixed", iterations=w["iters"], records=False)

    sampler = ClockSampler(local_rank)
    if not args.quick:
        sampler.start()
        t_end = time.time() + 1.0  # keep the GPU busy ~1 s before warm-up so the clock samples see load
        while time.time() < t_end:
            step()
    for _ in range(max(1, args.warmup)):
        step()
    launches0 = p.kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    te = 0
    last = None
    for _ in range(args.steps):
        last = step()
        te += last.traversed_edges
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = p.kernel_launches() - launches0
    elapsed = e0.elapsed_time(e1) / 1e3
    final_labels = p.labels()
    # Per-kernel device times for the roofline: the same K steps again, with CUDA events recorded around the
    # profiled kernels inside the captured graphs (a graph of their own, captured in one untimed step).  The
    # events lengthen a run by ~1 ms, so the headline steps above run without them.
    p.lib.dmolp_set_profiling(p.ctx, 1)
    step()
    p.lib.dmolp_set_profiling(p.ctx, 1)  # reset the accumulated kernel times
    pe0 = torch.cuda.Event(enable_timing=True)
    pe1 = torch.cuda.Event(enable_timing=True)
    pe0.record(stream)
    for _ in range(args.steps):
        step()
    pe1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if not args.quick else None
    prof_elapsed = pe0.elapsed_time(pe1) / 1e3
    prof = {}
    for kid, name in ((0, "boundary_test"), (1, "lp_decide"), (2, "window_mark"), (3, "cut_update"),
                      (4, "window_select")):
        import ctypes

        ms, n, by = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
        p.lib.dmolp_kernel_profile(p.ctx, kid, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(by))
        prof[name] = dict(ms=ms.value, launches=n.value, bytes=by.value)
    p.lib.dmolp_set_profiling(p.ctx, 0)
    parity = golden_parity(w, labels1, final_labels, last)

    rec_step = None
    if args.records:
        p._check(p.lib.dmolp_labels_restore(p.ctx))
        rec_step = p.phase2(w["k"], mode="fixed", iterations=w["iters"], records=True)
    if rec_step is not None:
        for r in rec_step.records:
            print(json.dumps({f: getattr(r, f) for f, _ in r._fields_}), file=sys.stderr)
        p._check(p.lib.dmolp_labels_restore(p.ctx))
        p.phase2(w["k"], mode="fixed", iterations=w["iters"], records=False)
    if args.quick:
        p.close()
        return {"metric": "LP traversed edges/s", "value": te / elapsed, "unit": "TE/s", "ms_per_step":
                elapsed / args.steps * 1e3, "quick": True, "kernels": prof, "gpu_launches": int(launches),
                "parity": parity,
                "phase1": {"gpu_ms": m1.gpu_ms, "stage_ms": m1.stage_ms, "rounds": m1.rounds}}
    # ---- end to end through the public API, host buffers in pinned memory ----
    off_h = torch.from_numpy(g.offsets).pin_memory()
    col_h = torch.from_numpy(g.indices).pin_memory()
    raw_h = torch.from_numpy(g.raw_deg()).pin_memory()
    lab_h = torch.from_numpy(labels1).pin_memory()
    out_h = torch.empty_like(lab_h).pin_memory()
    import ctypes

    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q0 = torch.cuda.Event(enable_timing=True)
    q1 = torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    e2e_te = 0
    for _ in range(e2e_steps):
        p._check(p.lib.dmolp_graph_upload(p.ctx, g.num_vertices, g.num_arcs, ctypes.c_void_p(off_h.data_ptr()),
                                          ctypes.c_void_p(col_h.data_ptr()), ctypes.c_void_p(raw_h.data_ptr())))
        p._check(p.lib.dmolp_labels_set(p.ctx, ctypes.c_void_p(lab_h.data_ptr())))
        r = p.phase2(w["k"], mode="fixed", iterations=w["iters"], records=False)
        e2e_te += r.traversed_edges
        p._check(p.lib.dmolp_labels_get(p.ctx, ctypes.c_void_p(out_h.data_ptr())))
    q1.record(stream)
    torch.cuda.synchronize()
    e2e_wall = time.perf_counter() - t0
    e2e_elapsed = q0.elapsed_time(q1) / 1e3
    assert np.array_equal(out_h.numpy(), final_labels), "end-to-end labels differ from the resident run"
    h2d = g.offsets.nbytes + g.indices.nbytes + g.raw_deg().nbytes + labels1.nbytes
    d2h = labels1.nbytes
    # where an end-to-end step's time goes (one more step, untimed above; each call returns synchronised)
    parts = {}
    t = time.perf_counter()
    p._check(p.lib.dmolp_graph_upload(p.ctx, g.num_vertices, g.num_arcs, ctypes.c_void_p(off_h.data_ptr()),
                                      ctypes.c_void_p(col_h.data_ptr()), ctypes.c_void_p(raw_h.data_ptr())))
    parts["upload_ms"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    p._check(p.lib.dmolp_labels_set(p.ctx, ctypes.c_void_p(lab_h.data_ptr())))
    torch.cuda.synchronize()
    parts["labels_set_ms"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    p.symmetric()
    parts["symmetry_test_ms"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    p.phase2(w["k"], mode="fixed", iterations=w["iters"], records=False)
    parts["phase2_first_run_ms"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    p._check(p.lib.dmolp_labels_get(p.ctx, ctypes.c_void_p(out_h.data_ptr())))
    parts["labels_get_ms"] = (time.perf_counter() - t) * 1e3

    t_max, e2e_max = max_over_ranks(dist, [elapsed, e2e_elapsed])
    p.close()
    if rank != 0:
        return None

    peak, peak_kind = measured_peaks()
    dom = max(prof, key=lambda k: prof[k]["ms"])
    d = prof[dom]
    per_launch_bytes = d["bytes"] / max(1, d["launches"])
    per_launch_s = d["ms"] / 1e3 / max(1, d["launches"])
    achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else None
    line = {
        "metric": "LP traversed edges/s",
        "value": te * world / t_max,
        "unit": "TE/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded generator)",
        "config": {"workload": describe(w), "k": w["k"], "iterations": w["iters"], "mode": "fixed",
                   "label_cap": "reference (min(k,32))", "num_vertices": g.num_vertices, "num_arcs": g.num_arcs,
                   "te_per_step": te // args.steps, "edge_cut": last.edge_cut,
                   "vertex_balance": last.vertex_balance, "edge_balance": last.edge_balance,
                   "phase1_gpu_ms": m1.gpu_ms, "phase1_stage_ms": m1.stage_ms, "phase1_rounds": m1.rounds,
                   "phase1_initial_edge_cut": m1.initial_edge_cut,
                   "l2": "inputs larger than L2 (CSR arcs %.0f MB)" % (g.indices.nbytes / 1e6),
                   "parallelism": f"replicas x{world}",
                   "parity": None if parity is None else parity["ok"], "parity_detail": parity},
        "e2e": {"value": e2e_te * world / e2e_max, "unit": "TE/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "wall_s": e2e_wall, "steps": e2e_steps, "parts": parts},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                     "traffic": traffic_from_profiles(dom, args.workload),
                     "algorithmic_bytes_per_launch": per_launch_bytes, "avg_launch_ms": per_launch_s * 1e3,
                     "timing": "CUDA events around each launch, in K further steps of the same workload "
                               "(%.3f ms per step with the events)" % (prof_elapsed / args.steps * 1e3),
                     "kernels": prof},
        "clocks": clocks,
    }
    return line


# ------------------------------------------------------------------------------------------- ingestion
def reference_load(path: str, timeout: float = 600) -> dict:
    """The reference's own load_graph (oracle/_ref, built from its sources) on the file: seconds."""
    import oracle

    with tempfile.TemporaryDirectory() as td:
        pr = subprocess.run([oracle.REF_HARNESS, path, "1", "1", "--out", td, "--load-only", "--threads", "1"],
                            capture_output=True, text=True, timeout=timeout)
        if pr.returncode != 0:
            raise RuntimeError(pr.stderr[-500:])
        return json.loads(pr.stdout.strip().splitlines()[-1])


def ingest_text_file(g, td: str) -> str:
    from dmolp_b200 import graphs

    path = os.path.join(td, "graph.txt")
    graphs.write_adjtext(g, path)
    return path


def run_ingest(args, w, rank: int, world: int, local_rank: int, dist) -> dict | None:
    """Adjacency text -> resident CSR: the reference's load_graph + CSR build (src/phase1/init.cpp:25-100,
    src/phase1/partition.cpp:227-262) as the device parse.  A step parses the whole text once: `value` with the
    text already in HBM (dmolp_graph_upload_adjtext_device), `e2e` from the file (page cache) through
    dmolp_graph_load_adjtext, file read and host-to-device copy included."""
    import torch

    from dmolp_b200.partitioner import Partitioner, load_adjtext

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    g = make_graph(w)
    td = tempfile.mkdtemp(prefix="dmolp_ingest_")
    try:
        path = ingest_text_file(g, td)
        host = np.fromfile(path, np.uint8)
        nbytes = int(host.size)
        text = torch.from_numpy(host).to(dev)
        p = Partitioner(local_rank)
        stream = torch.cuda.ExternalStream(p.lib.dmolp_stream(p.ctx), device=dev)
        p.upload_adjtext(text)
        h = p.graph_arrays()  # parity at full size: the generator's CSR, raw degree = CSR degree
        parity = bool(np.array_equal(h.offsets, g.offsets) and np.array_equal(h.indices, g.indices)
                      and np.array_equal(h.raw_degree, g.degree()))
        del h
        sampler = ClockSampler(local_rank)
        if not args.quick:
            sampler.start()
            t_end = time.time() + 1.5  # keep the GPU busy before warm-up so the clock samples see load
            while time.time() < t_end:
                p.upload_adjtext(text)
        for _ in range(max(1, args.warmup)):
            p.upload_adjtext(text)
        launches0 = p.kernel_launches()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        infos = [p.upload_adjtext(text) for _ in range(args.steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        elapsed = e0.elapsed_time(e1) / 1e3
        launches = p.kernel_launches() - launches0
        clocks = sampler.stop() if not args.quick else None
        # end to end from the file: read through the pinned ring, copy, parse, resident state
        e2e_n = 0 if args.quick else max(1, min(args.steps, 5))
        if e2e_n:
            p.upload_adjtext(path)  # warm-up: pinned staging ring, page cache
        t0 = time.perf_counter()
        e2e_infos = [p.upload_adjtext(path) for _ in range(e2e_n)]
        e2e_s = time.perf_counter() - t0
        t_max, e2e_max = max_over_ranks(dist, [elapsed, e2e_s])
        host_loader = None
        ref = None
        if rank == 0 and world == 1 and not args.quick and not args.no_cpu_baseline:
            t0 = time.perf_counter()
            hg = load_adjtext(path)
            host_loader = {"seconds": time.perf_counter() - t0, "cores": os.cpu_count() or 1,
                           "identical_csr": bool(np.array_equal(hg.offsets, g.offsets)
                                                 and np.array_equal(hg.indices, g.indices)),
                           "kind": "this package's host loader (OpenMP, adjtext.cpp)"}
            del hg
            import oracle

            if oracle.reference_available():
                try:
                    ref = reference_load(path)
                except Exception as e:  # report, do not hide
                    ref = {"error": str(e)[:300]}
        p.close()
    finally:
        for f in os.listdir(td):
            os.remove(os.path.join(td, f))
        os.rmdir(td)
    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    i0 = infos[0]
    ntok, nv = int(i0["num_tokens"]), int(i0["num_vertices"])
    count_ms = statistics.mean(i["count_ms"] for i in infos)
    emit_ms = statistics.mean(i["emit_ms"] for i in infos)
    body = nbytes  # header and trailing newline are a few bytes
    kern = {"k_txt_count": {"ms": count_ms, "bytes": body}, "k_txt_emit": {"ms": emit_ms, "bytes": body + 4 * ntok + 8 * nv}}
    dom = max(kern, key=lambda k: kern[k]["ms"])
    achieved = kern[dom]["bytes"] / (kern[dom]["ms"] / 1e3) / 1e9
    line = {
        "metric": "adjacency text parsed into the resident CSR, bytes/s",
        "value": nbytes * args.steps * world / t_max / 1e9,
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic (seeded generator, written as the reference's adjacency text)",
        "config": {"workload": "R-MAT scale 22, edge factor 16, seed 7, as adjacency text (%.2f GB)" % (nbytes / 1e9),
                   "text_bytes": nbytes, "num_vertices": nv, "num_tokens": ntok, "num_arcs": int(i0["num_arcs"]),
                   "arcs_per_s": int(i0["num_arcs"]) * args.steps * world / t_max,
                   "parity_full_size": parity, "parse_ms_per_step": statistics.mean(i["parse_ms"] for i in infos),
                   "l2": "inputs larger than L2 (text %.0f MB)" % (nbytes / 1e6), "parallelism": f"replicas x{world}"},
        "e2e": ({"value": nbytes * e2e_n * world / e2e_max / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                 "d2h_bytes_per_step": 4 * nv, "steps": e2e_n,
                 "read_ms_per_step": statistics.mean(i["read_ms"] for i in e2e_infos),
                 "parse_ms_per_step": statistics.mean(i["parse_ms"] for i in e2e_infos),
                 "seconds_per_step": e2e_max / e2e_n,
                 "path": "dmolp_graph_load_adjtext: file (page cache) -> pinned ring -> HBM -> parse -> resident graph"}
                if e2e_n else None),
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_source": peak_kind,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic_from_profiles(dom, args.workload),
                     "algorithmic_bytes_per_launch": kern[dom]["bytes"], "avg_launch_ms": kern[dom]["ms"],
                     "kernels": kern},
        "clocks": clocks,
    }
    if ref is not None:
        if "load_seconds" in ref:
            line["cpu_baseline"] = {"value": nbytes / ref["load_seconds"] / 1e9, "unit": "GB/s", "cores": 1,
                                    "kind": "reference", "seconds": ref["load_seconds"],
                                    "sample": "the whole text through the reference's load_graph (file -> adjacency "
                                              "map; its CSR build inside phase 1 not included)"}
        else:
            line["cpu_baseline"] = ref
    if host_loader is not None:
        host_loader["value"] = nbytes / host_loader["seconds"] / 1e9
        host_loader["unit"] = "GB/s"
        line["host_loader"] = host_loader
    return line


# ------------------------------------------------------------------------------------------- batched
def run_batch(args, w, rank: int, world: int, local_rank: int, dist) -> dict | None:
    """Graphs per second of phase 2 over a batch of independent graphs: the batched persistent launch
    against the single-graph path run on one instance after another (the plain method), from the same
    phase-1 partitions; every instance must end with identical labels either way."""
    import torch

    from dmolp_b200.batch import Batch, random_instances, union
    from dmolp_b200.partitioner import Partitioner

    torch.cuda.set_device(local_rank)
    n = w["n"]
    t0 = time.perf_counter()
    inst = random_instances(n, seed=rank_seed(w["seed"], rank), vmin=w["vmin"], vmax=w["vmax"])
    gen_s = time.perf_counter() - t0
    arrays = union(inst)
    nv_tot, na_tot = int(arrays[0][-1]), int(arrays[1][-1])

    # ---- phase 1 (single-graph path) for every instance: the starting partitions ----
    p = Partitioner(local_rank)
    lab1, p1_ms, p1_each = [], 0.0, []
    t0 = time.perf_counter()
    for it in inst:
        t1 = time.perf_counter()
        p.upload(it.graph)
        m1 = p.phase1(it.k, w["theta"])
        p1_ms += m1.gpu_ms
        lab1.append(p.labels())
        p1_each.append(time.perf_counter() - t1)
    p1_wall = time.perf_counter() - t0

    # ---- plain: phase 2 of the single-graph path, one instance after another ----
    ns = n if args.plain_sample <= 0 else min(n, args.plain_sample)
    plain_ms, plain_wall, plain_labels, plain_cut = 0.0, 0.0, [], 0
    for it, l1 in zip(inst[:ns], lab1[:ns]):
        p.upload(it.graph)
        p.set_labels(l1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m2 = p.phase2(it.k, mode="ref", records=False)
        plain_labels.append(p.labels())
        plain_wall += time.perf_counter() - t0
        plain_ms += m2.gpu_ms
        plain_cut += m2.edge_cut
    p.close()

    # ---- batched ----
    b = Batch(local_rank)
    b.upload(arrays=arrays)
    b.set_labels(lab1)
    t0 = time.perf_counter()
    tune = b.autotune("ref", 0, "ref")
    tune_s = time.perf_counter() - t0
    b.save_labels()
    for _ in range(max(1, args.warmup)):
        b.restore_labels()
        b.run("ref", results=False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
        b.restore_labels()
        ms.append(b.run("ref", results=False)[1])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    b.restore_labels()
    res, one_ms = b.run("ref", results=True)
    final = b.split(b.labels())
    identical = all(np.array_equal(final[i], plain_labels[i]) for i in range(ns))
    batch_cut = sum(r["edge_cut"] for r in res[:ns])
    elapsed = sum(ms) / 1e3
    by = sum(8.0 * r["arcs_read"] + 20.0 * r["vertex_visits"] for r in res)

    # ---- end to end: host arrays in, labels and results out ----
    pinned = [torch.from_numpy(a).pin_memory().numpy() for a in arrays]
    lab_h = torch.from_numpy(np.concatenate(lab1)).pin_memory().numpy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.upload(arrays=pinned)
    b.tuning = {k: tune[k] for k in ("block_threads", "thread_row_max", "blocks_per_sm", "reserved")}
    b.set_labels(lab_h)
    res2, _ = b.run("ref", results=True)
    out = b.labels()
    e2e_s = time.perf_counter() - t0
    assert np.array_equal(out, np.concatenate(final)), "end-to-end labels differ"
    b.close()

    # ---- whole pipelines, phase 1 + phase 2 for every graph, wall clock including host work:
    #      plain one graph after another (the single-graph path), plain batched (batched phase 1 + batched
    #      phase 2), batched + learned (the proposal for every graph -- features, network, decoder, gate --
    #      batched phase 1 for the graphs the gate declines, batched phase 2) ----
    pipelines = None
    try:
        from dmolp_b200.learned import WEIGHTS, Proposal

        plain_total_s = p1_wall + plain_wall * n / max(1, ns)
        all_plain_cut = float(sum(r["edge_cut"] for r in res))
        b2 = Batch(local_rank)
        b2.upload(arrays=arrays)
        b2.tuning = {k: tune[k] for k in ("block_threads", "thread_row_max", "blocks_per_sm", "reserved")}
        b2.phase1(w["theta"])  # hub lists are computed once per upload on the host: not part of a run
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b2.phase1(w["theta"])
        res_p, lms_p = b2.run("ref")
        batched_plain_s = time.perf_counter() - t0
        lab_p = b2.split(b2.labels())
        same_as_plain = all(np.array_equal(lab_p[i], final[i]) for i in range(n))
        model = Proposal(local_rank, WEIGHTS)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = model.propose(b2)
        prop_s = time.perf_counter() - t0
        if st.any():
            b2.phase1(w["theta"], only=st != 0)
        res_l, lms = b2.run("ref")
        learned_s = time.perf_counter() - t0
        b2.close()
        model.close()
        pipelines = {
            "plain_one_graph_after_another": {"graphs_per_s": n / plain_total_s, "wall_s": plain_total_s},
            "plain_batched": {"graphs_per_s": n / batched_plain_s, "wall_s": batched_plain_s,
                              "identical_labels_to_one_by_one": same_as_plain},
            "batched_learned": {"graphs_per_s": n / learned_s, "wall_s": learned_s, "proposal_wall_s": prop_s,
                                "fallbacks": int((st != 0).sum()),
                                "cut_ratio_vs_plain": float(sum(r["edge_cut"] for r in res_l)) / max(1.0, all_plain_cut),
                                "vertex_balance_mean": float(np.mean([r["vertex_balance"] for r in res_l]))},
            "plain_vertex_balance_mean": float(np.mean([r["vertex_balance"] for r in res])),
            "speedup_batched_learned_vs_plain": plain_total_s / learned_s,
            "speedup_plain_batched_vs_plain": plain_total_s / batched_plain_s}
    except Exception as e:  # report, do not hide
        pipelines = {"error": str(e)[:300]}

    (t_max,) = max_over_ranks(dist, [elapsed])
    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    per_launch_s = elapsed / max(1, len(ms))
    achieved = by / per_launch_s / 1e9
    plain_gps = ns / (plain_ms / 1e3)
    value = n * args.steps * world / t_max
    return {
        "metric": "phase-2 graphs/s (batched)", "value": value, "unit": "graphs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generators)",
        "config": {"workload": describe(w), "instances": n, "num_vertices": nv_tot, "num_arcs": na_tot,
                   "mode": "ref", "label_cap": "reference (min(k,32))", "tuning": tune,
                   "autotune_s": tune_s, "generate_s": gen_s,
                   "plain": {"instances_timed": ns, "graphs_per_s_device": plain_gps,
                             "graphs_per_s_wall": ns / plain_wall, "lp_ms_device": plain_ms},
                   "speedup_vs_plain_device": value / world / plain_gps,
                   "identical_labels_to_plain": identical, "edge_cut_sum_batched": batch_cut,
                   "edge_cut_sum_plain": plain_cut,
                   "phase1_single_graph_ms_device": p1_ms, "phase1_single_graph_wall_s": p1_wall,
                   "iterations_mean": float(np.mean([r["iterations_run"] for r in res])),
                   "pipelines": pipelines,
                   "l2": "batch CSR %.0f MB > L2" % (na_tot * 4 / 1e6), "parallelism": f"replicas x{world}"},
        "e2e": {"value": n * world / e2e_s, "unit": "graphs/s", "wall_s": e2e_s,
                "h2d_bytes_per_step": int(sum(a.nbytes for a in arrays) + lab_h.nbytes),
                "d2h_bytes_per_step": int(lab_h.nbytes)},
        "gpu_launches": 2 * args.steps,
        "roofline": {"bound": "hbm", "kernel": "k_batch_lp", "achieved": achieved, "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic_from_profiles("k_batch_lp", args.workload),
                     "algorithmic_bytes_per_launch": by, "avg_launch_ms": per_launch_s * 1e3},
    }


LEARNED_EVAL = [  # held-out graphs of the learned proposal's evaluation: R-MAT scale 24, 3-D geometric 2 M, k = 32
    dict(name="rmat24", kind="rmat", scale=24, edge_factor=16, seed=9, k=32, theta=10000),
    dict(name="knn3d-2M", kind="knn", n=2_000_000, dim=3, knn=12, seed=41, k=32, theta=10000),
]


def learned_eval_summary(device: int) -> dict:
    """The learned proposal on large held-out graphs against the plain method: edge cut, vertex / edge balance
    and iterations to converge of phase 2 (reference stopping rules) from each start, the gate's decision, and
    the proposal with the gate ignored."""
    from dmolp_b200 import graphs
    from dmolp_b200.learned import WEIGHTS, Proposal, evaluate_large

    model = Proposal(device, WEIGHTS)
    out = {}
    try:
        for spec in LEARNED_EVAL:
            t0 = time.perf_counter()
            if spec["kind"] == "rmat":
                g = graphs.rmat(spec["scale"], spec["edge_factor"], seed=spec["seed"])
            else:
                g = graphs.knn(spec["n"], spec["dim"], spec["knn"], seed=spec["seed"])
            gen_s = time.perf_counter() - t0
            r = evaluate_large(model, g, spec["k"], spec["theta"], device)
            r["generate_s"] = gen_s
            pl = r["plain"]
            for key in ("learned", "proposal_gate_ignored"):
                if key in r:
                    r[key]["cut_ratio_vs_plain"] = r[key]["edge_cut"] / max(1, pl["edge_cut"])
            out[spec["name"]] = r
            del g
    finally:
        model.close()
    return out


def batched_summary(n: int, theta: int, device: int) -> dict:
    """A compact view of the batched forms for the default bench line: n graphs of the batched mix, whole
    pipeline (phase 1 + phase 2 with the reference's stopping rules) one graph after another on the
    single-graph path, batched, and batched + learned (the proposal where its gate accepts it, batched
    phase 1 elsewhere); wall clock, edge cut against the one-by-one run."""
    import torch

    from dmolp_b200.batch import Batch, random_instances
    from dmolp_b200.learned import WEIGHTS, Proposal
    from dmolp_b200.partitioner import Partitioner

    inst = random_instances(n, seed=11, vmin=1000, vmax=200_000)
    p = Partitioner(device)
    cuts = []
    t0 = time.perf_counter()
    for it in inst:
        p.upload(it.graph)
        p.phase1(it.k, theta)
        cuts.append(p.phase2(it.k, mode="ref", records=False).edge_cut)
    one_s = time.perf_counter() - t0
    p.close()
    b = Batch(device)
    b.upload(inst)
    b.phase1(theta)  # the host-side hub lists are built once per upload
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.phase1(theta)
    res, _ = b.run("ref")
    bat_s = time.perf_counter() - t0
    same = [r["edge_cut"] for r in res] == cuts
    m = Proposal(device, WEIGHTS)
    m.propose(b)  # workspace allocation, once per batch size
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = m.propose(b)
    if st.any():
        b.phase1(theta, only=st != 0)
    res_l, _ = b.run("ref")
    lrn_s = time.perf_counter() - t0
    m.close()
    b.close()
    tot = float(sum(cuts))
    return {"graphs": n, "workload": "batched mix (V log-uniform in [1000, 200000], half k-NN, half preferential "
                                     "attachment, k in 2..64), phase 1 theta %d + phase 2 reference rules" % theta,
            "plain_one_by_one_graphs_per_s": n / one_s, "plain_batched_graphs_per_s": n / bat_s,
            "plain_batched_identical_cuts": same, "batched_learned_graphs_per_s": n / lrn_s,
            "batched_learned_cut_ratio": float(sum(r["edge_cut"] for r in res_l)) / max(1.0, tot),
            "batched_learned_fallbacks": int((st != 0).sum()),
            "speedup_batched_learned_vs_plain": one_s / lrn_s}


# ------------------------------------------------------------------------------------------- CPU baselines
def reference_iterations(g, labels1, w, iters: int, threads: int, gpu: bool = False, timeout: float = 3600) -> list:
    """The reference's own phase-2 code (oracle/_ref/ref_harness, built from its sources) on the host cores:
    one fixed-mode run of `iters` LP iterations from the phase-1 labels, continuing from iteration to
    iteration as the workload does.  Returns per iteration (seconds, traversed edges): the harness times the
    reference's steps only (penalties, window expansion, the LP step and its changes, statistics, cut), not
    its own traversed-edge count.  gpu=True: the reference's own CUDA path (boundaryLPKernel_unified, built
    unmodified for sm_100a) instead of the CPU restatement of its kernel."""
    import oracle

    with tempfile.TemporaryDirectory() as td:
        from dmolp_b200 import graphs

        txt = os.path.join(td, "g.txt")
        graphs.write_adjtext(g, txt)
        lab = os.path.join(td, "labels1.bin")
        labels1.astype(np.int32).tofile(lab)
        out = os.path.join(td, "o")
        cmd = [oracle.REF_HARNESS, txt, str(w["k"]), str(w["theta"]), "--out", out, "--mode", "fixed", "--iters",
               str(iters), "--threads", str(threads), "--labels-in", lab, "--no-seed-dump"] + (["--gpu"] if gpu else [])
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        pr = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
        if pr.returncode != 0:
            raise RuntimeError(pr.stderr[-1000:])
        trace = [json.loads(l) for l in open(os.path.join(out, "trace.jsonl")) if l.strip()]
    its, prev = [], 0.0
    for t in trace:
        its.append((t["seconds"] - prev, sum(t["te"])))
        prev = t["seconds"]
    return its


def iteration_steps(g, labels1, w, n: int, threads: int, gpu: bool = False) -> list:
    """n consecutive LP iterations of the workload (a new run from the phase-1 labels after every
    w["iters"] iterations), as (seconds, traversed edges) per iteration."""
    its = []
    while len(its) < n:
        its += reference_iterations(g, labels1, w, min(w["iters"], n - len(its)), threads, gpu)
    return its


def port_cpu_run(g, labels1, w, iters: int):
    import oracle

    t0 = time.perf_counter()
    o = oracle.phase2(g.offsets, g.indices, labels1, w["k"], "fixed", iters)
    return dict(lp_seconds=time.perf_counter() - t0, te_total=o.res.te_total)


def cpu_baseline(g, labels1, w, args) -> dict:
    import oracle

    threads = os.cpu_count() or 1
    iters = args.cpu_sample_iters
    sample = f"LP iterations 1..{iters} of {w['iters']} on the full graph (one run from the phase-1 labels)"
    if oracle.reference_available():
        its = iteration_steps(g, labels1, w, iters, threads)
        secs, te = sum(x for x, _ in its), sum(y for _, y in its)
        out = {"value": te / secs, "unit": "TE/s", "cores": threads, "kind": "reference", "sample": sample,
               "seconds": secs, "note": "the reference's early iterations are its slowest per traversed edge; "
                                        "--impl reference times iterations later in the run as well"}
        try:  # the reference's own GPU path on the same B200, same sample
            gi = iteration_steps(g, labels1, w, iters, threads, gpu=True)
            gs, gt = sum(x for x, _ in gi), sum(y for _, y in gi)
            out["reference_gpu"] = {"value": gt / gs, "unit": "TE/s", "sample": sample, "seconds": gs,
                                    "kind": "reference run_phase2 steps with its boundaryLPKernel_unified (sm_100a)"}
        except Exception as e:  # report, do not hide
            out["reference_gpu"] = {"error": str(e)[:300]}
        return out
    r = port_cpu_run(g, labels1, w, iters)
    return {"value": r["te_total"] / r["lp_seconds"], "unit": "TE/s", "cores": 1, "kind": "port",
            "sample": sample, "seconds": r["lp_seconds"]}


def ingest_summary(g, device: int) -> dict:
    """A compact view of graph ingestion for the default bench line: the same graph as the reference's
    adjacency text, parsed on the device from HBM and from the file, next to the reference's load_graph."""
    import torch

    import oracle
    from dmolp_b200.partitioner import Partitioner

    dev = torch.device("cuda", device)
    td = tempfile.mkdtemp(prefix="dmolp_ingest_sum_")
    try:
        path = ingest_text_file(g, td)
        host = np.fromfile(path, np.uint8)
        nbytes = int(host.size)
        text = torch.from_numpy(host).to(dev)
        del host
        p = Partitioner(device)
        p.upload_adjtext(text)
        h = p.graph_arrays()
        same = bool(np.array_equal(h.offsets, g.offsets) and np.array_equal(h.indices, g.indices))
        del h
        dev_ms = [p.upload_adjtext(text)["total_ms"] for _ in range(5)]
        file_ms = [p.upload_adjtext(path)["total_ms"] for _ in range(3)]
        p.close()
        del text
        out = {"text_bytes": nbytes, "identical_csr": same,
               "device_text_gb_per_s": nbytes / (min(dev_ms) / 1e3) / 1e9,
               "file_to_resident_graph_ms": min(file_ms),
               "file_to_resident_graph_gb_per_s": nbytes / (min(file_ms) / 1e3) / 1e9}
        if oracle.reference_available():
            try:
                r = reference_load(path)
                out["reference_load_graph_s"] = r["load_seconds"]
                out["speedup_file_vs_reference_load_graph"] = r["load_seconds"] / (min(file_ms) / 1e3)
            except Exception as e:  # report, do not hide
                out["reference_load_graph"] = {"error": str(e)[:200]}
        return out
    finally:
        for f in os.listdir(td):
            os.remove(os.path.join(td, f))
        os.rmdir(td)


def run_reference_ingest(args, w) -> dict:
    """--impl reference for the ingestion workload: the reference's load_graph on the same text, one whole
    load per step, single-threaded as the reference reads."""
    import oracle

    g = make_graph(w)
    td = tempfile.mkdtemp(prefix="dmolp_ingest_ref_")
    try:
        path = ingest_text_file(g, td)
        nbytes = os.path.getsize(path)
        if oracle.reference_available():
            runs = [reference_load(path)["load_seconds"] for _ in range(args.warmup + args.steps)]
            kind = "reference"
        else:
            from dmolp_b200.partitioner import load_adjtext

            runs = []
            for _ in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                load_adjtext(path)
                runs.append(time.perf_counter() - t0)
            kind = "port"
    finally:
        for f in os.listdir(td):
            os.remove(os.path.join(td, f))
        os.rmdir(td)
    secs = sum(runs[args.warmup:]) or sum(runs)
    n = len(runs[args.warmup:]) or len(runs)
    value = nbytes * n / secs / 1e9
    return {
        "impl": "reference", "metric": "adjacency text parsed into the resident CSR, bytes/s", "value": value,
        "unit": "GB/s", "n_gpus": args.gpus, "steps": n, "warmup": args.warmup, "ms_per_step": secs / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator, written as the reference's adjacency text)",
        "config": {"workload": "R-MAT scale 22, edge factor 16, seed 7, as adjacency text (%.2f GB)" % (nbytes / 1e9),
                   "text_bytes": nbytes},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": 1, "kind": kind,
                         "sample": "per step: the whole text through load_graph (file -> adjacency map)"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference_arm(args, w) -> dict:
    """--impl reference: the reference's own implementation of the path on this box's host cores.  A step is
    one LP iteration of the workload's run, taken in order from one continuous run (from the phase-1
    labels; a new run after every w["iters"] iterations): the first W iterations are the warm-up, the next K
    are timed.  Per traversed edge the reference's first iterations are its slowest, so this sample sits at
    or above the rate of a whole run (the line reports that rate too when the steps cover one)."""
    import oracle

    if w["kind"] == "ingest":
        return run_reference_ingest(args, w)
    if w["kind"] == "batch":
        return {"impl": "reference", "unavailable": "the reference has no batched path; its per-graph CPU phase 2 "
                                                    "is the rmat22/knn-c0 reference arm"}
    if w["kind"] == "learned":
        return {"impl": "reference", "unavailable": "the reference has no learned proposal"}
    g = make_graph(w)
    # phase-1 labels from the oracle (the reference's phase 1 is undefined on R-MAT: fewer seeds than parts)
    labels1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), w["k"], w["theta"]).labels
    threads = os.cpu_count() or 1
    n = args.warmup + args.steps
    if oracle.reference_available():
        its = iteration_steps(g, labels1, w, n, threads)
        kind, cores = "reference", threads
    else:
        its = []
        for _ in range(n):
            r = port_cpu_run(g, labels1, w, 1)
            its.append((r["lp_seconds"], r["te_total"]))
        kind, cores = "port", 1
    timed = its[args.warmup:] or its
    secs = sum(x for x, _ in timed)
    te = sum(y for _, y in timed)
    value = te / secs
    first = args.warmup + 1
    sample = (f"per step: one LP iteration of the {w['iters']}-iteration run, in order; warm-up iterations 1..{args.warmup}, "
              f"timed iterations {first}..{args.warmup + len(timed)} (counted modulo a new run every {w['iters']})")
    line = {
        "impl": "reference", "metric": "LP traversed edges/s", "value": value, "unit": "TE/s", "n_gpus": args.gpus,
        "steps": len(timed), "warmup": args.warmup, "ms_per_step": secs / len(timed) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator)",
        "config": {"workload": describe(w), "k": w["k"], "iterations": w["iters"], "mode": "fixed",
                   "label_cap": "reference (min(k,32))", "num_vertices": g.num_vertices, "num_arcs": g.num_arcs,
                   "l2": "host run", "parallelism": "host threads x%d" % cores},
        "cpu_baseline": {"value": value, "unit": "TE/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "TE/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations": [{"seconds": x, "traversed_edges": y} for x, y in its],
    }
    if len(its) >= w["iters"]:
        run = its[:w["iters"]]
        line["whole_run"] = {"value": sum(y for _, y in run) / sum(x for x, _ in run), "unit": "TE/s",
                             "seconds": sum(x for x, _ in run), "iterations": w["iters"]}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="rmat22", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample-iters", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="timed steps only: no clock soak, e2e or CPU baseline")
    ap.add_argument("--records", action="store_true", help="print one step's per-iteration records to stderr")
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="batched workload: instances timed on the single-graph path (0 = all)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference_arm(args, w)), flush=True)
        return

    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    if w["kind"] == "learned":
        if rank == 0:
            print(json.dumps({"metric": "learned proposal vs plain (edge cut, balance, iterations)",
                              "learned_eval": learned_eval_summary(local_rank)}), flush=True)
        return
    runner = {"batch": run_batch, "ingest": run_ingest}.get(w["kind"], run_ours)
    line = runner(args, w, rank, world, local_rank, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and line is not None:
        if world == 1 and not args.no_cpu_baseline and not args.quick and w["kind"] not in ("batch", "ingest"):
            g = make_graph(w)
            import oracle

            labels1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), w["k"], w["theta"]).labels
            try:
                line["cpu_baseline"] = cpu_baseline(g, labels1, w, args)
            except Exception as e:  # report, do not hide
                line["cpu_baseline"] = {"error": str(e)[:300]}
        if world == 1 and not args.quick and w["kind"] not in ("batch", "ingest"):
            try:
                line["batched"] = batched_summary(2048, 1000, local_rank)  # the batched config: 2048 graphs
            except Exception as e:  # report, do not hide
                line["batched"] = {"error": str(e)[:300]}
            try:
                line["learned_eval"] = learned_eval_summary(local_rank)
            except Exception as e:  # report, do not hide
                line["learned_eval"] = {"error": str(e)[:300]}
            try:
                line["ingest"] = ingest_summary(make_graph(w), local_rank)
            except Exception as e:  # report, do not hide
                line["ingest"] = {"error": str(e)[:300]}
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
