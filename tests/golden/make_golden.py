"""Regenerate the golden fixtures from the REFERENCE itself.

    python tests/golden/make_golden.py

Each case builds a seeded synthetic graph with dmolp_b200.graphs, writes it in the reference's adjacency
text format, runs the reference's own sources (oracle/_ref/ref_harness, built by `make -C oracle` from the
reference tree) single-threaded, and stores what it produced in cases.json (scalars, hashes, per-iteration
records) and <case>.npz (label arrays).  The tests then hold the oracle and the CUDA path to these values.

Cases where the reference's phase 1 is undefined (fewer seeds than parts: it reads past its seed vector)
are run with --labels-in: phase 2 of the reference starts from the oracle's phase-1 labels, which pins the
LP loop on those graphs.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from dmolp_b200 import graphs  # noqa: E402

# name -> (graph spec, k, theta, [(mode, iters)], labels_from)
CASES = {
    "knn3d_2k": (dict(kind="knn", n=2000, dim=3, k=12, seed=1), 8, 100, [("fixed", 20), ("ref", 0)], "phase1"),
    "knn2d_3k": (dict(kind="knn", n=3000, dim=2, k=8, seed=3), 4, 50, [("fixed", 15), ("ref", 0)], "phase1"),
    "knn3d_c0": (dict(kind="knn", n=55476, dim=3, k=12, seed=1), 8, 1000, [("fixed", 20), ("ref", 0)], "phase1"),
    "knn3d_c0_k32": (dict(kind="knn", n=55476, dim=3, k=12, seed=1), 32, 1000, [("fixed", 20)], "phase1"),
    "rmat12_k16": (dict(kind="rmat", scale=12, edge_factor=16, seed=7), 16, 100, [("fixed", 30), ("ref", 0)],
                   "oracle_phase1"),
    "rmat13_k64": (dict(kind="rmat", scale=13, edge_factor=8, seed=11), 64, 200, [("fixed", 12)], "oracle_phase1"),
    "ba3k_k8": (dict(kind="ba", n=3000, m=4, seed=5), 8, 100, [("fixed", 20), ("ref", 0)], "oracle_phase1"),
    "knn3d_2k_rand64": (dict(kind="knn", n=2000, dim=3, k=12, seed=2), 64, 100, [("fixed", 10)], "random:64:9"),
    "knn3d_2k_rand5": (dict(kind="knn", n=2000, dim=3, k=10, seed=4), 5, 100, [("fixed", 25), ("ref", 0)],
                       "random:5:3"),
    "path12": (dict(kind="edges", n=12, edges=[(i, i + 1) for i in range(11)]), 2, 1, [("fixed", 8), ("ref", 0)],
               "oracle_phase1"),
    "two_cliques": (dict(kind="edges", n=12, edges=[(i, j) for i in range(6) for j in range(i + 1, 6)] +
                         [(i, j) for i in range(6, 12) for j in range(i + 1, 12)] + [(5, 6)]), 2, 2,
                    [("fixed", 8), ("ref", 0)], "oracle_phase1"),
    "isolated_mix": (dict(kind="edges", n=20, edges=[(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (10, 11), (11, 12)]),
                     3, 1, [("fixed", 6), ("ref", 0)], "oracle_phase1"),
}


def build_graph(spec: dict) -> graphs.Graph:
    kind = spec["kind"]
    if kind == "knn":
        return graphs.knn(spec["n"], spec["dim"], spec["k"], spec["seed"])
    if kind == "rmat":
        return graphs.rmat(spec["scale"], spec["edge_factor"], seed=spec["seed"])
    if kind == "ba":
        return graphs.barabasi_albert(spec["n"], spec["m"], spec["seed"])
    if kind == "edges":
        return graphs.from_edges(spec["n"], spec["edges"])
    raise ValueError(kind)


def graph_hash(g: graphs.Graph) -> str:
    return "%016x" % oracle.fnv1a(np.concatenate([g.offsets.view(np.uint8), g.indices.view(np.uint8)]))


def initial_labels(name, g, k, theta, how):
    if how == "phase1":
        return None
    if how == "oracle_phase1":
        return oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, theta).labels
    _, kk, seed = how.split(":")
    rng = np.random.default_rng(int(seed))
    return rng.integers(0, int(kk), size=g.num_vertices).astype(np.int32)


def main() -> None:
    if not oracle.reference_available():
        sys.exit("oracle/_ref/ref_harness is not built (make -C oracle with the reference tree present)")
    out = {}
    only = set(sys.argv[1:])
    old = {}
    path = os.path.join(HERE, "cases.json")
    if only and os.path.exists(path):
        old = json.load(open(path))
    for name, (spec, k, theta, runs, how) in CASES.items():
        if only and name not in only:
            if name in old:
                out[name] = old[name]
            continue
        g = build_graph(spec)
        case = dict(spec={kk: vv for kk, vv in spec.items() if kk != "edges"}, k=k, theta=theta,
                    graph_hash=graph_hash(g), num_vertices=g.num_vertices, num_arcs=g.num_arcs, labels_from=how,
                    runs={})
        arrays = {}
        with tempfile.TemporaryDirectory() as td:
            txt = os.path.join(td, "g.txt")
            graphs.write_adjtext(g, txt)
            lab0 = initial_labels(name, g, k, theta, how)
            lab_path = None
            if lab0 is not None:
                lab_path = os.path.join(td, "labels_in.bin")
                lab0.astype(np.int32).tofile(lab_path)
                arrays["labels_in"] = lab0
            for mode, iters in runs:
                od = os.path.join(td, f"{mode}")
                r = oracle.run_reference(txt, k, theta, od, mode=mode, iters=iters or 20, labels_in=lab_path)
                p1 = r["phase1"]
                case["phase1"] = {kk: vv for kk, vv in p1.items() if kk not in ("hubs", "seconds")}
                if p1.get("hubs") is not None:
                    case["phase1"]["hubs_hash"] = "%016x" % oracle.fnv1a(np.asarray(p1["hubs"], np.int32))
                if "unpinned" in p1 and lab0 is None:
                    # phase 1 undefined in the reference: redo with labels-in so phase 2 is still pinned
                    raise RuntimeError(f"{name}: reference phase 1 unpinned ({p1['unpinned']}); use labels-in")
                if lab0 is None:
                    arrays["labels1"] = r["labels1"]
                res = r["result"]
                case["runs"][mode] = dict(iters=iters, result=res, trace=r["trace"])
                arrays[f"labels2_{mode}"] = r["labels2"]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        out[name] = case
        print(name, "V", g.num_vertices, "arcs", g.num_arcs, {m: case["runs"][m]["result"]["edge_cut"] for m in case["runs"]})
    json.dump(out, open(path, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
