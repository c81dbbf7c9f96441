"""Full-size goldens from the REFERENCE: the benchmarked R-MAT scale-22 graph over all of its LP iterations.

    python tests/golden/make_golden_full.py [k ...]        # default: 32 16 64 (one process per k)

For each k the graph of the rmat22 bench workload (R-MAT scale 22, edge factor 16, (.57, .19, .19), seed 7,
symmetrised, self-loops and duplicates removed, ids permuted: 4,194,304 vertices, 128,308,142 arcs) is written
as the reference's adjacency text.  Phase-1 labels come from the oracle: the reference's phase 1 is undefined
on this graph (the first hub's 2-hop ball covers every hub, so its seed rule finds fewer seeds than parts and
partition_expansion reads past its seed vector, src/phase1/partition.cpp:347).  From those labels the
reference's own phase-2 steps run (oracle/_ref/ref_harness, fixed mode, 30 iterations, one thread: its
vector<bool> race needs a single thread, src/phase2/gpu_lp_boundary.cu:40-63).

Stored in rmat22_full.json, per k: per iteration the window size, its sorted-FNV hash and order-independent
checksum, candidates, changes, edge cut, labels hash, part vertex / intra-edge counts, penalty and RE bits and
the traversed-edge terms; the final result (edge cut, balance bits, traversed edges) and the final labels hash.
One k takes 20-40 minutes of one CPU core.
"""
from __future__ import annotations

import json
import multiprocessing
import os
import sys
import tempfile
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

GRAPH = dict(scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7)
THETA = 10000
ITERS = 30
OUT = os.path.join(HERE, "rmat22_full.json")


def build_graph():
    from dmolp_b200 import graphs

    return graphs.rmat(GRAPH["scale"], GRAPH["edge_factor"], GRAPH["a"], GRAPH["b"], GRAPH["c"], seed=GRAPH["seed"])


def graph_hash(g) -> str:
    return "%016x" % (oracle.fnv1a(g.offsets) ^ (oracle.fnv1a(g.indices) * 31 & 0xFFFFFFFFFFFFFFFF))


def run_k(k: int, txt: str, work: str) -> dict:
    g = build_graph()
    t0 = time.time()
    o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, THETA)
    lab_path = os.path.join(work, f"labels1_k{k}.bin")
    o1.labels.astype(np.int32).tofile(lab_path)
    r = oracle.run_reference(txt, k, THETA, os.path.join(work, f"ref_k{k}"), mode="fixed", iters=ITERS, threads=1,
                             labels_in=lab_path, seed_dump=False)
    assert r["labels2"].shape[0] == g.num_vertices
    res = r["result"]
    return dict(k=k, theta=THETA, iters=ITERS, graph=GRAPH, graph_hash=graph_hash(g), num_vertices=g.num_vertices,
                num_arcs=g.num_arcs, labels1_hash="%016x" % oracle.fnv1a(o1.labels),
                phase1_initial_edge_cut=int(o1.res.initial_edge_cut), phase1_seeds=o1.seeds.tolist(),
                labels2_hash="%016x" % oracle.fnv1a(r["labels2"]), result=res, trace=r["trace"],
                seconds=time.time() - t0, labels_from="oracle phase 1 (reference phase 1 undefined: fewer seeds)")


def main() -> None:
    if not oracle.reference_available():
        sys.exit("oracle/_ref/ref_harness is not built (make -C oracle with the reference tree present)")
    ks = [int(x) for x in sys.argv[1:]] or [32, 16, 64]
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    with tempfile.TemporaryDirectory() as work:
        txt = os.path.join(work, "rmat22.txt")
        from dmolp_b200 import graphs

        graphs.write_adjtext(build_graph(), txt)
        # spawned workers: a forked child of a process whose OpenMP runtime has started can hang in it
        with ProcessPoolExecutor(max_workers=len(ks), mp_context=multiprocessing.get_context("spawn")) as ex:
            futs = {k: ex.submit(run_k, k, txt, work) for k in ks}
            for k, f in futs.items():
                case = f.result()
                out[f"k{k}"] = case
                with open(OUT + ".tmp", "w") as fh:  # replaced whole, never seen half-written
                    json.dump(out, fh, indent=1, sort_keys=True)
                os.replace(OUT + ".tmp", OUT)
                print(f"k={k}: edge cut {case['result']['edge_cut']}, {case['seconds']:.0f} s", flush=True)


if __name__ == "__main__":
    main()
