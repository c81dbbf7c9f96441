"""The reference's C++ interface over the B200 library (libdmolp_dropin.so): symbols, type layout, the
host-only entry points on the CPU, the device ones and the reference's own main.cpp on the GPU."""
import json
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from conftest import ROOT, f64_hex, golden_graph

LIB = os.path.join(ROOT, "dmolp_b200", "lib")
DROPIN = os.path.join(LIB, "libdmolp_dropin.so")
MAIN = os.path.join(ROOT, "oracle", "_ref", "dmolp_main_dropin")

REFERENCE_SIGNATURES = [
    "run_phase1(int, int, char const*, int, int, bool, bool, Graph&, GhostNodes&)",
    "run_phase2(int, int, int, Graph&, GhostNodes&, int)",
    "load_graph(char const*, int, int,", "gather_degrees(", "find_hub_nodes(", "find_first_seed(", "find_seeds(int, int, int, unsigned long,",
    "partition_expansion(int, int, int, int,", "random_partition(int, int, int, int,",
    "createBoundarySubgraphUnified(", "expandBoundaryNodes(", "runBoundaryLPOnGPU_SubgraphUnified(",
    "runBoundaryLPOnGPU_Chunked(", "createChunkSubgraph(", "freeChunkSubgraph(BoundarySubgraph&)",
    "runBoundaryLPOnGPU_Streaming(", "runBoundaryLPOnGPU_Safe(", "runBoundaryLPOnGPU_PinnedOptimized(",
    "cleanupGPUResources()",
]


def build_driver() -> str:
    out = os.path.join(LIB, "dropin_driver")
    src = os.path.join(ROOT, "tests", "dropin_driver.cpp")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "dmolp_b200", "csrc"), "-o", out, src,
                        "-L", LIB, "-ldmolp_dropin", "-ldmolp_b200", "-Wl,-rpath," + LIB], check=True)
    return out


def run_driver(txt, k, theta, iters, host_only=False, env=None):
    cmd = [build_driver(), txt, str(k), str(theta), str(iters)] + (["--host-only"] if host_only else [])
    p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return {d["what"]: d for d in (json.loads(l) for l in p.stdout.splitlines() if l.startswith("{\"what\""))}


def test_dropin_exports_reference_signatures():
    assert os.path.exists(DROPIN)
    out = subprocess.run(["nm", "-DC", "--defined-only", DROPIN], capture_output=True, text=True).stdout
    for sig in REFERENCE_SIGNATURES:
        assert sig in out, sig


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "layout_check")),
                    reason="built only where the reference headers exist")
def test_type_layout_matches_reference_headers():
    # the binary only exists if its static_asserts on size and member offsets compiled
    assert subprocess.run([os.path.join(ROOT, "oracle", "_ref", "layout_check")]).returncode == 0


def test_host_entry_points_match_reference():
    from dmolp_b200 import graphs

    name = "knn3d_2k"
    g = golden_graph(name)
    with tempfile.TemporaryDirectory() as td:
        txt = os.path.join(td, "g.txt")
        graphs.write_adjtext(g, txt)
        d = run_driver(txt, 8, 100, 5, host_only=True)
    h = d["host"]
    import json as _j
    case = _j.load(open(os.path.join(ROOT, "tests", "golden", "cases.json")))[name]
    assert h["V"] == g.num_vertices and h["E"] == g.num_arcs // 2
    assert h["hubs_hash"] == case["phase1"]["hubs_hash"]
    assert h["first"] == case["phase1"]["first_seed"]
    s = d["subgraph"]
    # window of vertices 0..19 plus their neighbours
    ids = set(range(20))
    for v in range(20):
        ids.update(g.indices[g.offsets[v]:g.offsets[v + 1]].tolist())
    assert s["nodes"] == len(ids) and s["boundary"] == 20
    assert s["mapping_hash"] == "%016x" % oracle.fnv1a(np.array(sorted(ids), np.int32))
    assert s["random_labels_hash"] == "%016x" % oracle.fnv1a((np.arange(g.num_vertices) % 8).astype(np.int32))


@pytest.mark.gpu
def test_device_entry_points_match_oracle():
    from dmolp_b200 import graphs

    name = "knn3d_2k"
    g = golden_graph(name)
    k, theta, iters = 8, 100, 12
    o1 = oracle.phase1(g.offsets, g.indices, g.raw_deg(), k, theta)
    o2 = oracle.phase2(g.offsets, g.indices, o1.labels, k, "fixed", iters)
    with tempfile.TemporaryDirectory() as td:
        txt = os.path.join(td, "g.txt")
        graphs.write_adjtext(g, txt)
        d = run_driver(txt, k, theta, iters, env=dict(os.environ, DMOLP_LP_ITERATIONS=str(iters)))
    assert d["lower_phase1"]["seeds"] == o1.seeds.tolist()
    assert d["lower_phase1"]["labels_hash"] == "%016x" % oracle.fnv1a(o1.labels)
    p1 = d["phase1"]
    assert p1["cut"] == o1.res.initial_edge_cut and p1["labels_hash"] == "%016x" % oracle.fnv1a(o1.labels)
    assert p1["vc"] == o1.vertex_counts.tolist() and p1["ec"] == o1.edge_counts.tolist()
    p2 = d["phase2"]
    assert p2["cut"] == o2.res.edge_cut
    assert p2["labels_hash"] == "%016x" % oracle.fnv1a(o2.labels)
    s = d["single_step"]
    c1, c2, c3 = s["changes"]
    assert c1 == c2 == c3 and s["same_nodes"] == 1 and s["safe_consistent"] == 1


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(MAIN), reason="built only where the reference sources exist")
def test_reference_main_runs_on_the_dropin():
    """The reference's own driver (src/main.cpp and src/utils.cpp, unmodified) linked against the drop-in
    library, on a golden graph: its report must show the reference's phase-1 and phase-2 edge cuts."""
    import json as _j

    from dmolp_b200 import graphs

    name = "knn3d_2k"
    case = _j.load(open(os.path.join(ROOT, "tests", "golden", "cases.json")))[name]
    g = golden_graph(name)
    with tempfile.TemporaryDirectory() as td:
        txt = os.path.join(td, "g.txt")
        graphs.write_adjtext(g, txt)
        p = subprocess.run([MAIN, "-m", "bfs", txt, str(case["k"]), str(case["theta"])], capture_output=True,
                           text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    m = re.search(r"Initial edge cut: (\d+)", p.stdout)
    assert m and int(m.group(1)) == case["phase1"]["initial_edge_cut"]
    cuts = re.findall(r"Phase 2 \S+:\s+(\d+)", p.stdout)
    assert cuts and int(cuts[0]) == case["runs"]["ref"]["result"]["edge_cut"], p.stdout[-3000:]
