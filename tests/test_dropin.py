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
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "dropin_driver_ref")  # the same driver on the reference's objects

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


def run_driver(txt, k, theta, iters, host_only=False, env=None, reference=False):
    exe = REF_DRIVER if reference else build_driver()
    cmd = [exe, txt, str(k), str(theta), str(iters)] + (["--host-only"] if host_only else [])
    # one OpenMP thread: the reference's subgraph construction races on a vector<bool> with more
    env = dict(env or os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=900)
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


# Texts for the host entry points: duplicates, self-loops, an empty line and rows without their reverse arcs;
# random_partition drops self-loops and duplicates (src/phase1/random.cpp:89-90).
HOST_TEXTS = {
    "dups_selfloops": "7\n1 1 2 0 3\n0 0 2\n1 0 0 6\n\n5 5 3\n4\n2 2 2\n",
    "path": "6\n1\n0 2\n1 3\n2 4\n3 5\n4\n",
}


@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="built only where the reference sources exist")
@pytest.mark.parametrize("name", sorted(HOST_TEXTS) + ["knn5000"])
def test_host_entry_points_equal_the_reference_functions(name):
    """load_graph, gather_degrees, find_hub_nodes, find_first_seed, random_partition (its CSR and labels),
    createBoundarySubgraphUnified and createChunkSubgraph: the drop-in's answers equal the reference's own
    functions' on the same text (the same driver linked against either)."""
    from dmolp_b200 import graphs

    with tempfile.TemporaryDirectory() as td:
        txt = os.path.join(td, "g.txt")
        if name in HOST_TEXTS:
            open(txt, "w").write(HOST_TEXTS[name])
        else:
            graphs.write_adjtext(graphs.knn(5000, 3, 10, seed=12), txt)
        ours = run_driver(txt, 3, 2, 5, host_only=True)
        ref = run_driver(txt, 3, 2, 5, host_only=True, reference=True)
    assert ours == ref


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="built only where the reference sources exist")
def test_device_entry_points_equal_the_reference_functions():
    """Every entry point of the driver against the reference's own functions (its phase 1, its run_phase2
    loop, its single-step GPU functions with its kernel built for sm_100a), on a 5,000-vertex 3-D k-NN graph:
    lower-level and whole phase 1, run_phase2 with the reference's stopping rules, one LP step through
    runBoundaryLPOnGPU_SubgraphUnified, _Chunked with room for one 1024-node chunk (the subgraph needs four:
    arcs across chunks are dropped, gpu_lp_boundary.cu:571-675) and _Streaming with and without room, and the
    -m random path (random_partition, then run_phase2)."""
    from dmolp_b200 import graphs

    g = graphs.knn(5000, 3, 10, seed=12)
    k, theta = 6, 100
    with tempfile.TemporaryDirectory() as td:
        txt = os.path.join(td, "g.txt")
        graphs.write_adjtext(g, txt)
        ours = run_driver(txt, k, theta, 0)
        ref = run_driver(txt, k, theta, 0, reference=True)
    assert ours["chunks"]["subgraph_nodes"] > 3 * 1024  # four chunks of the minimum size
    for what in ("host", "subgraph", "lower_phase1", "phase1", "phase2", "step_unified", "step_chunked",
                 "step_streaming_chunked", "step_streaming", "chunks", "random_phase1", "random_phase2"):
        assert ours[what] == ref[what], what
    for key in ("window", "window_set_hash", "changes"):
        assert ours["single_step"][key] == ref["single_step"][key], key
    # the chunked paths drop arcs that cross chunks: they differ from the whole subgraph's step here
    assert ours["step_chunked"] != ours["step_unified"]
