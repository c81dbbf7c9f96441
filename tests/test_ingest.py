"""Device parse of the reference's adjacency text (dmolp_graph_upload_adjtext / dmolp_graph_load_adjtext)
against the oracle's loader, which restates the reference's load_graph + CSR build (src/phase1/init.cpp:15-100,
src/phase1/partition.cpp:227-262): offsets, indices and raw degrees must be identical, for the tricky texts
the host loader is tested on, NUL bytes, unsorted rows of every length class (thread, block, merge sort),
long lines spanning many parse tiles, seeded fuzz, and a generated graph that is then partitioned."""
import os
import tempfile

import numpy as np
import pytest

import oracle

TEXTS = {
    "plain": b"4\n1 2\n0 2\n0 1 3\n2\n",
    "dups_selfloop": b"3\n1 1 2 0\n0 0\n1 0\n",
    "leading_space": b"3\n 1\n0\n\n",
    "separators": b"3\n1,2\n0\t2\r\n0  1 \n",
    "unterminated_last": b"3\n1\n0\n1",
    "empty_lines": b"5\n\n\n3\n2\n\n",
    "header_only": b"7\n",
    "leading_zeros": b"3\n002 01\n0000\n1\n",
    "nul_mid_line": b"3\n1 2\x00 0\n2\x00\n\x00 1\n",
    "nul_runs": b"4\n3\x00\x00 1\x002\n0 1\n\x00\n1 2 3\x00\n",
    "trailing_separators": b"2\n1 ,; \n0\t\t\n",
    "long_digit_runs": b"3\n000000001 0000000000002 00000002\n00000000\n000000000000000000000001 2\n",
}


def oracle_csr(text: bytes):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.txt")
        with open(p, "wb") as f:
            f.write(text)
        return oracle.load_adjtext(p)


def check_same(part, text, via_file=False, via_device=False):
    off, col, raw = oracle_csr(text)
    if via_device:
        import torch

        t = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda() if text else torch.zeros(0, dtype=torch.uint8,
                                                                                                  device="cuda")
        info = part.upload_adjtext(t)
    elif via_file:
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "g.txt")
            with open(p, "wb") as f:
                f.write(text)
            info = part.upload_adjtext(p)
    else:
        info = part.upload_adjtext(text)
    g = part.graph_arrays()
    assert info["num_vertices"] == off.size - 1 and info["num_arcs"] == col.size
    assert info["num_tokens"] == int(raw.astype(np.int64).sum())
    assert np.array_equal(g.offsets, off)
    assert np.array_equal(g.indices, col)
    assert np.array_equal(g.raw_degree, raw)
    return info


def unsorted_text(seed=0):
    """Rows of every sort class: short (thread), up to 4096 tokens (one block), beyond (merge sort), with
    duplicates, self-loops, sorted rows with duplicates, and already strictly increasing rows."""
    rng = np.random.default_rng(seed)
    nv = 3000
    lens = list(rng.integers(0, 40, size=nv))
    for i, L in ((5, 700), (17, 4096), (18, 4097), (40, 9000), (41, 20000), (77, 70000)):
        lens[i] = L
    lines = []
    for v, L in enumerate(lens):
        row = rng.integers(0, nv, size=L)
        if v % 7 == 0:
            row = np.sort(row)  # sorted, may hold duplicates
        elif v % 7 == 1:
            row = np.unique(row)  # strictly increasing
        lines.append(" ".join(map(str, row.tolist())))
    return (f"{nv}\n" + "\n".join(lines) + "\n").encode()


def fuzz_text(seed):
    rng = np.random.default_rng(seed)
    nv = int(rng.integers(1, 60))
    seps = [b" ", b",", b"\t", b"  ", b" ;", b"\r", b"x"]
    out = [b"%d\n" % nv]
    for _ in range(nv):
        parts = []
        if rng.random() < 0.1:
            parts.append(seps[int(rng.integers(len(seps)))])
        for _ in range(int(rng.integers(0, 12))):
            parts.append(b"0" * int(rng.integers(0, 2)) + b"%d" % int(rng.integers(0, nv)))
            parts.append(seps[int(rng.integers(len(seps)))])
        if rng.random() < 0.1:
            parts.insert(int(rng.integers(len(parts) + 1)), b"\x00")
        out.append(b"".join(parts) + b"\n")
    if rng.random() < 0.3:
        out.append(b"1 2")  # unterminated: dropped
    return b"".join(out)


def test_oracle_loader_on_the_extra_texts():
    """The oracle (pinned to the reference's loader by the CPU tests) on the texts only this file uses."""
    off, col, raw = oracle_csr(TEXTS["nul_mid_line"])
    assert off.tolist() == [0, 2, 1 + 2, 3] and col.tolist() == [1, 2, 2] and raw.tolist() == [2, 1, 0]
    off, col, raw = oracle_csr(TEXTS["leading_zeros"])
    assert col.tolist() == [1, 2, 0, 1] and raw.tolist() == [2, 1, 1]
    off, col, raw = oracle_csr(TEXTS["header_only"])
    assert off.tolist() == [0] and col.size == 0


@pytest.fixture(scope="module")
def part():
    from dmolp_b200.partitioner import Partitioner

    p = Partitioner(0)
    yield p
    p.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(TEXTS))
def test_device_parse_matches_oracle(part, name):
    info = check_same(part, TEXTS[name])
    assert info["kernels"] > 0 or info["num_vertices"] == 0
    check_same(part, TEXTS[name], via_file=True)
    check_same(part, TEXTS[name], via_device=True)


@pytest.mark.gpu
def test_device_parse_sorts_and_dedupes_every_row_class(part):
    text = unsorted_text()
    info = check_same(part, text)
    assert info["rows_sorted_on_device"] > 0
    check_same(part, text, via_file=True)
    check_same(part, text, via_device=True)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(12))
def test_device_parse_fuzz(part, seed):
    check_same(part, fuzz_text(seed))


@pytest.mark.gpu
def test_device_parse_long_lines_across_tiles(part):
    """A hub line far longer than one 16 KiB parse tile, numbers straddling tile edges, and a file longer
    than one pinned staging slot (32 MiB)."""
    rng = np.random.default_rng(4)
    nv = 400_000
    lines = [" ".join(map(str, np.unique(rng.integers(0, nv, size=int(rng.integers(0, 30)))).tolist()))
             for _ in range(nv)]
    lines[3] = " ".join(map(str, np.arange(0, nv, 2).tolist()))  # ~600 KB of text on one line
    text = (f"{nv}\n" + "\n".join(lines) + "\n").encode()
    assert len(text) > 33 << 20
    info = check_same(part, text, via_file=True)
    assert info["rows_sorted_on_device"] == 0
    check_same(part, text, via_device=True)


@pytest.mark.gpu
def test_device_parse_rejects_bad_ids_and_keeps_previous_graph(part):
    from dmolp_b200.partitioner import DmolpError

    part.upload_adjtext(TEXTS["plain"])
    before = part.graph_arrays()
    for bad in (b"2\n1\n5\n", b"2\n1\n99999999999999999999\n", b"2\n1\n4294967296\n", b"2\n1\n2147483648\n",
                b"no newline"):
        with pytest.raises(DmolpError):
            part.upload_adjtext(bad)
    after = part.graph_arrays()
    assert np.array_equal(before.offsets, after.offsets) and np.array_equal(before.indices, after.indices)


@pytest.mark.gpu
def test_device_parsed_graph_partitions_like_host_loaded(part):
    """Generated graph -> text -> device parse -> phase 1 + phase 2 gives exactly the host path's results."""
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import Partitioner

    g = graphs.rmat(14, 8, seed=11)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.txt")
        graphs.write_adjtext(g, p)
        part.upload_adjtext(p)
    h = part.graph_arrays()
    assert np.array_equal(h.offsets, g.offsets) and np.array_equal(h.indices, g.indices)
    assert np.array_equal(h.raw_degree, g.degree())
    m1 = part.phase1(16, 1000)
    r1 = part.phase2(16, "fixed", 15, records=False)
    lab1 = part.labels()
    q = Partitioner(0)
    q.upload(g)
    m2 = q.phase1(16, 1000)
    r2 = q.phase2(16, "fixed", 15, records=False)
    assert m1.seeds == m2.seeds and m1.initial_edge_cut == m2.initial_edge_cut
    assert m1.total_edges == m2.total_edges
    assert r1.edge_cut == r2.edge_cut and np.array_equal(lab1, q.labels())
    q.close()


@pytest.mark.gpu
def test_run_phase1_from_file_matches_oracle(tmp_path):
    """The reference's run_phase1(graph_file, ...) form: the file parsed on the device, then phase 1 and
    phase 2 on the resident graph, against the oracle on the same text."""
    from dmolp_b200 import graphs
    from dmolp_b200.partitioner import run_phase1, run_phase2

    g = graphs.knn(3000, 3, 10, seed=2)
    path = str(tmp_path / "g.txt")
    graphs.write_adjtext(g, path)
    off, col, raw = oracle.load_adjtext(path)
    m, p = run_phase1(path, 8, 100)
    o1 = oracle.phase1(off, col, raw, 8, 100)
    assert np.array_equal(p.labels(), o1.labels) and m.seeds == o1.seeds.tolist()
    assert m.total_edges == int(raw.astype(np.int64).sum()) // 2
    r = run_phase2(p, 8, mode="fixed", iterations=10)
    o2 = oracle.phase2(off, col, o1.labels, 8, "fixed", 10)
    assert np.array_equal(p.labels(), o2.labels) and r.edge_cut == o2.res.edge_cut
    p.close()
