"""CPU tests of the product library's host side: the C ABI loads and exports
every declared symbol, the parser / batcher / generator agree with the
oracle's restatement, and errors come back as status codes."""
import ctypes
import json
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
import sigmo_b200 as sb
from sigmo_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").rglob("*.h"):
        names |= set(re.findall(r"SIGMO_API\s+[\w\s\*]+?\b(sigmo_\w+)\s*\(", h.read_text()))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(str(sb.library_path()))
    names = declared_symbols()
    assert len(names) >= 40
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_version_and_error_plumbing():
    assert b"sm_100a" in _lib.lib().sigmo_version()
    with pytest.raises(sb.SigmoError) as ei:
        sb.HostGraphs.from_text("n#2 l#3 0 1 1 1 e#1 0 1 1 7\n")  # 4 edge tokens for 1 edge
    assert ei.value.code == 5 and "Invalid graph format" in str(ei.value)
    with pytest.raises(sb.SigmoError) as ei:
        sb.HostGraphs.from_text("n#2 l#3 0 1 5 1 e#0\n")  # vertex id out of range
    assert ei.value.code == 5


@pytest.fixture(scope="module")
def golden(golden_dir):
    return json.loads((golden_dir / "golden.json").read_text())


def _same(h, b):
    for f in ("graph_offsets", "row_offsets", "column_indices", "node_labels", "edge_labels"):
        assert np.array_equal(np.asarray(getattr(h, f)), np.asarray(getattr(b, f))), f


def test_parser_matches_oracle_restatement(golden):
    for case in golden["cases"]:
        for key in ("query_text", "data_text"):
            _same(sb.io.parse(case[key]), oracle.parse_text(case[key]))


def test_parser_fixture_shapes(golden):
    case = [c for c in golden["cases"] if c["name"] == "reference_fixtures"]
    if not case:
        pytest.skip("golden file generated without the reference fixtures")
    d = sb.io.parse(case[0]["data_text"])
    q = sb.io.parse(case[0]["query_text"])
    assert d.num_graphs == 2 and d.total_nodes == 22 and d.sizes().tolist() == [13, 9]
    assert q.num_graphs == 4 and q.sizes().tolist() == [3, 4, 5, 4]


def test_two_token_edges_default_label_zero():
    h = sb.io.parse("n#3 l#2 0 1 1 2 2 1 e#2 0 1 1 2\n")
    assert h.edge_labels.tolist() == [0, 0, 0, 0]
    assert h.column_indices.tolist() == [1, 0, 2, 1]


def test_self_loop_csr_quirk():
    """toCSRGraph (graph.hpp:233-244): a self-loop writes one slot and leaves the
    second as vertex 0 (the reference's behaviour, kept)."""
    text = "n#3 l#2 0 1 1 2 2 1 e#2 1 1 1 1 2 1\n"
    h = sb.io.parse(text)
    _same(h, oracle.parse_text(text))
    assert h.row_offsets.tolist() == [0, 0, 3, 4]
    assert h.column_indices.tolist() == [1, 0, 2, 1]


def test_format_roundtrip_generated():
    m = sb.generate_molecules(50, 10, 40, seed=4)
    t = m.to_text()
    m2 = sb.io.parse(t)
    _same(m2, oracle.parse_text(t))
    assert m2.graph_offsets.tolist() == m.graph_offsets.tolist()
    assert m2.node_labels.tolist() == m.node_labels.tolist()
    # same topology (as sets of undirected edges per graph)
    def edges(h):
        s = set()
        for v in range(h.total_nodes):
            for i in range(h.row_offsets[v], h.row_offsets[v + 1]):
                s.add((v, int(h.column_indices[i])))
        return s
    assert edges(m) == edges(m2)


def test_slice_and_concat():
    m = sb.generate_molecules(30, 5, 25, seed=8)
    a, b = m.slice(0, 12), m.slice(12, 18)
    c = a.concat(b)
    _same(c, m)
    assert b.graph_offsets[0] == 0 and b.row_offsets[0] == 0


def test_generator_deterministic_and_drug_like():
    a = sb.generate_molecules(2000, 10, 40, seed=123)
    b = sb.generate_molecules(2000, 10, 40, seed=123)
    _same(a, b)
    c = sb.generate_molecules(2000, 10, 40, seed=124)
    assert a.total_nodes != c.total_nodes or a.node_labels.tolist() != c.node_labels.tolist()
    sizes = a.sizes()
    assert sizes.min() >= 10 and sizes.max() <= 40 and 20 < sizes.mean() < 30
    lab = np.bincount(a.node_labels, minlength=11) / a.total_nodes
    assert 0.6 < lab[8] < 0.8  # C
    assert 0.06 < lab[0] < 0.16 and 0.07 < lab[7] < 0.17  # N, O
    deg = np.diff(a.row_offsets.astype(np.int64))
    assert deg.max() <= 4
    # every molecule is connected (BFS from vertex 0 of each graph)
    go, ro, col = a.graph_offsets, a.row_offsets, a.column_indices
    for g in range(0, 2000, 97):
        s, e = int(go[g]), int(go[g + 1])
        seen, st = {s}, [s]
        while st:
            v = st.pop()
            for i in range(ro[v], ro[v + 1]):
                w = int(col[i])
                if w not in seen:
                    seen.add(w)
                    st.append(w)
        assert len(seen) == e - s


def test_queries_are_connected_and_sized():
    q = sb.generate_queries(300, 3, 30, seed=5, skew_lo=6, skew_hi=15)
    sz = q.sizes()
    assert sz.min() >= 3 and sz.max() <= 30
    assert ((sz >= 6) & (sz <= 15)).mean() > 0.6
    heavy = sb.generate_molecules(3000, 6, 120, seed=3, kind=1, median=22)
    hs = heavy.sizes()
    assert 18 <= np.median(hs) <= 26 and hs.max() > 64
    ring = sb.generate_molecules(200, 12, 60, seed=4, kind=2)
    auto = sb.generate_queries(100, 4, 12, seed=6, kind=3)
    assert ring.num_graphs == 200 and auto.num_graphs == 100


def test_queue_without_gpu_is_an_error_not_a_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sb.SigmoError) as ei:
        sb.Queue(0)
    assert ei.value.code == 6


def test_binary_batch_roundtrip_and_damage(tmp_path):
    g = sb.generate_molecules(300, 5, 40, seed=4401, kind=1, median=18.0)
    path = tmp_path / "batch.bin"
    g.save(path)
    h = sb.HostGraphs.load(path)
    for f in ("graph_offsets", "row_offsets", "column_indices", "node_labels", "edge_labels"):
        assert np.array_equal(getattr(g, f), getattr(h, f)), f
    raw = path.read_bytes()
    (tmp_path / "short.bin").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(sb.SigmoError) as ei:
        sb.HostGraphs.load(tmp_path / "short.bin")
    assert ei.value.code == 5
    bad = bytearray(raw)
    bad[-(g.total_edges * 5 + g.total_nodes) - 4:-(g.total_edges * 5 + g.total_nodes)] = (10**9).to_bytes(4, "little")
    (tmp_path / "bad.bin").write_bytes(bytes(bad))
    with pytest.raises(sb.SigmoError):
        sb.HostGraphs.load(tmp_path / "bad.bin")
    with pytest.raises(sb.SigmoError):
        sb.HostGraphs.load(tmp_path / "missing.bin")


def test_local_arrays_rebuild_the_batch():
    g = sb.generate_molecules(200, 3, 30, seed=4402)
    n, e, rows, cols = g.local_arrays()
    goff = np.concatenate([[0], np.cumsum(n.astype(np.int64))])
    ebase = np.concatenate([[0], np.cumsum(e.astype(np.int64))])
    # global row pointers and neighbour ids from the local arrays
    rr = []
    for k in range(len(n)):
        start = goff[k] + k
        rr.append(rows[start:start + n[k]].astype(np.int64) + ebase[k])
    rr.append([ebase[-1]])
    assert np.array_equal(np.concatenate(rr), g.row_offsets.astype(np.int64))
    assert np.array_equal(cols.astype(np.int64) + np.repeat(goff[:-1], e), g.column_indices.astype(np.int64))


def test_host_workload_library_matches_the_product_generator():
    """bench.py's reference arm makes its inputs with oracle/libsigmo_workload.so
    (the same generator compiled for the host alone); its graphs and slices are
    the product library's."""
    from oracle import workload

    for kind, args in ((0, (400, 10, 60)), (1, (300, 6, 120)), (2, (200, 10, 64))):
        a = workload.generate_molecules(*args, seed=91 + kind, kind=kind)
        b = sb.generate_molecules(*args, seed=91 + kind, kind=kind)
        _same(b, a)
        _same(b.slice(37, 120), workload.slice_graphs(a, 37, 120))
    for qkind in (0, 3):
        _same(sb.generate_queries(50, 3, 30, seed=7, kind=qkind, skew_lo=6, skew_hi=15),
              workload.generate_queries(50, 3, 30, seed=7, kind=qkind, skew_lo=6, skew_hi=15))
