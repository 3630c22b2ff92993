"""CPU tests of the oracle: the reference's surviving known-answer tests, the
committed golden vectors, an independent brute-force count, and the REF_PTX
closed form of the join."""
import json
import random

import networkx as nx
import numpy as np
import pytest

import oracle
import pyref
from oracle import EXACT, REF_PTX, REF_X86


@pytest.fixture(scope="module")
def golden(golden_dir):
    return json.loads((golden_dir / "golden.json").read_text())


# ---- SignatureTest.CheckSignatureMethods (library/test/candidates.cpp:13-32) ----
@pytest.mark.parametrize("impl", ["oracle", "pyref"])
def test_signature_word_kat(impl):
    L = oracle.lib()
    sset = L.orc_sig_set if impl == "oracle" else pyref.sig_set
    sget = L.orc_sig_get if impl == "oracle" else pyref.sig_get
    sinc = L.orc_sig_increment if impl == "oracle" else pyref.sig_inc
    s = 0
    s = sset(s, 0, 1)
    s = sset(s, 2, 3)
    s = sset(s, 5, 2)
    s = sset(s, 15, 1)
    assert s == 0b0001000000000000000000000000000000000000001000000000001100000001
    assert sget(s, 15) == 1
    s = sinc(s, 15, 1)
    assert s == 0b0010000000000000000000000000000000000000001000000000001100000001
    s = sinc(s, 14, 1)
    assert s == 0b0010000100000000000000000000000000000000001000000000001100000001
    s = sinc(s, 14, 14)
    assert s == 0b0010111100000000000000000000000000000000001000000000001100000001
    # saturation and the "no-op, not clamp" rule (signature.hpp:44-51)
    assert sinc(sset(0, 3, 15), 3, 1) == sset(0, 3, 15)
    assert sinc(sset(0, 3, 14), 3, 5) == sset(0, 3, 14)
    assert sinc(0, 16, 1) == 0 and sget(0xFFFF, 20) == 0


# ---- CandidateTest.CheckInsertAndRemove (library/test/candidates.cpp:119-143) ----
def test_candidate_bit_layout_kat():
    """Candidates 0, 31, 32, 124 of row 0 (128 targets).  The reference's
    expected values are 64-bit literals; with its current uint32 words they
    hold for the row read as a little-endian uint64 stream."""
    q = oracle.Batch(np.array([0, 2], np.uint32), np.array([0, 0, 0], np.uint32), np.zeros(0, np.uint32),
                     np.array([5, 6], np.uint8), np.zeros(0, np.uint8))
    lab = np.zeros(128, np.uint8)
    lab[[0, 31, 32, 124]] = 5
    d = oracle.Batch(np.array([0, 128], np.uint32), np.zeros(129, np.uint32), np.zeros(0, np.uint32), lab,
                     np.zeros(0, np.uint8))
    bits = oracle.filter_candidates(q, d)
    assert bits.shape == (2, 4)  # single_node_size = 4 uint32 words
    as64 = bits.reshape(-1).view(np.uint64)
    assert int(as64[0]) == 0b0000000000000000000000000000000110000000000000000000000000000001
    assert int(as64[1]) == 0b0001000000000000000000000000000000000000000000000000000000000000
    assert int(np.unpackbits(bits[0].view(np.uint8)).sum()) == 4
    bits[0, 1] &= ~np.uint32(1)  # remove(0, 32)
    assert int(as64[0]) == 0b0000000000000000000000000000000010000000000000000000000000000001
    # insert(1, 0): row 1 starts at uint32 word 4 == uint64 word 2
    lab2 = np.zeros(128, np.uint8)
    lab2[0] = 6
    d2 = oracle.Batch(d.graph_offsets, d.row_offsets, d.column_indices, lab2, d.edge_labels)
    b2 = oracle.filter_candidates(q, d2).reshape(-1).view(np.uint64)
    assert int(b2[2]) == 1 and int(b2[3]) == 0


# ---- GraphTest.IntoDataDevice (library/test/graphs.cpp:59-120) on the fixture ----
def test_batched_csr_layout_fixture(golden):
    case = next(c for c in golden["cases"] if c["name"] in ("reference_fixtures", "synthetic_small"))
    b = oracle.parse_text(case["data_text"])
    lines = [l for l in case["data_text"].splitlines() if l.strip()]
    go, ro, col, nl = [0], [], [], []
    vo = eo = 0
    for l in lines:
        n, labels, edges = oracle.parse_line(l)
        r, c, lab, _ = oracle.to_csr(n, labels, edges)
        go.append(go[-1] + n)
        ro += [x + eo for x in r[:-1]]
        col += [x + vo for x in c]
        nl += lab
        vo, eo = vo + n, eo + len(c)
    ro.append(eo)
    assert b.graph_offsets.tolist() == go and b.row_offsets.tolist() == ro
    assert b.column_indices.tolist() == col and b.node_labels.tolist() == nl
    assert b.row_offsets[0] == 0


def test_fixture_values_by_hand(golden):
    case = [c for c in golden["cases"] if c["name"] == "reference_fixtures"]
    if not case:
        pytest.skip("golden file generated without the reference fixtures")
    b = oracle.parse_text(case[0]["data_text"])
    assert b.graph_offsets.tolist() == [0, 13, 22]
    # graph 0 vertex 0 has one neighbour (2); vertex 2 has 0, 1, 3
    assert b.row_offsets[:4].tolist() == [0, 1, 2, 5]
    assert b.column_indices[:5].tolist() == [2, 2, 0, 1, 3]
    # graph 1 starts at vertex 13, edge entry 26; its vertex 0 -> local 2
    assert b.row_offsets[13] == 26 and b.column_indices[26] == 15
    assert b.node_labels[:4].tolist() == [3, 3, 1, 3]


# ---- FilterTest.SingleFilter (library/test/filter.cpp:14-68) ---------------------
def test_filter_superset_kat(golden):
    for case in golden["cases"]:
        q, d = oracle.parse_text(case["query_text"]), oracle.parse_text(case["data_text"])
        sq, sd = oracle.generate_signatures(q), oracle.generate_signatures(d)
        bits = oracle.filter_candidates(q, d)
        for qi in range(q.total_nodes):
            for di in range(d.total_nodes):
                if q.node_labels[qi] != d.node_labels[di]:
                    continue
                if all(pyref.sig_get(int(sq[qi]), l) <= pyref.sig_get(int(sd[di]), l) for l in range(16)):
                    assert (bits[qi, di // 32] >> np.uint32(di % 32)) & 1


# ---- oracle vs the golden vectors -------------------------------------------
def _runs(golden):
    for case in golden["cases"]:
        for run in case["runs"]:
            yield case, run


def test_oracle_matches_golden(golden):
    n = 0
    for case, run in _runs(golden):
        q, d = oracle.parse_text(case["query_text"]), oracle.parse_text(case["data_text"])
        prof, R = run["profile"], run["iterations"]
        out = oracle.run_pipeline(q, d, R, prof, find_first=False, keep=True)
        ctx = f"{case['name']} prof={prof} R={R}"
        for it in range(R + 1):
            assert out["sig_data"][it].tolist() == run["sig_data"][it], ctx
            assert out["sig_query"][it].tolist() == run["sig_query"][it], ctx
            assert out["bitsets"][it].tolist() == run["bitsets"][it], f"{ctx} iteration {it}"
        assert out["offsets"].tolist() == run["offsets"], ctx
        assert out["indices"].tolist() == run["indices"], ctx
        assert out["total"] == run["total_all"] and out["per_pair"].tolist() == run["per_pair_all"], ctx
        t1, p1 = oracle.join(q, d, out["bits"], out["offsets"], out["indices"], prof, True)
        assert t1 == run["total_first"] and p1.tolist() == run["per_pair_first"], ctx
        n += 1
    assert n >= 20


def test_golden_covers_hazards(golden):
    """The edge-case set must actually exercise the profile differences."""
    edge = next(c for c in golden["cases"] if c["name"] == "edge_cases")
    by = {(r["profile"], r["iterations"]): r for r in edge["runs"]}
    assert by[(REF_PTX, 0)]["offsets"] != by[(REF_X86, 0)]["offsets"]  # 32-aligned graph end (range mask)
    assert by[(REF_PTX, 1)]["sig_data"][1] != by[(EXACT, 1)]["sig_data"][1]  # > 64-vertex graph (bitset width)
    assert by[(REF_PTX, 0)]["total_all"] != by[(EXACT, 0)]["total_all"]  # non-injective counting


# ---- independent cross-checks -----------------------------------------------------
def _small_random(seed, nd=8, nq=4):
    import sigmo_b200 as sb

    d = sb.generate_molecules(nd, 6, 22, seed=seed)
    q = sb.generate_queries(nq, 3, 6, seed=seed + 100)
    return oracle.parse_text(q.to_text()), oracle.parse_text(d.to_text())


@pytest.mark.parametrize("seed", [3, 17])
@pytest.mark.parametrize("prof", [REF_PTX, REF_X86, EXACT])
def test_oracle_vs_pyref_random(seed, prof):
    q, d = _small_random(seed)
    R = 3
    ref = pyref.run_pipeline(q, d, R, prof, False, wg=2)
    out = oracle.run_pipeline(q, d, R, prof, False, wg=2, keep=True)
    for it in range(R + 1):
        assert out["bitsets"][it].tolist() == pyref.rows_to_words(ref["bitsets"][it], d.total_nodes)
    assert out["offsets"].tolist() == ref["offsets"] and out["indices"].tolist() == ref["indices"]
    assert out["per_pair"].tolist() == ref["per_pair"]


def _nx(batch, g):
    s, e = int(batch.graph_offsets[g]), int(batch.graph_offsets[g + 1])
    G = nx.Graph()
    for v in range(s, e):
        G.add_node(v - s, label=int(batch.node_labels[v]))
    for v in range(s, e):
        for i in range(batch.row_offsets[v], batch.row_offsets[v + 1]):
            G.add_edge(v - s, int(batch.column_indices[i]) - s)
    return G


def test_exact_join_equals_bruteforce_induced_count():
    """EXACT profile, label filter only (R=0): the join counts injective
    induced label-preserving embeddings, which networkx enumerates."""
    q, d = _small_random(5, nd=10, nq=5)
    out = oracle.run_pipeline(q, d, 0, EXACT, False)
    slot = 0
    checked = 0
    for g in range(d.num_graphs):
        G = _nx(d, g)
        for k in range(out["offsets"][g], out["offsets"][g + 1]):
            qg = int(out["indices"][k])
            Q = _nx(q, qg)
            gm = nx.algorithms.isomorphism.GraphMatcher(G, Q, node_match=lambda a, b: a["label"] == b["label"])
            assert int(out["per_pair"][k]) == sum(1 for _ in gm.subgraph_isomorphisms_iter())
            checked += 1
        slot += 1
    # and every non-admitted pair has no embedding
    admitted = {(g, int(out["indices"][k])) for g in range(d.num_graphs) for k in range(out["offsets"][g], out["offsets"][g + 1])}
    for g in range(d.num_graphs):
        G = _nx(d, g)
        for qg in range(q.num_graphs):
            if (g, qg) in admitted or q.graph_offsets[qg + 1] - q.graph_offsets[qg] <= 1:
                continue
            gm = nx.algorithms.isomorphism.GraphMatcher(G, _nx(q, qg), node_match=lambda a, b: a["label"] == b["label"])
            assert not gm.subgraph_is_isomorphic()
    assert checked > 5


def test_ptx_closed_form_for_high_offset_graphs():
    """REF_PTX: for data graphs starting at vertex >= 256 the literal DFS must
    equal the closed-form tuple count."""
    import sigmo_b200 as sb

    d = oracle.parse_text(sb.generate_molecules(60, 8, 24, seed=9).to_text())
    q = oracle.parse_text(sb.generate_queries(6, 3, 6, seed=10).to_text())
    for R in (0, 2):
        for ff in (False, True):
            out = oracle.run_pipeline(q, d, R, REF_PTX, ff)
            _, closed = oracle.join_closed_form(q, d, out["bits"], out["offsets"], out["indices"], ff)
            first_high = int(np.searchsorted(d.graph_offsets[:-1], 256, side="left"))
            lo = int(out["offsets"][first_high])
            assert out["per_pair"][lo:].tolist() == closed[lo:].tolist()
            assert lo < len(closed)


def test_join_work_group_size_changes_only_low_offset_graphs():
    import sigmo_b200 as sb

    d = oracle.parse_text(sb.generate_molecules(40, 8, 24, seed=21).to_text())
    q = oracle.parse_text(sb.generate_queries(40, 3, 6, seed=22).to_text())
    out = oracle.run_pipeline(q, d, 2, REF_PTX, False, skip_join=False, wg=128)
    _, per2 = oracle.join(q, d, out["bits"], out["offsets"], out["indices"], REF_PTX, False, wg=2)
    first_high = int(np.searchsorted(d.graph_offsets[:-1], 256, side="left"))
    lo = int(out["offsets"][first_high])
    assert out["per_pair"][lo:].tolist() == per2[lo:].tolist()


def test_digest_is_order_sensitive():
    rng = np.random.default_rng(0)
    b = rng.integers(0, 2**32, size=(5, 7), dtype=np.uint64).astype(np.uint32)
    d0 = oracle.digest(b)
    b2 = b.copy()
    b2[[0, 1]] = b2[[1, 0]]
    assert d0 != oracle.digest(b2)
    b3 = b.copy()
    b3[2, 3] ^= 1
    assert d0 != oracle.digest(b3)


def _edge_label_map(b, g):
    s, e = int(b.graph_offsets[g]), int(b.graph_offsets[g + 1])
    lab = {}
    for v in range(s, e):
        for i in range(int(b.row_offsets[v]), int(b.row_offsets[v + 1])):
            lab[(v, int(b.column_indices[i]))] = int(b.edge_labels[i])
    return lab


@pytest.mark.parametrize("profile", [oracle.EXACT, oracle.REF_PTX])
def test_wildcard_join_counts_bond_labelled_embeddings(profile):
    """joinWildcardCandidates, find-all: the root's starting candidates
    partition the search, so the total is the number of tuples of candidates
    with induced adjacency and equal bond labels on query edges (injective for
    EXACT; under REF_PTX the visited set is inert for graphs starting at
    vertex >= 256, so those graphs count non-injective tuples)."""
    import itertools

    import sigmo_b200 as sb

    d = sb.generate_molecules(40, 6, 12, seed=3301)
    q = sb.generate_queries(6, 3, 5, seed=3302)
    qb, db = oracle.as_batch(q), oracle.as_batch(d)
    out = oracle.run_pipeline(qb, db, 2, profile, False)
    bits, off, idx = out["bits"], out["offsets"], out["indices"]
    total, per = oracle.join_wildcard(qb, db, bits, off, idx, profile, False)
    W = bits.shape[1]
    ql_all = {}
    for g in range(db.num_graphs):
        s, e = int(db.graph_offsets[g]), int(db.graph_offsets[g + 1])
        if profile == oracle.REF_PTX and s < 256:
            continue  # the literal visited set is live there; covered by the GPU parity test
        dlab = _edge_label_map(db, g)
        for slot in range(int(off[g]), int(off[g + 1])):
            qg = int(idx[slot])
            qo, qe = int(qb.graph_offsets[qg]), int(qb.graph_offsets[qg + 1])
            if qg not in ql_all:
                ql_all[qg] = _edge_label_map(qb, qg)
            qlab = ql_all[qg]
            cands = []
            for v in range(qo, qe):
                row = bits[v]
                cands.append([x for x in range(s, e) if (int(row[x >> 5]) >> (x & 31)) & 1])
            cnt = 0
            for tup in itertools.product(*cands):
                if profile == oracle.EXACT and len(set(tup)) < len(tup):
                    continue
                ok = True
                for i in range(qe - qo):
                    for j in range(i + 1, qe - qo):
                        qa = (qo + i, qo + j) in qlab
                        da = (tup[i], tup[j]) in dlab
                        if qa != da or (qa and qlab[(qo + i, qo + j)] != dlab[(tup[i], tup[j])]):
                            ok = False
                            break
                    if not ok:
                        break
                cnt += ok
            assert per[slot] == cnt, (g, qg, per[slot], cnt)
    assert total == int(per.sum())
