"""GPU parity: every stage of the sm_100a path, called through the C ABI,
against the oracle and the committed golden vectors — bit-exact signatures and
candidate bitsets after every refinement iteration, identical GMCR, identical
per-(query, data graph) counts in find-all and flags in find-first."""
import json

import numpy as np
import pytest

import oracle
import sigmo_b200 as sb

pytestmark = pytest.mark.gpu

DEVICE_PROFILES = (oracle.REF_PTX, oracle.EXACT)


def run_plain(qh, dh, R, profile, find_first, wg=128, keep=False):
    """The reference driver's stage order (library/src/sigmo.cpp:98-160)."""
    queue = sb.Queue(0, profile=profile, join_work_group_size=wg)
    qg, dg = sb.createDeviceCSRGraph(queue, qh), sb.createDeviceCSRGraph(queue, dh)
    cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
    sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
    sig.generateDataSignatures(dg)
    sig.generateQuerySignatures(qg)
    sb.filterCandidates(queue, qg, dg, sig, cand)
    hist = {"sig_data": [], "sig_query": [], "bitsets": []}

    def snap():
        if keep:
            hist["sig_data"].append(sig.getDataSignatures())
            hist["sig_query"].append(sig.getQuerySignatures())
            hist["bitsets"].append(cand.getHostCandidates())

    snap()
    for r in range(1, R + 1):
        sig.refineDataSignatures(dg, r)
        sig.refineQuerySignatures(qg, r)
        sb.refineCandidates(queue, qg, dg, sig, cand)
        snap()
    gm = sb.GMCR(queue)
    gm.generateGMCR(qg, dg, cand)
    nm = np.zeros(1, np.uint64)
    _, per = sb.joinCandidates(queue, qg, dg, cand, gm, nm, find_first, per_pair=True)
    off, idx = gm.getGMCR()
    hist.update(offsets=off, indices=idx, per_pair=per, total=int(nm[0]), digest=cand.digest(),
                final=cand.getHostCandidates() if keep else None, launches=queue.launch_count())
    return hist


def run_batched(qh, dh, R, profile, find_first, wg=128, keep_bits=False, join_kernel=None, **tuning):
    """keep_bits: the bitset route (final bitset materialised); otherwise the
    plane route, which never writes the bitset.  join_kernel: None the
    library default (2, the per-lane DFS with CTA-local slot regions), 0 the
    per-lane DFS machine with one work cursor, 1 the warp-cooperative frontier
    join; further tuning fields by name."""
    queue = sb.Queue(0, profile=profile, join_work_group_size=wg)
    if join_kernel is not None:
        tuning["join_kernel"] = join_kernel
    if tuning:
        queue.set_tuning(**tuning)
    qg, dg = sb.createDeviceCSRGraph(queue, qh), sb.createDeviceCSRGraph(queue, dh)
    cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes) if keep_bits else None
    gm = sb.GMCR(queue)
    res = sb.match_batched(queue, qg, dg, R, find_first, cand, gm, materialize=keep_bits)
    off, idx = gm.getGMCR()
    return {"offsets": off, "indices": idx, "per_pair": gm.getPairCounts(), "total": res["total_matches"],
            "digest": cand.digest() if keep_bits else None, "final": cand.getHostCandidates() if keep_bits else None,
            "res": res}


def run_both_batched(qh, dh, R, profile, find_first, wg=128):
    return [run_batched(qh, dh, R, profile, find_first, wg, keep_bits=False),
            run_batched(qh, dh, R, profile, find_first, wg, keep_bits=True)]


@pytest.fixture(scope="module")
def golden(golden_dir):
    return json.loads((golden_dir / "golden.json").read_text())


def _golden_runs(golden):
    for case in golden["cases"]:
        for run in case["runs"]:
            if run["profile"] in DEVICE_PROFILES:
                yield case, run


def test_plain_stages_match_golden(golden):
    n = 0
    for case, run in _golden_runs(golden):
        qh, dh = sb.io.parse(case["query_text"]), sb.io.parse(case["data_text"])
        R, prof = run["iterations"], run["profile"]
        ctx = f"{case['name']} profile={prof} R={R}"
        out = run_plain(qh, dh, R, prof, False, keep=True)
        for it in range(R + 1):
            assert out["sig_data"][it].tolist() == run["sig_data"][it], f"{ctx} data signatures, iteration {it}"
            assert out["sig_query"][it].tolist() == run["sig_query"][it], f"{ctx} query signatures, iteration {it}"
            assert out["bitsets"][it].tolist() == run["bitsets"][it], f"{ctx} bitset, iteration {it}"
        assert out["offsets"].tolist() == run["offsets"], ctx
        assert out["indices"].tolist() == run["indices"], ctx
        assert out["per_pair"].tolist() == run["per_pair_all"], ctx
        assert out["total"] == run["total_all"], ctx
        first = run_plain(qh, dh, R, prof, True)
        assert first["per_pair"].tolist() == run["per_pair_first"], ctx
        assert first["total"] == run["total_first"], ctx
        n += 1
    assert n >= 15


def test_batched_form_matches_golden(golden):
    for case, run in _golden_runs(golden):
        qh, dh = sb.io.parse(case["query_text"]), sb.io.parse(case["data_text"])
        R, prof = run["iterations"], run["profile"]
        ctx = f"{case['name']} profile={prof} R={R}"
        for ff, key in ((False, "all"), (True, "first")):
            for out in run_both_batched(qh, dh, R, prof, ff):
                if out["final"] is not None:
                    assert out["final"].tolist() == run["bitsets"][-1], ctx
                assert out["offsets"].tolist() == run["offsets"], ctx
                assert out["indices"].tolist() == run["indices"], ctx
                assert out["per_pair"].tolist() == run[f"per_pair_{key}"], f"{ctx} {key}"
                assert out["total"] == run[f"total_{key}"], f"{ctx} {key}"


def _oracle(qh, dh, R, prof, ff, wg=128, keep=False):
    return oracle.run_pipeline(qh, dh, R, prof, ff, wg=wg, keep=keep)


def _check(out, ref, ctx):
    if isinstance(out, list):
        for o in out:
            _check(o, ref, ctx)
        return
    assert out["offsets"].tolist() == ref["offsets"].tolist(), ctx
    assert out["indices"].tolist() == ref["indices"].tolist(), ctx
    assert np.array_equal(out["per_pair"], ref["per_pair"]), ctx
    assert out["total"] == ref["total"], ctx
    if out["digest"] is not None:
        assert out["digest"] == oracle.digest(ref["bits"]), ctx


@pytest.mark.parametrize("prof", DEVICE_PROFILES)
def test_small_drug_like_config(prof):
    """1,000 molecules of 10-40 atoms, 20 queries of 4-12 atoms, 6 refinement
    iterations, find-all and find-first; every iteration's bitset compared."""
    dh = sb.generate_molecules(1000, 10, 40, seed=1001)
    qh = sb.generate_queries(20, 4, 12, seed=1002)
    R = 6
    ref = _oracle(qh, dh, R, prof, False, keep=True)
    out = run_plain(qh, dh, R, prof, False, keep=True)
    for it in range(R + 1):
        assert np.array_equal(out["sig_data"][it], ref["sig_data"][it]), it
        assert np.array_equal(out["sig_query"][it], ref["sig_query"][it]), it
        assert np.array_equal(out["bitsets"][it], ref["bitsets"][it]), it
    _check(out, ref, "plain find-all")
    _check(run_both_batched(qh, dh, R, prof, False), ref, "batched find-all")
    ref1 = _oracle(qh, dh, R, prof, True)
    _check(run_plain(qh, dh, R, prof, True), ref1, "plain find-first")
    _check(run_both_batched(qh, dh, R, prof, True), ref1, "batched find-first")
    assert ref["total"] > 0 and len(ref["indices"]) > 0


@pytest.mark.parametrize("wg", [32, 64, 256])
def test_join_work_group_sizes(wg):
    """The literal join's pair-to-item assignment follows the work-group size."""
    dh = sb.generate_molecules(120, 8, 30, seed=77)
    qh = sb.generate_queries(300, 3, 8, seed=78)
    ref = _oracle(qh, dh, 2, oracle.REF_PTX, False, wg=wg)
    _check(run_plain(qh, dh, 2, oracle.REF_PTX, False, wg=wg), ref, f"plain wg={wg}")
    _check(run_both_batched(qh, dh, 2, oracle.REF_PTX, False, wg=wg), ref, f"batched wg={wg}")


@pytest.mark.parametrize("prof", DEVICE_PROFILES)
def test_heavy_tail_graphs_over_64_atoms(prof):
    dh = sb.generate_molecules(400, 6, 120, seed=31, kind=1, median=30)
    assert int(dh.sizes().max()) > 64
    qh = sb.generate_queries(25, 3, 12, seed=32)
    for R in (1, 4):
        ref = _oracle(qh, dh, R, prof, False, keep=True)
        out = run_plain(qh, dh, R, prof, False, keep=True)
        for it in range(R + 1):
            assert np.array_equal(out["bitsets"][it], ref["bitsets"][it]), (R, it)
        _check(out, ref, f"plain R={R}")
        _check(run_both_batched(qh, dh, R, prof, False), ref, f"batched R={R}")


@pytest.mark.parametrize("prof", DEVICE_PROFILES)
def test_symmetry_stress_small(prof):
    dh = sb.generate_molecules(150, 12, 50, seed=41, kind=2)
    qh = sb.generate_queries(12, 4, 10, seed=42, kind=3)
    ref = _oracle(qh, dh, 3, prof, False)
    _check(run_plain(qh, dh, 3, prof, False), ref, "plain")
    _check(run_both_batched(qh, dh, 3, prof, False), ref, "batched")
    assert ref["per_pair"].max() >= 12  # automorphic patterns give many embeddings


JOIN_SHAPES = [
    dict(join_kernel=1),  # warp-cooperative frontier join
    dict(join_kernel=0),  # per-lane DFS machine, one work cursor
    dict(join_kernel=2, join_pool=16, join_blocks_per_sm=3),  # CTA regions off: every slot from the shared pool
    dict(join_kernel=2, join_pool=1, join_blocks_per_sm=1),  # nearly all slots from the CTAs' own regions
]


@pytest.mark.parametrize("prof", DEVICE_PROFILES)
@pytest.mark.parametrize("ff", [False, True])
@pytest.mark.parametrize("shape", range(len(JOIN_SHAPES)))
def test_join_kernels_match_oracle(prof, ff, shape):
    """Every join phase-B kernel and work split gives the oracle's GMCR and
    per-pair counts: drug-like pairs, queries over 16 vertices and molecules
    over 64 atoms (both take the generic kernel), and automorphic queries on
    ring-rich molecules (thousands of embeddings per pair, the deepest DFS
    levels); the default shape gives the same counts."""
    cases = [
        (sb.generate_molecules(1500, 10, 60, seed=5101), sb.generate_queries(120, 3, 24, seed=5102, skew_lo=6, skew_hi=15), 6),
        (sb.generate_molecules(400, 6, 120, seed=5103, kind=1, median=30), sb.generate_queries(30, 3, 14, seed=5104), 4),
        (sb.generate_molecules(200, 12, 50, seed=5105, kind=2), sb.generate_queries(16, 4, 12, seed=5106, kind=3), 3),
    ]
    for i, (dh, qh, R) in enumerate(cases):
        ref = _oracle(qh, dh, R, prof, ff)
        out = run_batched(qh, dh, R, prof, ff, **JOIN_SHAPES[shape])
        _check(out, ref, f"case {i}")
        assert np.array_equal(out["per_pair"], run_batched(qh, dh, R, prof, ff)["per_pair"]), f"case {i}"
    assert ref["per_pair"].max() >= (1 if ff else 12)


@pytest.mark.parametrize("prof", DEVICE_PROFILES)
def test_empty_batches(prof):
    """An empty query batch, an empty data batch, or both: zero pairs and zero
    matches in the batched form (ordinary and graph replay) and the plain
    stage sequence."""
    empty = sb.io.parse("")
    d = sb.generate_molecules(300, 10, 30, seed=5)
    q = sb.generate_queries(10, 3, 10, seed=6)
    for qh, dh in ((empty, d), (q, empty), (empty, empty)):
        queue = sb.Queue(0, profile=prof)
        qg, dg = sb.createDeviceCSRGraph(queue, qh), sb.createDeviceCSRGraph(queue, dh)
        gm = sb.GMCR(queue)
        for ff in (False, True):
            for graph in (False, True, True):
                r = sb.match_batched(queue, qg, dg, 3, ff, None, gm, graph=graph)
                assert r["total_matches"] == 0 and r["admitted_pairs"] == 0
        out = run_plain(qh, dh, 3, prof, False)
        assert out["total"] == 0 and len(out["indices"]) == 0


def test_edge_inputs():
    # a single data graph, queries of 2 vertices, a 1-vertex query, a data graph
    # with no edges, wildcard query labels and labels >= 16
    q = "n#2 l#2 0 8 1 8 e#1 0 1 1\nn#1 l#1 0 8 e#0\nn#3 l#2 0 255 1 8 2 20 e#2 0 1 1 1 2 1\n"
    d = ("n#5 l#3 0 8 1 8 2 20 3 7 4 8 e#4 0 1 1 1 2 1 2 3 1 3 4 1\n"
         "n#3 l#1 0 8 1 8 2 8 e#0\n"
         "n#4 l#2 0 8 1 20 2 8 3 8 e#3 0 1 1 1 2 1 2 3 1\n")
    qh, dh = sb.io.parse(q), sb.io.parse(d)
    for prof in DEVICE_PROFILES:
        for R in (0, 3):
            for ff in (False, True):
                ref = _oracle(qh, dh, R, prof, ff)
                _check(run_plain(qh, dh, R, prof, ff), ref, f"plain {prof} {R} {ff}")
                _check(run_both_batched(qh, dh, R, prof, ff), ref, f"batched {prof} {R} {ff}")


def test_graph_ending_on_word_boundary_masks():
    """REF_PTX drops the last word of a multi-word range whose end is
    32-aligned (candidates.hpp:98); EXACT keeps it."""
    lines = ["n#20 l#1 " + " ".join(f"{i} 8" for i in range(20)) + " e#19 " + " ".join(f"{i} {i+1} 1" for i in range(19)),
             "n#44 l#1 " + " ".join(f"{i} 8" for i in range(44)) + " e#43 " + " ".join(f"{i} {i+1} 1" for i in range(43))]
    dh = sb.io.parse("\n".join(lines) + "\n")
    qh = sb.io.parse("n#3 l#1 0 8 1 8 2 8 e#2 0 1 1 1 2 1\n")
    outs = {}
    for prof in DEVICE_PROFILES:
        ref = _oracle(qh, dh, 0, prof, False)
        out = run_plain(qh, dh, 0, prof, False)
        _check(out, ref, str(prof))
        _check(run_both_batched(qh, dh, 0, prof, False), ref, str(prof))
        outs[prof] = out
    assert outs[oracle.REF_PTX]["total"] != outs[oracle.EXACT]["total"]


def test_stage_events_and_launch_count():
    dh = sb.generate_molecules(200, 10, 30, seed=5)
    qh = sb.generate_queries(10, 4, 8, seed=6)
    queue = sb.Queue(0)
    qg, dg = sb.createDeviceCSRGraph(queue, qh), sb.createDeviceCSRGraph(queue, dh)
    sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
    ev = sig.generateDataSignatures(dg)
    assert ev.getProfilingInfo() >= 0.0
    assert queue.launch_count() > 0
    mem, name = queue.device_info()
    assert mem > 0 and name


def test_mid_size_slice_against_oracle():
    """20,000 molecules x 120 queries (a slice of the 100k x 600 workload's
    generator), 6 iterations, both modes: device == oracle."""
    dh = sb.generate_molecules(20000, 10, 60, seed=2024)
    qh = sb.generate_queries(120, 3, 30, seed=2025, skew_lo=6, skew_hi=15)
    for ff in (False, True):
        ref = _oracle(qh, dh, 6, oracle.REF_PTX, ff)
        _check(run_both_batched(qh, dh, 6, oracle.REF_PTX, ff), ref, f"batched ff={ff}")
        _check(run_plain(qh, dh, 6, oracle.REF_PTX, ff), ref, f"plain ff={ff}")


@pytest.mark.gpu
def test_device_batch_assembly_matches_host_batching():
    d = sb.generate_molecules(3000, 5, 60, seed=4501, kind=1, median=20.0)
    q = sb.generate_queries(40, 3, 12, seed=4502)
    queue = sb.Queue(0)
    qg = sb.createDeviceCSRGraph(queue, q)
    dh = sb.createDeviceCSRGraph(queue, d)
    dl = sb.createDeviceCSRGraphFromLocal(queue, d)
    assert (dl.num_graphs, dl.total_nodes, dl.total_edges, dl.max_graph_nodes) == \
        (dh.num_graphs, dh.total_nodes, dh.total_edges, dh.max_graph_nodes)
    g1, g2 = sb.GMCR(queue), sb.GMCR(queue)
    r1 = sb.match_batched(queue, qg, dh, 4, False, None, g1)
    r2 = sb.match_batched(queue, qg, dl, 4, False, None, g2)
    assert r1["total_matches"] == r2["total_matches"] and r1["admitted_pairs"] == r2["admitted_pairs"]
    assert np.array_equal(g1.getPairCounts(), g2.getPairCounts())
    # a local neighbour id outside its graph is refused
    n, e, rows, cols = d.local_arrays()
    cols = cols.copy()
    cols[5] = n[0] + 7
    import ctypes
    from sigmo_b200 import _lib as L
    h = ctypes.c_void_p()
    nl, el = np.ascontiguousarray(d.node_labels), np.ascontiguousarray(d.edge_labels)
    rc = L.lib().sigmo_graph_create_from_local(queue._h, d.num_graphs, n.ctypes.data, e.ctypes.data, rows.ctypes.data,
                                               cols.ctypes.data, nl.ctypes.data, el.ctypes.data, ctypes.byref(h))
    assert rc == 1 and "outside its graph" in L.last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("profile,wg", [("ref-ptx", 128), ("ref-ptx", 64), ("exact", 128)])
def test_wildcard_join_matches_oracle(profile, wg):
    """joinWildcardCandidates (bond labels, max-candidate root, sub-group
    split) on the plain form's final bitset and GMCR, find-all and
    find-first, per slot against the oracle.  The batch includes the molecules
    below vertex 256, where the reference's visited bitset is live."""
    d = sb.generate_molecules(1200, 8, 40, seed=4601)
    q = sb.generate_queries(30, 3, 10, seed=4602, skew_lo=4, skew_hi=8)
    prof = {"ref-ptx": oracle.REF_PTX, "exact": oracle.EXACT}[profile]
    queue = sb.Queue(0, profile=profile, join_work_group_size=wg)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
    sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
    sig.generateDataSignatures(dg)
    sig.generateQuerySignatures(qg)
    sb.filterCandidates(queue, qg, dg, sig, cand)
    for r in range(1, 4):
        sig.refineDataSignatures(dg, r)
        sig.refineQuerySignatures(qg, r)
        sb.refineCandidates(queue, qg, dg, sig, cand)
    gm = sb.GMCR(queue)
    gm.generateGMCR(qg, dg, cand)
    off, idx = gm.getGMCR()
    bits = cand.getHostCandidates()
    for ff in (False, True):
        nm = np.zeros(1, np.uint64)
        _, per = sb.isomorphism.join.joinWildcardCandidates(queue, qg, dg, cand, gm, nm, ff, per_pair=True)
        want_total, want_per = oracle.join_wildcard(q, d, bits, off, idx, prof, ff, wg)
        assert int(nm[0]) == want_total
        assert np.array_equal(per, want_per)


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [[], ["--batched"]])
def test_cli_driver_matches_oracle(tmp_path, extra):
    """The reference driver rewritten on the C++ API (sigmo_b200/sigmo_cli):
    text files in, the full report out (candidate analysis included, the
    per-query-vertex counts on stderr), read the way SIGMo's log parser reads
    it (tests/cli_report.py restates scripts/utils/output_analyzer.py) and
    compared with the oracle: graph and vertex counts, work-group size, the
    candidate counts and their summary, refinement steps and matches."""
    import subprocess
    from pathlib import Path

    from cli_report import expected_from_oracle, parse_report

    d = sb.generate_molecules(800, 10, 40, seed=4701)
    q = sb.generate_queries(25, 3, 10, seed=4702)
    (tmp_path / "d.dat").write_text(d.to_text())
    (tmp_path / "q.dat").write_text(q.to_text())
    cli = Path(sb.__file__).resolve().parent / "sigmo_cli"
    qb, db = oracle.parse_text(q.to_text()), oracle.parse_text(d.to_text())
    for find_all in (True, False):
        cmd = [str(cli), "-Q", str(tmp_path / "q.dat"), "-D", str(tmp_path / "d.dat"), "-i", "3", "-p",
               "--max-data-graphs", "1000000", "--max-query-graphs", "1000000"] + (["--find-all"] if find_all else []) + extra
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        got = parse_report(out.stdout, out.stderr)
        ref = oracle.run_pipeline(qb, db, 3, oracle.REF_PTX, not find_all)
        want = expected_from_oracle(qb, db, ref["bits"], ref["total"], 3, find_all)
        if extra:  # the batched pipeline prints one summary line instead of the per-step lines
            want["n_refinement_steps"] = 0
        for k, v in want.items():
            assert got[k] == v, (find_all, extra, k)


@pytest.mark.gpu
@pytest.mark.parametrize("ff", [False, True])
def test_shards_keep_the_unsharded_results(ff):
    """Data graphs split into contiguous shards (global vertex ids kept as a
    vertex base): the shards' GMCR segments and per-pair counts, concatenated,
    are the unsharded run's, which are the oracle's.  REF_PTX, where results
    depend on global ids."""
    d = sb.generate_molecules(6000, 10, 60, seed=4801)
    q = sb.generate_queries(60, 3, 20, seed=4802, skew_lo=5, skew_hi=12)
    queue = sb.Queue(0)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    gm = sb.GMCR(queue)
    full = sb.match_batched(queue, qg, dg, 5, ff, None, gm)
    off, idx = gm.getGMCR()
    counts = gm.getPairCounts()
    plan = sb.shard_plan(d, 3)
    assert plan[1][2] >= 256 and sum(c for _, c, _ in plan) == d.num_graphs
    tot, seg_idx, seg_cnt = 0, [], []
    for first, count, base in plan:
        sg = sb.createDeviceShard(queue, d, first, count)
        gms = sb.GMCR(queue)
        r = sb.match_batched(queue, qg, sg, 5, ff, None, gms)
        o, i = gms.getGMCR()
        assert np.array_equal(o.astype(np.int64), off[first:first + count + 1].astype(np.int64) - int(off[first]))
        # CUDA-graph replay on the shard (shards with a base >= 256 have no literal join)
        gmg = sb.GMCR(queue)
        for _ in range(2):
            rg = sb.match_batched(queue, qg, sg, 5, ff, None, gmg, graph=True)
            assert rg["total_matches"] == r["total_matches"]
            assert np.array_equal(gmg.getPairCounts(), gms.getPairCounts())
        tot += r["total_matches"]
        seg_idx.append(i)
        seg_cnt.append(gms.getPairCounts())
    assert tot == full["total_matches"]
    assert np.array_equal(np.concatenate(seg_idx), idx) and np.array_equal(np.concatenate(seg_cnt), counts)
    # and the unsharded run is the oracle's
    ref = _oracle(q, d, 5, oracle.REF_PTX, ff)
    assert np.array_equal(off, ref["offsets"]) and np.array_equal(idx, ref["indices"])
    assert np.array_equal(counts, ref["per_pair"]) and full["total_matches"] == ref["total"]
    with pytest.raises(sb.SigmoError):
        sb.createDeviceCSRGraph(queue, d.slice(10, 5)).set_vertex_base(100)


@pytest.mark.gpu
def _batch_planes(q, R):
    """The candidate planes of a query batch: its distinct labels and
    (iteration, label, count) thresholds."""
    sig = oracle.generate_signatures(q)
    reach = oracle.new_reach(len(sig), oracle.REF_PTX)
    thresholds = set()
    for r in range(1, R + 1):
        sig = oracle.refine_signatures(q, r, oracle.REF_PTX, sig, reach)
        for v in sig.tolist():
            thresholds.update((r, l, (v >> (4 * l)) & 15) for l in range(16) if (v >> (4 * l)) & 15)
    return len(thresholds) + len(set(oracle.as_batch(q).node_labels.tolist()))


def test_query_batch_admitted_in_groups():
    """A query batch whose candidate planes exceed one admission tile's
    shared-memory budget of 96 KB (2,000 queries of 3-64 atoms, 6 iterations:
    about 200 planes; molecules up to 107 atoms, so every vertex set is two
    words and a plane row of a 32-graph tile is 512 B) is admitted group by
    group into one plane array; GMCR and per-pair counts equal the oracle's."""
    d = sb.generate_molecules(1500, 6, 120, seed=4903, kind=1, median=22.0)
    q = sb.generate_queries(2000, 3, 64, seed=4901)
    R = 6
    assert 64 < d.sizes().max() <= 128  # two words per vertex set
    assert _batch_planes(q, R) * 2 * 32 * 8 > 96 * 1024  # more than one tile: the batch is split into groups
    ref = _oracle(q, d, R, oracle.REF_PTX, False)
    got = run_both_batched(q, d, R, oracle.REF_PTX, False)
    _check(got, ref, "grouped admission")


@pytest.mark.parametrize("prof", DEVICE_PROFILES)
def test_molecules_of_129_to_192_atoms(prof):
    """A batch whose largest molecule has 129-192 atoms (146 here): every
    local vertex set takes four words (the width the kernels are built for),
    through the stage-per-launch and batched forms, with planes of four words
    split into admission groups; everything equals the oracle."""
    d = sb.generate_molecules(1500, 6, 250, seed=4903, kind=1, median=30.0)
    q = sb.generate_queries(1000, 3, 40, seed=4901)
    R = 6
    assert 128 < d.sizes().max() <= 192
    assert _batch_planes(q, R) * 4 * 32 * 8 > 96 * 1024  # four-word planes: more than one tile
    ref = _oracle(q, d, R, prof, False)
    _check(run_both_batched(q, d, R, prof, False), ref, "batched")
    _check(run_plain(q, d, R, prof, False), ref, "plain")


@pytest.mark.parametrize("prof", (oracle.REF_PTX, oracle.REF_X86))
def test_gmcr_pass_span_shapes(prof):
    """The plain form's GMCR pass stages each CTA's word span of 256 data
    graphs in shared memory: molecules of 600-900 atoms (spans at and over one
    stage, so some CTAs read global memory, and graphs spanning up to 29
    words; 200-256 atoms under REF_X86, a few rows per stage), and molecules
    of 1-3 atoms (up to 32 graphs per bitset word).
    Bitset and GMCR against the oracle; the small molecules also through the
    join."""
    q = sb.generate_queries(20, 3, 8, seed=53)
    # REF_X86's stage calls take graphs of up to 256 vertices
    big = (sb.generate_molecules(300, 600, 900, seed=51, median=750.0) if prof == oracle.REF_PTX
           else sb.generate_molecules(600, 200, 256, seed=51, median=228.0))
    for name, d in (("big", big), ("tiny", sb.generate_molecules(6000, 1, 3, seed=52, median=2.0))):
        sd, sq = oracle.generate_signatures(d), oracle.generate_signatures(q)
        bits = oracle.filter_candidates(q, d)
        rd, rq = oracle.new_reach(len(sd), prof), oracle.new_reach(len(sq), prof)
        for r in (1, 2):
            sd = oracle.refine_signatures(d, r, prof, sd, rd)
            sq = oracle.refine_signatures(q, r, prof, sq, rq)
            bits = oracle.refine_candidates(q, d, sq, sd, bits)
        off, idx = oracle.gmcr(q, d, bits, prof)
        assert len(idx) > 0, name
        queue = sb.Queue(0, profile=prof)
        qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
        cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
        sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
        sig.generateDataSignatures(dg)
        sig.generateQuerySignatures(qg)
        sb.filterCandidates(queue, qg, dg, sig, cand)
        for r in (1, 2):
            sig.refineDataSignatures(dg, r)
            sig.refineQuerySignatures(qg, r)
            sb.refineCandidates(queue, qg, dg, sig, cand)
        assert np.array_equal(cand.getHostCandidates(), bits), name
        gm = sb.GMCR(queue)
        gm.generateGMCR(qg, dg, cand)
        goff, gidx = gm.getGMCR()
        assert np.array_equal(goff, off) and np.array_equal(gidx, idx), name
        if name == "tiny":
            nm = np.zeros(1, np.uint64)
            _, per = sb.joinCandidates(queue, qg, dg, cand, gm, nm, True, per_pair=True)
            ref_total, ref_per = oracle.join(q, d, bits, off, idx, prof, True)
            assert int(nm[0]) == ref_total and np.array_equal(per, ref_per), name
