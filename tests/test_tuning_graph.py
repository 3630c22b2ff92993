"""CUDA-graph replay of the batched form and the join autotuner.

Graph mode (SIGMO_MATCH_CUDA_GRAPH) must give the same totals and per-pair
counts as the ordinary call on every replay, and recapture when the inputs
change; every launch shape the autotuner tries must give the same result.
"""
import numpy as np
import pytest

import oracle
import sigmo_b200 as sb

pytestmark = pytest.mark.gpu

R = 4


def _graphs(queue, nd, nq, seed):
    d = sb.generate_molecules(nd, 10, 40, seed=seed)
    q = sb.generate_queries(nq, 3, 20, seed=seed + 1, skew_lo=5, skew_hi=12)
    return q, d, sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)


def test_graph_mode_replays_match_the_ordinary_call():
    queue = sb.Queue(0)
    q, d, qg, dg = _graphs(queue, 3000, 60, 1701)
    ref_m = sb.GMCR(queue)
    ref = sb.match_batched(queue, qg, dg, R, False, None, ref_m)
    ref_counts = ref_m.getPairCounts()
    gm = sb.GMCR(queue)
    for call in range(4):  # run + capture, then replays
        res = sb.match_batched(queue, qg, dg, R, False, None, gm, graph=True)
        assert res["total_matches"] == ref["total_matches"], f"call {call}"
        assert res["admitted_pairs"] == ref["admitted_pairs"]
        assert np.array_equal(gm.getPairCounts(), ref_counts), f"call {call}"
    # find-first on the same handle: a different key, so a new capture
    ff = sb.match_batched(queue, qg, dg, R, True, None, gm, graph=True)
    ff2 = sb.match_batched(queue, qg, dg, R, True, None, gm, graph=True)
    assert ff["total_matches"] == ff2["total_matches"] == int((ref_counts > 0).sum())
    # other data graphs on the same GMCR object
    q2, d2, qg2, dg2 = _graphs(queue, 1200, 30, 1711)
    want = oracle.run_pipeline(q2, d2, R, oracle.REF_PTX, False)
    for _ in range(2):
        r2 = sb.match_batched(queue, qg2, dg2, R, False, None, gm, graph=True)
        assert r2["total_matches"] == want["total"]
        assert np.array_equal(gm.getPairCounts(), want["per_pair"])


def test_autotune_keeps_results_and_sets_the_queue():
    queue = sb.Queue(0)
    q, d, qg, dg = _graphs(queue, 4000, 80, 1721)
    base = sb.match_batched(queue, qg, dg, R, False, None, sb.GMCR(queue))
    base_ff = sb.match_batched(queue, qg, dg, R, True, None, sb.GMCR(queue))
    t = sb.autotune(queue, qg, dg, R, False, reps=1)
    assert t["ms_join"] > 0 and t["ms_join_default"] > 0
    assert t["ms_join"] <= t["ms_join_default"] * 1.05
    got = queue.get_tuning()
    for k in ("join_blocks_per_sm", "join_chunk", "overflow_blocks", "overflow_serial", "mask_chunk_slots", "overflow_split",
              "join_kernel", "join_pool"):
        assert got[k] == t[k]
    after = sb.match_batched(queue, qg, dg, R, False, None, sb.GMCR(queue))
    assert after["total_matches"] == base["total_matches"]
    # explicit shapes, including the serial overflow path and small mask chunks
    for split in (1, 3, 32):
        queue.set_tuning(join_blocks_per_sm=1, join_chunk=16, overflow_blocks=148, overflow_serial=1, mask_chunk_slots=1,
                         overflow_split=split)
        gm = sb.GMCR(queue)
        r = sb.match_batched(queue, qg, dg, R, False, None, gm)
        assert r["total_matches"] == base["total_matches"]
        f = sb.match_batched(queue, qg, dg, R, True, None, gm)
        assert f["total_matches"] == base_ff["total_matches"]
    # every phase-B kernel under graph replay, the default one with CTA regions and without
    for shape in (dict(join_kernel=1, join_blocks_per_sm=3), dict(join_kernel=0, join_blocks_per_sm=3),
                  dict(join_kernel=2, join_blocks_per_sm=4, join_pool=2), dict(join_kernel=2, join_blocks_per_sm=4, join_pool=16)):
        queue.set_tuning(join_chunk=4, mask_chunk_slots=8, overflow_split=16, **shape)
        gm = sb.GMCR(queue)
        for _ in range(3):
            r = sb.match_batched(queue, qg, dg, R, False, None, gm, graph=True)
            assert r["total_matches"] == base["total_matches"], shape
    with pytest.raises(sb.SigmoError):
        queue.set_tuning(join_blocks_per_sm=9)
    with pytest.raises(sb.SigmoError):
        queue.set_tuning(join_kernel=3)
    with pytest.raises(sb.SigmoError):
        queue.set_tuning(join_pool=17)


def test_graph_mode_exact_profile():
    """Graph replay under the EXACT profile equals the oracle on every replay."""
    queue = sb.Queue(0, profile=oracle.EXACT)
    d = sb.generate_molecules(1500, 10, 40, seed=1731)
    q = sb.generate_queries(40, 3, 20, seed=1732, skew_lo=5, skew_hi=12)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    want = oracle.run_pipeline(q, d, R, oracle.EXACT, False)
    gm = sb.GMCR(queue)
    for call in range(3):
        r = sb.match_batched(queue, qg, dg, R, False, None, gm, graph=True)
        assert r["total_matches"] == want["total"], f"call {call}"
        assert np.array_equal(gm.getPairCounts(), want["per_pair"]), f"call {call}"


def test_no_admitted_pairs():
    """A query batch that no molecule admits (labels the generator never
    emits): zero pairs and zero matches in an ordinary call, under graph
    replay, and as a serving request."""
    d = sb.generate_molecules(800, 10, 30, seed=1741)
    q = sb.io.parse("n#3 l#1 0 13 1 13 2 14 e#2 0 1 1 1 2 1\nn#2 l#1 0 15 1 15 e#1 0 1 1\n")
    for prof in (oracle.REF_PTX, oracle.EXACT):
        queue = sb.Queue(0, profile=prof)
        qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
        gm = sb.GMCR(queue)
        for ff in (False, True):
            r = sb.match_batched(queue, qg, dg, R, ff, None, gm)
            assert r["admitted_pairs"] == 0 and r["total_matches"] == 0
            for _ in range(2):
                r = sb.match_batched(queue, qg, dg, R, ff, None, gm, graph=True)
                assert r["admitted_pairs"] == 0 and r["total_matches"] == 0
    with sb.Server(d, iterations=R, find_first=True, max_inflight=1) as srv:
        t = srv.submit(q, pairs=True)
        res = srv.wait(t)
        assert res["status"] == 0 and res["matched_pairs"] == 0 and res["total_matches"] == 0
        m, tot = srv.query_totals(t, q.num_graphs)
        assert not m.any() and not tot.any()
        assert len(srv.pairs(t)[0]) == 0


def test_several_mask_chunks_on_two_streams():
    """More admitted slots than one level-mask chunk: chunks alternate between
    two streams (each with its own mask buffer and work cursor).  Ordinary
    calls and graph replays, with the overflow join after or beside the main
    join, give the single-chunk per-pair counts."""
    queue = sb.Queue(0)
    d = sb.generate_molecules(40000, 10, 60, seed=20251)
    q = sb.generate_queries(600, 3, 30, seed=20252, skew_lo=6, skew_hi=15)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    gm = sb.GMCR(queue)
    ref = sb.match_batched(queue, qg, dg, 6, False, None, gm)
    assert ref["admitted_pairs"] > 2 * (1 << 20)  # three chunks of 2^20 slots
    ref_counts = gm.getPairCounts()
    for serial in (1, 0):
        queue.set_tuning(mask_chunk_slots=1, overflow_serial=serial)
        g2 = sb.GMCR(queue)
        for graph in (False, True, True):
            r = sb.match_batched(queue, qg, dg, 6, False, None, g2, graph=graph)
            assert r["total_matches"] == ref["total_matches"], (serial, graph)
            assert np.array_equal(g2.getPairCounts(), ref_counts), (serial, graph)
