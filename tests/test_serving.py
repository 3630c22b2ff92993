"""The serving loop (sigmo_server_*): resident database, continuous batching,
admission by projected device memory, per-request results.

The property the loop must keep: a request's results (per query graph and
molecule) are the same whether it runs alone or batched with others.  The
per-pair counts are also checked against the oracle for one request.
"""
import numpy as np
import pytest

import oracle
import sigmo_b200 as sb
from sigmo_b200 import _lib as L

pytestmark = pytest.mark.gpu

R = 3


def _requests(seed, n, lo=1, hi=12):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = int(rng.integers(lo, hi + 1))
        out.append(sb.generate_queries(k, 3, 12, seed=seed * 100 + i, skew_lo=4, skew_hi=9))
    return out


def _run_all(server, reqs, pairs=True, sequential=False):
    res = []
    if sequential:
        for q in reqs:
            t = server.submit(q, pairs=pairs)
            res.append((t, server.wait(t)))
    else:
        tickets = [server.submit(q, pairs=pairs) for q in reqs]
        res = [(t, server.wait(t)) for t in tickets]
    out = []
    for (t, r), q in zip(res, reqs):
        m, tot = server.query_totals(t, q.num_graphs)
        p = server.pairs(t) if pairs else None
        out.append((r, m, tot, p))
        server.release(t)
    return out


def test_serving_alone_equals_mix_and_oracle():
    db = sb.generate_molecules(2500, 10, 40, seed=901)
    reqs = _requests(902, 8)
    with sb.Server(db, iterations=R, find_first=True, max_inflight=2, max_batch_queries=24, batch_window_us=200_000) as srv:
        mixed = _run_all(srv, reqs)
        alone = _run_all(srv, reqs, sequential=True)
        st = srv.stats()
    assert max(r["batch_requests"] for r, *_ in mixed) > 1, "no request was batched with another"
    assert all(r["batch_requests"] == 1 for r, *_ in alone)
    for (rm, mm, tm, pm), (ra, ma, ta, pa) in zip(mixed, alone):
        assert rm["status"] == 0 and ra["status"] == 0
        assert np.array_equal(mm, ma) and np.array_equal(tm, ta)
        for x, y in zip(pm, pa):
            assert np.array_equal(x, y)
        assert rm["matched_pairs"] == len(pm[0]) and rm["total_matches"] == int(pm[2].sum())
        assert (pm[2] == 1).all()  # find-first: match flags
        assert rm["ms_latency"] >= rm["ms_queue"] and rm["ms_device"] > 0
    assert st["requests_completed"] == 2 * len(reqs) and st["requests_failed"] == 0
    # one request against the oracle (per GMCR slot counts -> matched pairs)
    q = reqs[0]
    ref = oracle.run_pipeline(q, db, R, oracle.REF_PTX, True)
    off, idx, per = ref["offsets"], ref["indices"], ref["per_pair"]
    graph_of_slot = np.repeat(np.arange(db.num_graphs), np.diff(off.astype(np.int64)))
    keep = per != 0
    want = (idx[keep].astype(np.uint32), graph_of_slot[keep].astype(np.uint32), per[keep].astype(np.uint64))
    got = mixed[0][3]
    for x, y in zip(got, want):
        assert np.array_equal(x, y)


def test_serving_find_all_matches_batched_form():
    db = sb.generate_molecules(1500, 10, 40, seed=911)
    reqs = _requests(912, 5, 2, 10)
    with sb.Server(db, iterations=R, find_first=False, max_inflight=3, max_batch_queries=16, batch_window_us=100_000) as srv:
        out = _run_all(srv, reqs)
    queue = sb.Queue(0)
    dg = sb.createDeviceCSRGraph(queue, db)
    for (r, m, tot, p), q in zip(out, reqs):
        qg = sb.createDeviceCSRGraph(queue, q)
        gm = sb.GMCR(queue)
        res = sb.match_batched(queue, qg, dg, R, False, None, gm)
        assert r["total_matches"] == res["total_matches"]
        counts = gm.getPairCounts()
        off, idx = gm.getGMCR()
        per_q = np.zeros(q.num_graphs, np.uint64)
        np.add.at(per_q, idx.astype(np.int64), counts)
        assert np.array_equal(tot, per_q)


def test_serving_memory_admission():
    db = sb.generate_molecules(1200, 10, 30, seed=921)
    reqs = _requests(922, 6, 4, 8)
    # find one batch's footprint, then allow a little more than one batch
    with sb.Server(db, iterations=R, max_inflight=1) as probe:
        t = probe.submit(reqs[0])
        one = probe.wait(t)["projected_bytes"]
    assert one > 0
    budget = int(one * 1.5)
    with sb.Server(db, iterations=R, max_inflight=3, max_batch_queries=8, memory_budget=budget) as srv:
        out = _run_all(srv, reqs, pairs=False)
        st = srv.stats()
        # a request larger than the whole budget fails on its own, the server keeps serving
        big = sb.generate_queries(400, 3, 12, seed=923)
        t = srv.submit(big)
        with pytest.raises(sb.SigmoError) as ei:
            srv.wait(t)
        assert ei.value.code == 3 and "memory budget" in str(ei.value)
        t2 = srv.submit(reqs[0])
        assert srv.wait(t2)["status"] == 0
    assert st["max_batches_in_flight"] == 1, "two batches were admitted above the budget"
    assert st["peak_reserved_bytes"] <= budget
    assert all(r["status"] == 0 for r, *_ in out)


def test_serving_rejects_bad_requests():
    db = sb.generate_molecules(50, 10, 20, seed=931)
    with sb.Server(db, iterations=R) as srv:
        big = sb.io.parse("n#70 l#1 " + " ".join(f"{i} 8" for i in range(70)) + " e#69 " +
                          " ".join(f"{i} {i + 1}" for i in range(69)) + "\n")
        with pytest.raises(sb.SigmoError) as ei:
            srv.submit(big)
        assert ei.value.code == 4
        with pytest.raises(sb.SigmoError):
            srv.wait(12345)


def test_serving_exact_profile_heavy_tail_against_oracle():
    """EXACT profile, find-all, on a database with molecules over 64 atoms and
    requests with queries over 16 vertices (both take the generic join):
    per-query totals equal the oracle's per-pair counts summed per query."""
    db = sb.generate_molecules(600, 6, 110, seed=931, kind=1, median=30)
    assert int(db.sizes().max()) > 64
    reqs = [sb.generate_queries(6, 3, 20, seed=932 + i, skew_lo=10, skew_hi=20) for i in range(3)]
    assert max(int(q.sizes().max()) for q in reqs) > 16
    with sb.Server(db, profile="exact", iterations=R, find_first=False, max_inflight=2, max_batch_queries=12,
                   batch_window_us=100_000) as srv:
        out = _run_all(srv, reqs, pairs=False)
    for (r, m, tot, _), q in zip(out, reqs):
        assert r["status"] == 0
        ref = oracle.run_pipeline(q, db, R, oracle.EXACT, False)
        per_q = np.zeros(q.num_graphs, np.uint64)
        np.add.at(per_q, ref["indices"].astype(np.int64), ref["per_pair"].astype(np.uint64))
        assert np.array_equal(tot, per_q)
        assert r["total_matches"] == int(per_q.sum())
