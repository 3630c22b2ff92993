"""The join step budget: a join lane (a warp for the frontier join) that leaves
more DFS levels than the queue's budget stops, the kernels raise a status word,
and the call returns SIGMO_ERR_TIMEOUT instead of running on; the queue stays
usable, and a budget that is not reached changes no result.  No GPU wait is
involved: the kernels count their own steps and return."""
import numpy as np
import pytest

import oracle
import sigmo_b200 as sb

pytestmark = pytest.mark.gpu

TIMEOUT = 7  # SIGMO_ERR_TIMEOUT


def _symmetric_case():
    # ring-rich molecules x automorphic queries: thousands of DFS levels per pair
    d = sb.generate_molecules(600, 12, 50, seed=941, kind=2)
    q = sb.generate_queries(16, 6, 12, seed=942, kind=3)
    return q, d


@pytest.mark.parametrize("join_kernel", [0, 1, 2])
@pytest.mark.parametrize("prof", ["ref-ptx", "exact"])
def test_budget_spent_returns_timeout_and_queue_recovers(join_kernel, prof):
    q, d = _symmetric_case()
    queue = sb.Queue(0, profile=prof)
    queue.set_tuning(join_kernel=join_kernel)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    gm = sb.GMCR(queue)
    want = sb.match_batched(queue, qg, dg, 3, False, None, gm)
    want_counts = gm.getPairCounts()
    assert want["total_matches"] > 10 * want["admitted_pairs"]

    queue.set_join_budget(1_000_000_000)  # never reached: same results, ordinary call and graph replay
    assert queue.join_budget() == 1_000_000_000
    for graph in (False, True, True):
        r = sb.match_batched(queue, qg, dg, 3, False, None, gm, graph=graph)
        assert r["total_matches"] == want["total_matches"] and np.array_equal(gm.getPairCounts(), want_counts)

    queue.set_join_budget(2)
    for graph in (False, True, True):
        with pytest.raises(sb.SigmoError) as ei:
            sb.match_batched(queue, qg, dg, 3, False, None, gm, graph=graph)
        assert ei.value.code == TIMEOUT and "step budget" in str(ei.value)

    queue.set_join_budget(0)
    r = sb.match_batched(queue, qg, dg, 3, False, None, gm)
    assert r["total_matches"] == want["total_matches"] and np.array_equal(gm.getPairCounts(), want_counts)


def test_budget_in_the_plain_join():
    """The stage-per-launch join (the reference's literal DFS) honours it too."""
    q, d = _symmetric_case()
    queue = sb.Queue(0)
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
    queue.set_join_budget(3)
    nm = np.zeros(1, np.uint64)
    with pytest.raises(sb.SigmoError) as ei:
        sb.joinCandidates(queue, qg, dg, cand, gm, nm, False)
    assert ei.value.code == TIMEOUT and int(nm[0]) == 0
    queue.set_join_budget(0)
    _, per = sb.joinCandidates(queue, qg, dg, cand, gm, nm, False, per_pair=True)
    ref = oracle.run_pipeline(q, d, 3, oracle.REF_PTX, False)
    assert int(nm[0]) == ref["total"] and np.array_equal(per, ref["per_pair"])


def test_server_fails_only_the_batch_over_budget():
    """A serving loop with a join budget of 40 DFS levels per lane: a request
    of automorphic queries on ring-rich molecules runs out and fails with
    SIGMO_ERR_TIMEOUT; a request of two-vertex queries (one level per pair)
    submitted after it still gets the oracle's answer."""
    d = sb.generate_molecules(3000, 12, 40, seed=951, kind=2)
    heavy = sb.generate_queries(8, 8, 12, seed=952, kind=3)
    light = sb.io.parse("n#2 l#1 0 8 1 8 e#1 0 1 1\nn#2 l#2 0 8 1 7 e#1 0 1 2\n")
    srv = sb.Server(d, iterations=3, find_first=False, max_inflight=1, join_step_budget=40)
    try:
        t1 = srv.submit(heavy)
        with pytest.raises(sb.SigmoError) as ei:
            srv.wait(t1)
        assert ei.value.code == TIMEOUT
        srv.release(t1)
        t2 = srv.submit(light)
        srv.wait(t2)
        _, total = srv.query_totals(t2, light.num_graphs)
        srv.release(t2)
    finally:
        srv.close()
    ref = oracle.run_pipeline(light, d, 3, oracle.REF_PTX, False)
    want = np.zeros(light.num_graphs, np.uint64)
    np.add.at(want, ref["indices"].astype(np.int64), ref["per_pair"])
    assert want.sum() > 0 and np.array_equal(total, want)
