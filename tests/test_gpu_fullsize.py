"""Bit-exactness at the benchmark workloads' own sizes.

* 100,000 drug-like molecules (10-60 atoms) x 600 queries (3-30 atoms), 6
  refinement iterations -- the bench workload in full: the stage-per-launch
  form's candidate bitset digest after the filter and after every refinement,
  GMCR offsets and indices, and per-pair counts in find-all and find-first;
  the batched form (ordinary calls and CUDA-graph replays) in both modes.
* The first 20,000 molecules of the 1,000,000-molecule uneven workload (6-120
  atoms, lognormal, macrocycles) x all 2,000 queries of 3-40 atoms: bitset
  digests, GMCR and per-pair counts, both modes, both forms.
* The first 20,000 molecules of the 2,000,000-molecule ring-rich workload x all
  300 automorphic queries: GMCR and find-first flags on the whole slice, and
  find-all counts (up to ~10^5 per pair) on every slot of the molecules below
  vertex 256 plus a seeded sample of 40,000 other slots.

The generator seeds every graph from (seed, kind, index), so the first k
molecules of a workload are the same graphs at any workload size.  Every check
is against the oracle (REF_PTX); pairs outside the reference's defined domain
(queries of >= 30 vertices, molecules of > 64 atoms) are counted and checked
like the rest, with the oracle's semantics.
"""
import numpy as np
import pytest

import oracle
import sigmo_b200 as sb

pytestmark = pytest.mark.gpu

DRUG100K = dict(lo=10, hi=60, kind=0, median=22.0, seed_d=20251, queries=600, qlo=3, qhi=30, qkind=0, skew=(6, 15),
                seed_q=20252)
UNEVEN1M = dict(lo=6, hi=120, kind=1, median=22.0, seed_d=30301, queries=2000, qlo=3, qhi=40, qkind=0, skew=(0, 0),
                seed_q=30302)
SYMMETRY2M = dict(lo=10, hi=64, kind=2, median=22.0, seed_d=50501, queries=300, qlo=4, qhi=14, qkind=3, skew=(0, 0),
                  seed_q=50502)
R = 6


def _inputs(wl, mols):
    d = sb.generate_molecules(mols, wl["lo"], wl["hi"], seed=wl["seed_d"], kind=wl["kind"], median=wl["median"])
    q = sb.generate_queries(wl["queries"], wl["qlo"], wl["qhi"], seed=wl["seed_q"], kind=wl["qkind"],
                            skew_lo=wl["skew"][0], skew_hi=wl["skew"][1])
    return q, d


def _all_threads():
    import os

    oracle.lib().orc_set_num_threads(max(1, len(os.sched_getaffinity(0))))


def _oracle_filter(q, d):
    """Signatures, filter, R refinements (a digest after each) and GMCR."""
    _all_threads()
    out = oracle.run_pipeline(q, d, R, oracle.REF_PTX, skip_join=True, digests=True)
    off, idx = oracle.gmcr(q, d, out["bits"], oracle.REF_PTX)
    return out["bits"], out["digests"], off, idx


def _out_of_domain(q, d, off, idx):
    qs = np.diff(np.asarray(q.graph_offsets, dtype=np.int64))
    ds = np.diff(np.asarray(d.graph_offsets, dtype=np.int64))
    g = np.repeat(np.arange(len(ds)), np.diff(off.astype(np.int64)))
    return int(((qs[idx.astype(np.int64)] >= 30) | (ds[g] > 64)).sum())


def _plain(queue, qg, dg):
    """The stage-per-launch form with the bitset digest after every stage."""
    cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
    sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
    sig.generateDataSignatures(dg)
    sig.generateQuerySignatures(qg)
    sb.filterCandidates(queue, qg, dg, sig, cand)
    digests = [cand.digest()]
    for r in range(1, R + 1):
        sig.refineDataSignatures(dg, r)
        sig.refineQuerySignatures(qg, r)
        sb.refineCandidates(queue, qg, dg, sig, cand)
        digests.append(cand.digest())
    gm = sb.GMCR(queue)
    gm.generateGMCR(qg, dg, cand)
    return cand, sig, gm, digests


def _plain_join(queue, qg, dg, cand, gm, ff):
    nm = np.zeros(1, np.uint64)
    _, per = sb.joinCandidates(queue, qg, dg, cand, gm, nm, ff, per_pair=True)
    return int(nm[0]), per


def _check_gmcr(gm, off, idx, ctx):
    o, i = gm.getGMCR()
    assert np.array_equal(o, off), f"{ctx}: GMCR offsets differ"
    assert np.array_equal(i, idx), f"{ctx}: GMCR indices differ"


def _check_forms(q, d, digests, off, idx, want, ctx, plain=True):
    """Both forms against the oracle: want = {find_first: (total, per_pair)}."""
    queue = sb.Queue(0)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    if plain:
        cand, sig, gm, dig = _plain(queue, qg, dg)
        assert dig == digests, f"{ctx}: plain-form bitset digests after iterations 0..{R} differ"
        _check_gmcr(gm, off, idx, f"{ctx} plain")
        for ff, (total, per) in want.items():
            t, p = _plain_join(queue, qg, dg, cand, gm, ff)
            assert t == total and np.array_equal(p, per), f"{ctx}: plain join, find_first={ff}"
        sig.close()
        cand.close()
        gm.close()
    for ff, (total, per) in want.items():
        gm = sb.GMCR(queue)
        res = sb.match_batched(queue, qg, dg, R, ff, None, gm)
        _check_gmcr(gm, off, idx, f"{ctx} batched ff={ff}")
        assert res["total_matches"] == total and np.array_equal(gm.getPairCounts(), per), f"{ctx}: batched ff={ff}"
        for rep in range(2):  # capture, then replay
            res = sb.match_batched(queue, qg, dg, R, ff, None, gm, graph=True)
            assert res["total_matches"] == total and np.array_equal(gm.getPairCounts(), per), \
                f"{ctx}: graph replay {rep} ff={ff}"
        gm.close()


def test_drug100k_full_size_bit_exact():
    q, d = _inputs(DRUG100K, 100_000)
    assert d.num_graphs * q.num_graphs == 60_000_000
    bits, digests, off, idx = _oracle_filter(q, d)
    want = {ff: oracle.join(q, d, bits, off, idx, oracle.REF_PTX, ff) for ff in (False, True)}
    del bits
    assert want[False][0] > 0 and len(idx) > 1_000_000
    ood = _out_of_domain(q, d, off, idx)
    print(f"drug100k: {len(idx)} admitted pairs, {want[False][0]} matches, {ood} admitted pairs out of domain")
    _check_forms(q, d, digests, off, idx, want, "drug100k")


def test_uneven1m_slice_bit_exact():
    q, d = _inputs(UNEVEN1M, 20_000)
    assert int(d.sizes().max()) > 64 and int(q.sizes().max()) >= 30
    bits, digests, off, idx = _oracle_filter(q, d)
    want = {ff: oracle.join(q, d, bits, off, idx, oracle.REF_PTX, ff) for ff in (False, True)}
    del bits
    ood = _out_of_domain(q, d, off, idx)
    assert ood > 0  # the out-of-domain class is exercised
    print(f"uneven1m slice: {len(idx)} admitted pairs, {want[False][0]} matches, {ood} admitted pairs out of domain")
    _check_forms(q, d, digests, off, idx, want, "uneven1m[:20000]")


def test_symmetry2m_slice_bit_exact():
    q, d = _inputs(SYMMETRY2M, 20_000)
    bits, digests, off, idx = _oracle_filter(q, d)
    total_ff, per_ff = oracle.join(q, d, bits, off, idx, oracle.REF_PTX, True)
    # find-all on a sub-GMCR: every slot of the molecules below vertex 256 (where
    # the reference's visited bitset is live and a work-item carries mapping[]
    # across its slots, so their segments stay whole) plus a seeded sample of
    # other slots, whose counts do not depend on which slots share a work-item
    goff = np.asarray(d.graph_offsets, dtype=np.int64)
    seg = np.diff(off.astype(np.int64))
    slot_graph = np.repeat(np.arange(d.num_graphs), seg)
    low = goff[slot_graph] < 256
    rng = np.random.default_rng(515)
    others = np.flatnonzero(~low)
    keep = np.zeros(len(idx), bool)
    keep[low] = True
    keep[rng.choice(others, size=min(40_000, len(others)), replace=False)] = True
    sub_off = np.zeros(d.num_graphs + 1, np.uint32)
    sub_off[1:] = np.cumsum(np.bincount(slot_graph[keep], minlength=d.num_graphs))
    sub_tot, sub_per = oracle.join(q, d, bits, sub_off, idx[keep], oracle.REF_PTX, False)
    del bits
    assert sub_per.max() >= 1000  # automorphic patterns: thousands of embeddings per pair
    print(f"symmetry2m slice: {len(idx)} admitted pairs, find-all checked on {int(keep.sum())} slots "
          f"(max {int(sub_per.max())} embeddings per pair)")

    queue = sb.Queue(0)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    cand, sig, gm, dig = _plain(queue, qg, dg)
    assert dig == digests, "plain-form bitset digests differ"
    _check_gmcr(gm, off, idx, "plain")
    t, p = _plain_join(queue, qg, dg, cand, gm, True)
    assert t == total_ff and np.array_equal(p, per_ff), "plain find-first"
    t, p = _plain_join(queue, qg, dg, cand, gm, False)
    assert np.array_equal(p[keep], sub_per), "plain find-all (sampled slots)"
    for ff in (True, False):
        g2 = sb.GMCR(queue)
        res = sb.match_batched(queue, qg, dg, R, ff, None, g2)
        _check_gmcr(g2, off, idx, f"batched ff={ff}")
        got = g2.getPairCounts()
        if ff:
            assert res["total_matches"] == total_ff and np.array_equal(got, per_ff), "batched find-first"
        else:
            assert np.array_equal(got[keep], sub_per), "batched find-all (sampled slots)"
            assert res["total_matches"] == t, "batched find-all total differs from the plain form's"
