"""The oracle against the reference's own code.

SIGMo's hot path (library/include/*.hpp) is compiled for the host by
oracle/ref_build.py (g++ with the SYCL stand-in oracle/sycl_host; the only
edit is a syntactic rewrite of four class-scope specialisations that g++
rejects) and run on seeded inputs.  Its signatures and candidate bitsets after
the filter and after every refinement, its GMCR and its find-all / find-first
totals must equal the oracle's REF_X86 profile (the host build follows x86-64
shift semantics).  The REF_PTX profile the device implements differs from
REF_X86 only in the shift helpers of the oracle (an over-wide shift gives 0
instead of using the count modulo the width).

* test_oracle_matches_reference_golden: against tests/golden/ref_golden.json
  (reference outputs committed by tests/golden/make_ref_golden.py), on any machine;
* the other tests rebuild and run the reference itself where its tree is present.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import ref_build, workload

GOLDEN = Path(__file__).resolve().parent / "golden"
REF_TESTDATA = Path("/root/reference/library/test/data")
needs_reference = pytest.mark.skipif(not ref_build.available(), reason="the reference tree is not present on this machine")


def _u64_digest(a):
    if a.size == 0:
        return 0
    return oracle.digest(np.ascontiguousarray(a, dtype=np.uint64).view(np.uint32).reshape(1, -1))


def _inputs(m, q):
    d = workload.generate_molecules(m[0], m[1], m[2], seed=m[3], kind=m[4])
    qq = workload.generate_queries(q[0], q[1], q[2], seed=q[3], kind=q[4])
    return qq, d


@pytest.fixture(scope="module")
def golden():
    return json.loads((GOLDEN / "ref_golden.json").read_text())


def test_oracle_matches_reference_golden(golden):
    assert len(golden["cases"]) >= 6
    for name, c in golden["cases"].items():
        q, d = _inputs(c["molecules"], c["queries"])
        R, wg = c["iterations"], c["join_work_group_size"]
        o = oracle.run_pipeline(q, d, R, oracle.REF_X86, False, wg=wg, keep=True)
        for it in range(R + 1):
            assert _u64_digest(o["sig_data"][it]) == c["sig_data"][it], (name, "data signatures", it)
            assert _u64_digest(o["sig_query"][it]) == c["sig_query"][it], (name, "query signatures", it)
            assert oracle.digest(o["bitsets"][it]) == c["bitsets"][it], (name, "bitset", it)
        assert o["offsets"].tolist() == c["offsets"] and o["indices"].tolist() == c["indices"], name
        assert o["total"] == c["total_all"], name
        assert oracle.run_pipeline(q, d, R, oracle.REF_X86, True, wg=wg)["total"] == c["total_first"], name


def _compare_live(q_text, d_text, R, wg=128):
    from oracle import ref

    r = ref.run(q_text, d_text, R, wg)
    q, d = oracle.parse_text(q_text), oracle.parse_text(d_text)
    o = oracle.run_pipeline(q, d, R, oracle.REF_X86, False, wg=wg, keep=True)
    for it in range(R + 1):
        assert np.array_equal(o["sig_data"][it], r["sig_data"][it]), ("data signatures", it)
        assert np.array_equal(o["sig_query"][it], r["sig_query"][it]), ("query signatures", it)
        assert np.array_equal(o["bitsets"][it], r["bitsets"][it]), ("bitset", it)
    assert np.array_equal(o["offsets"], r["offsets"]) and np.array_equal(o["indices"], r["indices"])
    assert o["total"] == r["total_all"]
    assert oracle.run_pipeline(q, d, R, oracle.REF_X86, True, wg=wg)["total"] == r["total_first"]
    return r


@needs_reference
def test_patch_rewrites_only_the_four_specialisations():
    """The only edit: four `template<> ... refineXSignatures<Algorithm::Y>(`
    heads become constrained overloads, and the two primary declarations they
    specialised go; every other line is unchanged."""
    import difflib

    src = (ref_build.REF_INCLUDE / "signature.hpp").read_text().splitlines()
    out = ref_build.patch_signature_header("\n".join(src)).splitlines()
    removed, added = [], []
    for line in difflib.ndiff(src, out):
        if line.startswith("- "):
            removed.append(line[2:].strip())
        elif line.startswith("+ "):
            added.append(line[2:].strip())
    assert removed.count("template<>") == 4
    assert sum(l.startswith("template<Algorithm _A = A> requires (_A == Algorithm::") for l in added) == 4
    heads = [l for l in removed if l.startswith("utils::BatchedEvent refine")]
    assert len(heads) == 6  # four specialised heads + two primary declarations
    assert len(added) == 8  # four constrained template heads + four heads without the <Algorithm::Y>
    for a in added:
        assert a.startswith("template<Algorithm _A = A> requires") or a.startswith("utils::BatchedEvent refine"), a


@needs_reference
def test_reference_fixture_files():
    """library/test/data/test_query.dat x test_data.dat, the reference's own
    test inputs, 0-3 refinements."""
    q_text = (REF_TESTDATA / "test_query.dat").read_text()
    d_text = (REF_TESTDATA / "test_data.dat").read_text()
    for R in (0, 1, 3):
        _compare_live(q_text, d_text, R)


@needs_reference
@pytest.mark.parametrize("wg", [32, 128])
def test_live_reference_on_fresh_seeds(wg):
    q, d = _inputs((250, 8, 36, 7301 + wg, 0), (24, 3, 9, 7302 + wg, 0))
    r = _compare_live(workload.format_text(q), workload.format_text(d), 4, wg)
    assert r["total_all"] > 0


@needs_reference
def test_live_reference_edge_cases():
    """A graph ending on a 32-vertex word boundary (the range-mask shift of
    candidates.hpp:98), wildcard query labels (isomorphism.hpp:49), labels >= 16
    (ignored by signatures), a data graph without edges."""
    lines = ["n#20 l#1 " + " ".join(f"{i} 8" for i in range(20)) + " e#19 " + " ".join(f"{i} {i+1} 1" for i in range(19)),
             "n#44 l#1 " + " ".join(f"{i} 8" for i in range(44)) + " e#43 " + " ".join(f"{i} {i+1} 1" for i in range(43)),
             "n#5 l#3 0 8 1 8 2 20 3 7 4 8 e#4 0 1 1 1 2 1 2 3 1 3 4 1",
             "n#3 l#1 0 8 1 8 2 8 e#0"]
    d_text = "\n".join(lines) + "\n"
    q_text = "n#3 l#1 0 8 1 8 2 8 e#2 0 1 1 1 2 1\nn#3 l#2 0 255 1 8 2 20 e#2 0 1 1 1 2 1\nn#2 l#1 0 8 1 7 e#1 0 1 1\n"
    for R in (0, 2):
        _compare_live(q_text, d_text, R)
