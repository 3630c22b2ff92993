"""Writes tests/golden/ref_golden.json: outputs of the reference's own code.

Runs SIGMo's hot path (library/include/*.hpp, built for the host by
oracle/ref_build.py with the SYCL stand-in oracle/sycl_host) on seeded
synthetic inputs and keeps, per case: the digest of the data and query
signatures and of the candidate bitset after the filter and after every
refinement, the GMCR offsets and indices, and the find-all and find-first
totals.  The host build follows x86-64 shift semantics, so these are the
oracle's REF_X86 profile values; tests/test_ref_cpu.py checks the oracle
against them on any machine, and against a live build of the reference where
the reference tree is present.

    python tests/golden/make_ref_golden.py     (needs the reference tree)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

# name: (molecules (count, min, max, seed, kind), queries (count, min, max, seed, kind), iterations, join work-group size)
CASES = {
    "drug1k_R6": ((1000, 10, 40, 1001, 0), (20, 4, 12, 1002, 0), 6, 128),
    "drug300_R0": ((300, 10, 40, 2101, 0), (15, 3, 10, 2102, 0), 0, 128),
    "drug300_R1_wg32": ((300, 10, 40, 2201, 0), (40, 3, 8, 2202, 0), 1, 32),
    "drug400_R3_wg256": ((400, 10, 60, 2301, 0), (30, 3, 14, 2302, 0), 3, 256),
    "uneven_R4": ((300, 6, 120, 2401, 1), (25, 3, 12, 2402, 0), 4, 128),
    "rings_R3": ((150, 12, 50, 2501, 2), (12, 4, 10, 2502, 3), 3, 64),
}


def inputs(case):
    from oracle import workload

    m, q, R, wg = case
    d = workload.generate_molecules(m[0], m[1], m[2], seed=m[3], kind=m[4])
    qq = workload.generate_queries(q[0], q[1], q[2], seed=q[3], kind=q[4])
    return qq, d, R, wg


def digest_u64(a: np.ndarray) -> int:
    """Order-dependent digest of a u64 vector (signatures)."""
    import oracle

    if a.size == 0:
        return 0
    return oracle.digest(a.astype(np.uint64).view(np.uint32).reshape(1, -1))


def main():
    import oracle
    from oracle import ref, workload

    out = {"generator": "oracle/libsigmo_workload.so (the product's seeded generator)", "cases": {}}
    for name, case in CASES.items():
        q, d, R, wg = inputs(case)
        r = ref.run(workload.format_text(q), workload.format_text(d), R, wg)
        out["cases"][name] = {
            "molecules": list(case[0]), "queries": list(case[1]), "iterations": R, "join_work_group_size": wg,
            "sig_data": [digest_u64(x) for x in r["sig_data"]],
            "sig_query": [digest_u64(x) for x in r["sig_query"]],
            "bitsets": [oracle.digest(x) for x in r["bitsets"]],
            "offsets": r["offsets"].tolist(), "indices": r["indices"].tolist(),
            "total_all": r["total_all"], "total_first": r["total_first"],
        }
        print(name, len(r["indices"]), r["total_all"], r["total_first"])
    (HERE / "ref_golden.json").write_text(json.dumps(out) + "\n")


if __name__ == "__main__":
    main()
