"""Generates tests/golden/golden.json: inputs and expected outputs of the hot
path, computed by the independent pure-Python restatement (tests/pyref.py).

Inputs:
  * the reference's own test fixtures (library/test/data/test_data.dat and
    test_query.dat, read from the reference checkout given by --reference);
  * a small seeded synthetic set from sigmo_b200's generator;
  * hand-built edge cases for the reference's shift/indexing hazards (a data
    graph ending on a 32-vertex boundary, a graph larger than 64 vertices, a
    data graph starting beyond vertex 256, a self-loop, wildcard and >=16
    labels, a 1-vertex query).

Run from the repository root:  python tests/golden/make_golden.py --reference <path>
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

import pyref  # noqa: E402
from oracle import parse_text  # noqa: E402  (pure-Python text restatement)


def line(n, labels, edges):
    s = f"n#{n} l#11 " + " ".join(f"{i} {labels[i]}" for i in range(n)) + f" e#{len(edges)} "
    s += " ".join(f"{u} {v} {l}" for u, v, l in edges)
    return s


def chain(n, lab=8):
    return line(n, [lab] * n, [(i, i + 1, 1) for i in range(n - 1)])


def ring(n, lab=8):
    return line(n, [lab] * n, [(i, (i + 1) % n, 4) for i in range(n)])


def edge_cases():
    data = []
    # graph 0: 20 vertices (ring of 6 + tail), graph 1: 44 vertices -> ends at 64
    data.append(line(20, [8] * 6 + [7, 0] + [8] * 12, [(i, (i + 1) % 6, 4) for i in range(6)] + [(5, 6, 1), (6, 7, 1)] +
                     [(7 + k, 8 + k, 1) for k in range(12)]))
    data.append(line(44, [8] * 40 + [7, 7, 0, 9], [(i, i + 1, 1) for i in range(43)] + [(0, 5, 1), (10, 15, 1)]))
    # graph 2: 70-vertex chain with a ring (more than 64 vertices)
    data.append(line(70, [8] * 68 + [7, 0], [(i, i + 1, 1) for i in range(69)] + [(0, 5, 1)]))
    # graph 3: self-loop and labels >= 16 / wildcard-labelled data vertex
    data.append(line(6, [8, 8, 20, 255, 7, 8], [(0, 1, 1), (1, 2, 1), (2, 3, 1), (3, 4, 1), (4, 5, 1), (1, 1, 1)]))
    # filler so the next graphs start past vertex 256
    for _ in range(8):
        data.append(ring(6))
        data.append(chain(18))
    data.append(ring(6))
    data.append(line(12, [8] * 6 + [7, 8, 8, 0, 8, 8], [(i, (i + 1) % 6, 4) for i in range(6)] + [(0, 6, 1), (6, 7, 1),
                     (7, 8, 1), (8, 9, 1), (9, 10, 1), (10, 11, 1)]))
    data.append(chain(9))
    queries = [
        line(3, [8, 8, 8], [(0, 1, 1), (1, 2, 1)]),            # C-C-C path
        line(3, [8, 8, 7], [(0, 1, 1), (1, 2, 1)]),            # C-C-O
        line(6, [8] * 6, [(i, (i + 1) % 6, 4) for i in range(6)]),  # 6-ring
        line(4, [255, 8, 8, 8], [(0, 1, 1), (1, 2, 1), (2, 3, 1)]),  # wildcard head
        line(1, [8], []),                                       # 1-vertex query (never admitted)
        line(4, [8, 8, 8, 8], [(0, 1, 1), (0, 2, 1), (0, 3, 1)]),  # star
    ]
    return "\n".join(queries) + "\n", "\n".join(data) + "\n"


def run_case(name, qtext, dtext, iterations_list, profiles=(0, 1, 2)):
    qb, db = parse_text(qtext), parse_text(dtext)
    runs = []
    for prof in profiles:
        for R in iterations_list:
            if prof == pyref.EXACT and max(int(x) for x in (db.graph_offsets[1:] - db.graph_offsets[:-1])) > 256:
                continue
            full = pyref.run_pipeline(qb, db, R, prof, False)
            first = pyref.run_pipeline(qb, db, R, prof, True)
            runs.append({
                "profile": prof,
                "iterations": R,
                "sig_data": full["sig_data"],
                "sig_query": full["sig_query"],
                "bitsets": [pyref.rows_to_words(r, db.total_nodes) for r in full["bitsets"]],
                "offsets": full["offsets"],
                "indices": full["indices"],
                "per_pair_all": full["per_pair"],
                "total_all": full["total"],
                "per_pair_first": first["per_pair"],
                "total_first": first["total"],
            })
    return {"name": name, "query_text": qtext, "data_text": dtext, "runs": runs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="path of the SIGMo checkout (for its test fixtures)")
    args = ap.parse_args()
    cases = []
    if args.reference:
        d = Path(args.reference) / "library" / "test" / "data"
        cases.append(run_case("reference_fixtures", (d / "test_query.dat").read_text(), (d / "test_data.dat").read_text(),
                              [0, 1, 3]))
    import sigmo_b200 as sb

    mols = sb.generate_molecules(12, 10, 30, seed=7)
    qs = sb.generate_queries(5, 3, 7, seed=11)
    cases.append(run_case("synthetic_small", qs.to_text(), mols.to_text(), [0, 2, 6]))
    qe, de = edge_cases()
    cases.append(run_case("edge_cases", qe, de, [0, 1, 4]))
    out = {"generator": "tests/golden/make_golden.py (tests/pyref.py)", "cases": cases}
    (HERE / "golden.json").write_text(json.dumps(out, separators=(",", ":")))
    print("wrote", HERE / "golden.json", sum(len(c["runs"]) for c in cases), "runs")


if __name__ == "__main__":
    main()
