"""The driver's text report, read by the reference's own log parser.

The committed reports (tests/golden/cli_*.out / .err, written on a GPU by
tests/golden/make_cli_reports.py) are parsed by the reference's
scripts/utils/output_analyzer.py (SIGMOOutputAnalyzer, imported from the
reference tree when it is present) and by tests/cli_report.py, which restates
its rules; the two must agree key by key, and the counts must be the oracle's
for the same seeded inputs: graph and vertex counts, the per-query-vertex
candidate counts and their total / average / median / zero count, refinement
steps and matches."""
import importlib.util
import json
from pathlib import Path

import pytest

import oracle
from cli_report import expected_from_oracle, parse_report

GOLDEN = Path(__file__).resolve().parent / "golden"
ANALYZER = Path("/root/reference/scripts/utils/output_analyzer.py")
SPEC = json.loads((GOLDEN / "cli_inputs.json").read_text())
KEYS = ("n_query_nodes", "n_query_graphs", "n_data_nodes", "n_data_graphs", "find_all", "join_work_group_size",
        "n_total_candidates", "n_avg_candidates", "n_median_candidates", "n_zero_candidates", "n_matches",
        "candidates_sizes")


@pytest.fixture(scope="module")
def expected():
    from oracle import workload

    m, qq, R = SPEC["inputs"]["molecules"], SPEC["inputs"]["queries"], SPEC["inputs"]["iterations"]
    d = workload.generate_molecules(m[0], m[1], m[2], seed=m[3])
    q = workload.generate_queries(qq[0], qq[1], qq[2], seed=qq[3])
    out = {}
    for ff in (False, True):
        ref = oracle.run_pipeline(q, d, R, oracle.REF_PTX, ff)
        out[not ff] = expected_from_oracle(q, d, ref["bits"], ref["total"], R, not ff)
    return out


def _report(name):
    return (GOLDEN / f"cli_{name}.out").read_text(), (GOLDEN / f"cli_{name}.err").read_text()


@pytest.mark.parametrize("name", sorted(SPEC["runs"]))
def test_report_matches_the_oracle(name, expected):
    out, err = _report(name)
    got = parse_report(out, err)
    want = expected["--find-all" in SPEC["runs"][name]]
    for k in KEYS:
        assert got[k] == want[k], (name, k)
    # the stage-per-launch form prints one line per refinement step
    assert got["n_refinement_steps"] == (0 if "--batched" in SPEC["runs"][name] else want["n_refinement_steps"])
    for k in ("graph_data_memory", "candidates_memory", "total_memory", "total_gpu_time", "total_time"):
        assert k in got, (name, k)


@pytest.mark.skipif(not ANALYZER.exists(), reason="the reference tree is not present on this machine")
@pytest.mark.parametrize("name", sorted(SPEC["runs"]))
def test_reference_parser_reads_the_report(name):
    spec = importlib.util.spec_from_file_location("sigmo_output_analyzer", ANALYZER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out, err = _report(name)
    ref = mod.SIGMOOutputAnalyzer(out, err)
    mine = parse_report(out, err)
    fields = {k: v for k, v in vars(ref).items() if not k.startswith("_")}
    assert set(fields) <= set(mine), set(fields) - set(mine)
    for k, v in fields.items():
        assert mine[k] == v, (name, k, mine[k], v)
