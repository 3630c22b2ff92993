"""Reader of the sigmo driver's text report — TEST INFRASTRUCTURE.

Restates the parse rules of the reference's log parser
(scripts/utils/output_analyzer.py:5-111, class SIGMOOutputAnalyzer): the
same keys, taken from the same lines of stdout, and the per-query-vertex
candidate counts from the "Node i: c" lines of stderr.  tests/
test_cli_report_cpu.py checks this reader against the reference's own parser
on committed reports (when the reference is present); the GPU test of the CLI
then reads the driver's live output with it.
"""
from __future__ import annotations

_UNITS = {"B": 1, "KB": 1024, "MB": 1024 ** 2, "GB": 1024 ** 3}


def _dotted(s: str) -> int:
    """formatNumber's dot-separated thousands (library/src/utils.hpp:127-138)."""
    return int(s.replace(".", ""))


def _last_int_before_unit(line: str) -> int:
    return int(line.split(" ")[-2])


def parse_report(out: str, err: str = "") -> dict:
    r: dict = {"n_refinement_steps": 0}
    if err:
        r["candidates_sizes"] = [int(l.split(" ")[-1]) for l in err.split("\n") if l.startswith("Node")]
    lines = [l.strip() for l in out.split("\n")]
    section = None
    for line in lines:
        if line.startswith("-------------"):
            section = line.strip("- ")
            continue
        words = line.split(" ")
        if line.startswith("# Query Nodes"):
            r["n_query_nodes"] = int(words[-1])
        elif line.startswith("# Query Graphs"):
            r["n_query_graphs"] = int(words[-1])
        elif line.startswith("# Data Nodes"):
            r["n_data_nodes"] = int(words[-1])
        elif line.startswith("# Data Graphs"):
            r["n_data_graphs"] = int(words[-1])
        elif section == "Configs" and line.startswith("Filter domain"):
            r["filter_domain"] = words[-1]
        elif section == "Configs" and line.startswith("Filter Work Group Size"):
            r["filter_work_group_size"] = int(words[-1])
        elif section == "Configs" and line.startswith("Join Work Group Size"):
            r["join_work_group_size"] = int(words[-1])
        elif section == "Configs" and line.startswith("Find all"):
            r["find_all"] = words[-1] == "Yes"
        elif line.startswith("Allocated ") and line.endswith(" for graph data"):
            r["graph_data_memory"] = float(words[1]) * _UNITS[words[2]]
        elif line.startswith("Allocated ") and line.endswith(" for query data"):
            r["query_data_memory"] = float(words[1]) * _UNITS[words[2]]
        elif line.startswith("Allocated ") and line.endswith(" for candidates"):
            r["candidates_memory"] = float(words[1]) * _UNITS[words[2]]
        elif line.startswith("Allocated ") and line.endswith(" for data signatures"):
            r["data_signatures_memory"] = float(words[1]) * _UNITS[words[2]]
        elif line.startswith("Allocated ") and line.endswith(" for query signatures"):
            r["query_signatures_memory"] = float(words[1]) * _UNITS[words[2]]
        elif line.startswith("Total allocated memory"):
            r["total_memory"] = float(words[3]) * _UNITS[words[4]]
        elif line.startswith("# Total candidates:"):
            r["n_total_candidates"] = _dotted(words[-1])
        elif line.startswith("# Average candidates:"):
            r["n_avg_candidates"] = _dotted(words[-1])
        elif line.startswith("# Median candidates:"):
            r["n_median_candidates"] = _dotted(words[-1])
        elif line.startswith("# Zero candidates:"):
            r["n_zero_candidates"] = _dotted(words[-1])
        elif line.startswith("# Matches:"):
            r["n_matches"] = _dotted(words[-1])
        elif line.startswith("[*] Refinement step"):
            r["n_refinement_steps"] = int(words[-1].rstrip(":"))
        elif section == "Overall GPU Stats" and line.endswith(" ms"):
            key = {"Data signature time:": "data_signature_gpu_time", "Query signature time:": "query_signature_gpu_time",
                   "Filter time:": "filter_gpu_time", "Join time:": "join_gpu_time", "Total time:": "total_gpu_time"}
            for prefix, k in key.items():
                if line.startswith(prefix):
                    r[k] = _last_int_before_unit(line)
        elif section == "Overall Host Stats":
            if line.startswith("Setup Data time"):
                r["setup_data_host_time"] = int(words[3])
            elif line.endswith(" ms"):
                key = {"Filter time:": "filter_host_time", "Mapping time:": "mapping_host_time",
                       "Join time:": "join_host_time", "Total time:": "total_time"}
                for prefix, k in key.items():
                    if line.startswith(prefix):
                        r[k] = _last_int_before_unit(line)
    return r


def expected_from_oracle(q, d, bits, total_matches: int, iterations: int, find_all: bool, wg: int = 128) -> dict:
    """The report values the oracle predicts for a plain run (counts of the
    final bitset rows, CandidatesInspector's total / avg / median / zeros,
    library/src/utils.hpp:159-178)."""
    import numpy as np

    sizes = np.unpackbits(np.ascontiguousarray(bits).view(np.uint8), axis=1).sum(axis=1).astype(np.int64) \
        if bits.size else np.zeros(0, np.int64)
    srt = np.sort(sizes)
    total = int(sizes.sum())
    return {
        "n_query_nodes": int(q.total_nodes), "n_query_graphs": int(q.num_graphs), "n_data_nodes": int(d.total_nodes),
        "n_data_graphs": int(d.num_graphs), "find_all": find_all, "join_work_group_size": wg,
        "n_total_candidates": total, "n_avg_candidates": total // max(1, len(sizes)),
        "n_median_candidates": int(srt[len(srt) // 2]) if len(srt) else 0,
        "n_zero_candidates": int((sizes == 0).sum()), "n_matches": int(total_matches),
        "n_refinement_steps": iterations, "candidates_sizes": [int(x) for x in sizes],
    }
