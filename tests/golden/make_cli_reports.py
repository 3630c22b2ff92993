"""Writes the committed CLI report fixtures tests/golden/cli_*.out / .err.

Needs a CUDA GPU and the built driver (sigmo_b200/sigmo_cli): it runs the
driver on seeded synthetic inputs, as the reference's experiment scripts run
theirs, and keeps stdout and stderr.  tests/test_cli_report_cpu.py reads the
reports with the reference's own log parser and with tests/cli_report.py, and
checks both against the oracle.

    python tests/golden/make_cli_reports.py [output-dir]   (default: tests/golden)
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

# inputs: molecules and queries of the seeded generator, 3 refinement steps
INPUTS = {"molecules": [800, 10, 40, 4701], "queries": [25, 3, 10, 4702], "iterations": 3}
RUNS = {
    "plain_findall": ["--find-all"],
    "plain_findfirst": [],
    "batched_findall": ["--find-all", "--batched"],
}


def inputs():
    import sigmo_b200 as sb

    m, qq = INPUTS["molecules"], INPUTS["queries"]
    return sb.generate_queries(qq[0], qq[1], qq[2], seed=qq[3]), sb.generate_molecules(m[0], m[1], m[2], seed=m[3])


def run_cli(extra, q, d, tmp: Path):
    import sigmo_b200 as sb

    (tmp / "d.dat").write_text(d.to_text())
    (tmp / "q.dat").write_text(q.to_text())
    cli = Path(sb.__file__).resolve().parent / "sigmo_cli"
    cmd = [str(cli), "-Q", str(tmp / "q.dat"), "-D", str(tmp / "d.dat"), "-i", str(INPUTS["iterations"]), "-p",
           "--max-data-graphs", "1000000", "--max-query-graphs", "1000000"] + extra
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    if res.returncode != 0:
        raise RuntimeError(res.stderr)
    return res.stdout, res.stderr


def main():
    dest = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE
    dest.mkdir(parents=True, exist_ok=True)
    q, d = inputs()
    with tempfile.TemporaryDirectory() as t:
        for name, extra in RUNS.items():
            out, err = run_cli(extra, q, d, Path(t))
            (dest / f"cli_{name}.out").write_text(out)
            (dest / f"cli_{name}.err").write_text(err)
    (dest / "cli_inputs.json").write_text(json.dumps({"inputs": INPUTS, "runs": RUNS}, indent=1) + "\n")


if __name__ == "__main__":
    main()
