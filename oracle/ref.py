"""Runs the reference's own hot-path code on the host (oracle/_ref/ref_pipeline,
built by oracle/ref_build.py) — TEST INFRASTRUCTURE, the checker of the
oracle's restatement.  Only the tests import it.
"""
from __future__ import annotations

import subprocess
import tempfile
from pathlib import Path

import numpy as np

from . import ref_build

_DT = {1: np.uint8, 4: np.uint32, 8: np.uint64}


def read_dump(path: Path) -> dict:
    out = {}
    raw = path.read_bytes()
    pos = 0
    while pos < len(raw):
        nl = int(np.frombuffer(raw, np.uint32, 1, pos)[0])
        pos += 4
        name = raw[pos:pos + nl].decode()
        pos += nl
        es = int(np.frombuffer(raw, np.uint32, 1, pos)[0])
        pos += 4
        n = int(np.frombuffer(raw, np.uint64, 1, pos)[0])
        pos += 8
        out[name] = np.frombuffer(raw, _DT[es], n, pos).copy()
        pos += es * n
    return out


def run(query_text: str, data_text: str, iterations: int, join_wg: int = 128, timeout: float = 600) -> dict:
    """The reference driver's stages on two text batches: per iteration r the
    data / query signatures and the candidate bitset ([query vertex][words]),
    the GMCR, and the find-all / find-first totals."""
    exe = ref_build.build()
    with tempfile.TemporaryDirectory() as t:
        tp = Path(t)
        (tp / "q.dat").write_text(query_text)
        (tp / "d.dat").write_text(data_text)
        res = subprocess.run([str(exe), str(tp / "q.dat"), str(tp / "d.dat"), str(iterations), str(join_wg), str(tp / "out.bin")],
                             capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"reference run failed ({res.returncode}): {res.stderr[-2000:]}")
        d = read_dump(tp / "out.bin")
    nq = len(d["sig_query_0"])
    out = {"sig_data": [], "sig_query": [], "bitsets": []}
    for r in range(iterations + 1):
        out["sig_data"].append(d[f"sig_data_{r}"])
        out["sig_query"].append(d[f"sig_query_{r}"])
        bits = d[f"bits_{r}"]
        out["bitsets"].append(bits.reshape(nq, -1) if nq else bits.reshape(0, 0))
    out.update(offsets=d["gmcr_offsets"], indices=d["gmcr_indices"], total_all=int(d["total_all"][0]),
               total_first=int(d["total_first"][0]))
    return out
