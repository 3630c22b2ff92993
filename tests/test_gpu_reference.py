"""The device against the reference's own outputs.

tests/golden/ref_golden.json holds what SIGMo's own hot-path code computes
(library/include/*.hpp, built for the host by oracle/ref_build.py and run by
tests/golden/make_ref_golden.py) on seeded inputs: signature and candidate
bitset digests after the filter and after every refinement, the GMCR, and the
find-all / find-first totals.  The host build takes over-wide shift counts
modulo the register width; the stage-per-launch form run under the REF_X86
profile must reproduce every one of those values bit for bit.  (The device's
default REF_PTX profile differs from REF_X86 only in that shift rule and is
checked against the oracle, which tests/test_ref_cpu.py pins to the same
reference outputs.)"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
import sigmo_b200 as sb

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "ref_golden.json").read_text())


def _u64_digest(a):
    if a.size == 0:
        return 0
    return oracle.digest(np.ascontiguousarray(a, dtype=np.uint64).view(np.uint32).reshape(1, -1))


@pytest.mark.parametrize("name", sorted(GOLDEN["cases"]))
def test_plain_form_reproduces_the_reference(name):
    c = GOLDEN["cases"][name]
    m, qq = c["molecules"], c["queries"]
    d = sb.generate_molecules(m[0], m[1], m[2], seed=m[3], kind=m[4])
    q = sb.generate_queries(qq[0], qq[1], qq[2], seed=qq[3], kind=qq[4])
    R, wg = c["iterations"], c["join_work_group_size"]
    queue = sb.Queue(0, profile="ref-x86", join_work_group_size=wg)
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
    sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
    sig.generateDataSignatures(dg)
    sig.generateQuerySignatures(qg)
    sb.filterCandidates(queue, qg, dg, sig, cand)
    for r in range(R + 1):
        if r:
            sig.refineDataSignatures(dg, r)
            sig.refineQuerySignatures(qg, r)
            sb.refineCandidates(queue, qg, dg, sig, cand)
        assert _u64_digest(sig.getDataSignatures()) == c["sig_data"][r], (name, "data signatures", r)
        assert _u64_digest(sig.getQuerySignatures()) == c["sig_query"][r], (name, "query signatures", r)
        assert cand.digest() == c["bitsets"][r], (name, "bitset", r)
    gm = sb.GMCR(queue)
    gm.generateGMCR(qg, dg, cand)
    off, idx = gm.getGMCR()
    assert off.tolist() == c["offsets"] and idx.tolist() == c["indices"], name
    for ff, key in ((False, "total_all"), (True, "total_first")):
        nm = np.zeros(1, np.uint64)
        sb.joinCandidates(queue, qg, dg, cand, gm, nm, ff)
        assert int(nm[0]) == c[key], (name, key)


def test_batched_form_refuses_ref_x86():
    d = sb.generate_molecules(50, 10, 30, seed=5)
    q = sb.generate_queries(5, 3, 8, seed=6)
    queue = sb.Queue(0, profile="ref-x86")
    qg, dg = sb.createDeviceCSRGraph(queue, q), sb.createDeviceCSRGraph(queue, d)
    with pytest.raises(sb.SigmoError) as ei:
        sb.match_batched(queue, qg, dg, 3, False, None, sb.GMCR(queue))
    assert ei.value.code == 4


def test_ptx_shift_instructions_clamp(tmp_path):
    """REF_PTX rests on one hardware fact: the PTX shift instructions that the
    reference's over-wide shifts become on an NVIDIA GPU (shr.u32 / shl.b32 in
    the range masks, candidates.hpp:91-99; shl.b64 in the Bitset,
    utils.hpp:71-73) give 0 for a run-time count >= the register width, where
    x86-64 takes the count modulo the width.  This runs those instructions on
    the device (tests/ptx_shift_probe.cu, built here with nvcc)."""
    import shutil
    import subprocess

    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "ptx_shift_probe"
    src = Path(__file__).resolve().parent / "ptx_shift_probe.cu"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = [tuple(int(x) for x in line.split()) for line in out if line.strip()]
    assert len(rows) == 12
    m32 = 0xFFFFFFFF
    for n, shr, shl, shl64 in rows:
        assert shr == (m32 >> n if n < 32 else 0), n
        assert shl == ((m32 << n) & m32 if n < 32 else 0), n
        assert shl64 == (1 << n if n < 64 else 0), n
    # the x86-64 reading differs exactly where the counts are over-wide
    assert any(n >= 32 and shr != m32 >> (n & 31) for n, shr, _, _ in rows)
