"""Builds oracle/_ref/ref_pipeline: the reference's own hot-path code (SIGMo's
header-only library, library/include/*.hpp) compiled with g++ for the host
CPU — TEST INFRASTRUCTURE, the checker of the oracle.

The reference is SYCL 2020 and no SYCL compiler is installed here, so:

* oracle/sycl_host/sycl/sycl.hpp stands in for <sycl/sycl.hpp> (work-items
  run on the host; work-groups as cooperative fibers, see its header);
* g++ 13 rejects the four explicit specialisations that
  library/include/signature.hpp declares inside its class template
  (lines 213, 250, 298, 336: C++ allows them only at namespace scope before
  CWG 727).  The headers are copied into oracle/_ref/include/ and those four
  are rewritten, mechanically, as overloads constrained on the same template
  argument (`template<Algorithm _A = A> requires (_A == Algorithm::X)`), and
  the two primary declarations they specialised (lines 122-123, 154-155) are
  dropped.  Nothing else in the text changes; tests/test_ref_cpu.py fails if
  a rewrite does not apply exactly once.

The driver (oracle/ref_pipeline.cpp, this project's code) runs the
reference's stage order (library/src/sigmo.cpp:98-160) on two text files and
dumps every intermediate (signatures and candidate bitset after the filter
and after each refinement, GMCR, find-all and find-first totals).

The host build follows x86-64 semantics where the reference has undefined
behaviour (an over-wide shift uses the count modulo the register width), so it
pins the oracle's REF_X86 profile; it is compiled without optimisation so that
no compiler assumption about those shifts changes what the instructions do.

    python -m oracle.ref_build       (needs the reference tree; output in oracle/_ref/)
"""
from __future__ import annotations

import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_ROOT = Path("/root/reference")
REF_INCLUDE = REF_ROOT / "library" / "include"
OUT = HERE / "_ref"
BIN = OUT / "ref_pipeline"

# (pattern, replacement): each must match exactly once in signature.hpp
_SPECIALISATIONS = [
    (r"template<>\s*\n(\s*)utils::BatchedEvent refine(AM|CSR)Signatures<Algorithm::(ViewBased|PowerGraph)>\(",
     r"template<Algorithm _A = A> requires (_A == Algorithm::\3)\n\1utils::BatchedEvent refine\2Signatures("),
]
_PRIMARY_DECLS = [
    r"\n\s*template<Algorithm _A = A>\s*\n\s*utils::BatchedEvent refineAMSignatures\(DeviceBatchedAMGraph& graphs, size_t view_size, "
    r"SignatureScope s\);",
    r"\n\s*template<Algorithm _A = A>\s*\n\s*utils::BatchedEvent refineCSRSignatures\(DeviceBatchedCSRGraph& graphs, size_t view_size, "
    r"SignatureScope s\);",
]


def patch_signature_header(text: str) -> str:
    for pat in _PRIMARY_DECLS:
        text, n = re.subn(pat, "\n", text)
        if n != 1:
            raise RuntimeError(f"signature.hpp: primary declaration pattern matched {n} times")
    pat, rep = _SPECIALISATIONS[0]
    text, n = re.subn(pat, rep, text)
    if n != 4:
        raise RuntimeError(f"signature.hpp: expected 4 class-scope specialisations, rewrote {n}")
    return text


def available() -> bool:
    return REF_INCLUDE.is_dir()


def build(force: bool = False) -> Path:
    if BIN.exists() and not force:
        return BIN
    if not available():
        raise RuntimeError("the reference tree is not present; oracle/_ref cannot be built here")
    inc = OUT / "include"
    if inc.exists():
        shutil.rmtree(inc)
    inc.mkdir(parents=True)
    for src in sorted(REF_INCLUDE.glob("*.hpp")):
        text = src.read_text()
        if src.name == "signature.hpp":
            text = patch_signature_header(text)
        (inc / src.name).write_text(text)
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    cmd = [cxx, "-std=c++20", "-O0", "-w", "-DSIGMO_ALLOCATION=1", f"-I{HERE / 'sycl_host'}", f"-I{inc}",
           "-o", str(BIN), str(HERE / "ref_pipeline.cpp")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("building the reference failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr[-8000:])
    return BIN


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
