"""Builds libsigmo_b200.so in-tree with nvcc for sm_100a.

Usage: python -m sigmo_b200.build [--force] [-v]
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libsigmo_b200.so"
CLI = HERE / "sigmo_cli"
INCLUDE = HERE.parent / "include"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the sigmo_b200 CUDA library cannot be built")


def _host_compiler() -> str | None:
    # The system g++ (a toolchain wrapper in $CXX may lack parts of the runtime).
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and Path(cand).exists():
            return cand
    return None


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _fingerprint() -> str:
    h = hashlib.sha256()
    for p in sorted(CSRC.iterdir()) + sorted(INCLUDE.rglob("*.h*")) + sorted((HERE / "cli").glob("*")):
        if p.is_file():
            h.update(p.name.encode())
            h.update(p.read_bytes())
    h.update(" ".join(ARCH_FLAGS).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> Path:
    stamp = HERE / ".libsigmo_b200.stamp"
    fp = _fingerprint()
    if LIB.exists() and stamp.exists() and stamp.read_text() == fp and not force:
        return LIB
    cmd = [
        _nvcc(),
        *ARCH_FLAGS,
        "-O3",
        "-std=c++17",
        "-lineinfo",
        "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC",
        "-Xcompiler", "-fvisibility=hidden",
        "-shared",
        "-o", str(LIB),
    ]
    hc = _host_compiler()
    if hc:
        cmd += ["-ccbin", hc]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [str(s) for s in sources()]
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    res = subprocess.run(cmd, cwd=str(HERE), capture_output=True, text=True, env=env)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stdout + res.stderr)
    build_cli(hc)
    stamp.write_text(fp)
    return LIB


def build_cli(host_compiler: str | None = None) -> Path:
    """The command-line driver (same flags and report as the reference's
    sigmo driver), linked against the in-tree library."""
    cxx = host_compiler or _host_compiler() or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-o", str(CLI), str(HERE / "cli" / "sigmo_main.cpp"), f"-L{HERE}", "-lsigmo_b200",
           "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("building the CLI failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    return CLI


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
