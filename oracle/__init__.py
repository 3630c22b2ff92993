"""CPU oracle for SIGMo's hot path — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
arm, as the checker.  It wraps oracle/liboracle_sigmo.so (a C++/OpenMP
restatement of the reference, see sigmo_oracle.cpp) and adds a pure-Python
restatement of the text format and batching (library/include/graph.hpp:
154-314) so the product's own parser can be checked against it.

Profiles: REF_PTX (0, default contract), REF_X86 (1), EXACT (2).
"""
from __future__ import annotations

import ctypes
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_sigmo.so"

REF_PTX, REF_X86, EXACT = 0, 1, 2
PROFILES = {"ref-ptx": REF_PTX, "ref-x86": REF_X86, "exact": EXACT}


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


class _OrcGraph(ctypes.Structure):
    _fields_ = [
        ("num_graphs", ctypes.c_uint32),
        ("total_nodes", ctypes.c_uint64),
        ("total_edges", ctypes.c_uint64),
        ("graph_offsets", ctypes.c_void_p),
        ("row_offsets", ctypes.c_void_p),
        ("column_indices", ctypes.c_void_p),
        ("node_labels", ctypes.c_void_p),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER(_OrcGraph)
        vp, u32, u64, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        L.orc_generate_signatures.argtypes = [P, vp]
        L.orc_refine_signatures.argtypes = [P, u32, i32, vp, vp, u32]
        L.orc_refine_signatures.restype = i32
        L.orc_filter.argtypes = [P, P, vp]
        L.orc_refine.argtypes = [P, P, vp, vp, vp]
        L.orc_gmcr.argtypes = [P, P, vp, i32, vp, vp, u64]
        L.orc_gmcr.restype = u64
        L.orc_join.argtypes = [P, P, vp, vp, vp, i32, i32, u32, vp]
        L.orc_join.restype = u64
        L.orc_join_closed_form.argtypes = [P, P, vp, vp, vp, i32, vp]
        L.orc_join_closed_form.restype = u64
        L.orc_join_wildcard.argtypes = [P, vp, P, vp, vp, vp, vp, i32, i32, ctypes.c_uint32, vp]
        L.orc_join_wildcard.restype = u64
        L.orc_sig_set.argtypes = [u64, u32, u32]
        L.orc_sig_set.restype = u64
        L.orc_sig_get.argtypes = [u64, u32]
        L.orc_sig_get.restype = u32
        L.orc_sig_increment.argtypes = [u64, u32, u32]
        L.orc_sig_increment.restype = u64
        L.orc_digest.argtypes = [vp, u64, u64]
        L.orc_digest.restype = u64
        L.orc_num_threads.restype = i32
        L.orc_set_num_threads.argtypes = [i32]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Batch:
    """Batched CSR with global ids (the arrays createDeviceCSRGraph builds)."""

    graph_offsets: np.ndarray  # uint32 [G+1]
    row_offsets: np.ndarray  # uint32 [N+1]
    column_indices: np.ndarray  # uint32 [E]
    node_labels: np.ndarray  # uint8 [N]
    edge_labels: np.ndarray  # uint8 [E]

    @property
    def num_graphs(self) -> int:
        return len(self.graph_offsets) - 1

    @property
    def total_nodes(self) -> int:
        return len(self.node_labels)

    @property
    def total_edges(self) -> int:
        return len(self.column_indices)


def as_batch(g) -> Batch:
    """Accepts any object with the five batched arrays (e.g. sigmo_b200.HostGraphs)."""
    if isinstance(g, Batch):
        return g
    return Batch(
        np.ascontiguousarray(g.graph_offsets, dtype=np.uint32),
        np.ascontiguousarray(g.row_offsets, dtype=np.uint32),
        np.ascontiguousarray(g.column_indices, dtype=np.uint32),
        np.ascontiguousarray(g.node_labels, dtype=np.uint8),
        np.ascontiguousarray(g.edge_labels, dtype=np.uint8),
    )


def _cg(b: Batch) -> _OrcGraph:
    return _OrcGraph(
        b.num_graphs, b.total_nodes, b.total_edges, _ptr(b.graph_offsets).value, _ptr(b.row_offsets).value,
        _ptr(b.column_indices).value, _ptr(b.node_labels).value,
    )


# ---- text format: pure-Python restatement of graph.hpp:154-314 -------------
def parse_line(line: str):
    """IntermediateGraph(line) (graph.hpp:154-206): (n, labels, edges)."""
    tok = line.split()
    n = int(tok[0][2:])
    labels = [0] * n
    pos = 2
    for _ in range(n):
        node, lab = int(tok[pos]), int(tok[pos + 1])
        labels[node] = lab & 0xFF
        pos += 2
    ne = int(tok[pos][2:])
    rest = tok[pos + 1:]
    if len(rest) == ne * 3:
        edges = [(int(rest[3 * i]), int(rest[3 * i + 1]), int(rest[3 * i + 2]) & 0xFF) for i in range(ne)]
    elif len(rest) == ne * 2:
        edges = [(int(rest[2 * i]), int(rest[2 * i + 1]), 0) for i in range(ne)]
    else:
        raise ValueError("Invalid graph format")
    return n, labels, edges


def to_csr(n, labels, edges):
    """toCSRGraph (graph.hpp:216-247)."""
    ro = [0] * (n + 1)
    for u, v, _ in edges:
        ro[u + 1] += 1
        ro[v + 1] += 1
    for i in range(1, n + 1):
        ro[i] += ro[i - 1]
    col = [0] * ro[-1]
    el = [0] * ro[-1]
    cur = [0] * (n + 1)
    for u, v, l in edges:
        col[ro[u] + cur[u]] = v
        el[ro[u] + cur[u]] = l
        col[ro[v] + cur[v]] = u
        el[ro[v] + cur[v]] = l
        cur[u] += 1
        cur[v] += 1
    return ro, col, labels, el


def batch(csrs) -> Batch:
    """createDeviceCSRGraph host concatenation (graph.hpp:255-294)."""
    go, ro, col, nl, el = [0], [], [], [], []
    vo = eo = 0
    for r, c, lab, e in csrs:
        n = len(lab)
        go.append(go[-1] + n)
        ro.extend(x + eo for x in r[:-1])
        col.extend(x + vo for x in c)
        el.extend(e)
        nl.extend(lab)
        vo += n
        eo += len(c)
    ro.append(eo)
    return Batch(np.array(go, np.uint32), np.array(ro, np.uint32), np.array(col, np.uint32), np.array(nl, np.uint8),
                 np.array(el, np.uint8))


def parse_text(text: str) -> Batch:
    return batch([to_csr(*parse_line(l)) for l in text.splitlines() if l.strip()])


# ---- pipeline stages ---------------------------------------------------------
def words(n: int) -> int:
    return (n + 31) // 32


def generate_signatures(g, sig: np.ndarray | None = None) -> np.ndarray:
    b = as_batch(g)
    if sig is None:
        sig = np.zeros(b.total_nodes, np.uint64)
    if b.total_nodes:
        lib().orc_generate_signatures(ctypes.byref(_cg(b)), _ptr(sig))
    return sig


def new_reach(n: int, profile: int) -> np.ndarray:
    return np.zeros((n, 4 if profile == EXACT else 1), np.uint64)


def refine_signatures(g, view: int, profile: int, sig: np.ndarray, reach: np.ndarray) -> np.ndarray:
    b = as_batch(g)
    if b.total_nodes:
        rc = lib().orc_refine_signatures(ctypes.byref(_cg(b)), view, profile, _ptr(sig), _ptr(reach), reach.shape[1])
        if rc != 0:
            raise ValueError("graph outside the oracle's exact-profile domain (> 256 vertices)")
    return sig


def filter_candidates(qg, dg) -> np.ndarray:
    q, d = as_batch(qg), as_batch(dg)
    bits = np.zeros((q.total_nodes, words(d.total_nodes)), np.uint32)
    if bits.size:
        lib().orc_filter(ctypes.byref(_cg(q)), ctypes.byref(_cg(d)), _ptr(bits))
    return bits


def refine_candidates(qg, dg, sigq: np.ndarray, sigd: np.ndarray, bits: np.ndarray) -> np.ndarray:
    q, d = as_batch(qg), as_batch(dg)
    if bits.size:
        lib().orc_refine(ctypes.byref(_cg(q)), ctypes.byref(_cg(d)), _ptr(sigq), _ptr(sigd), _ptr(bits))
    return bits


def gmcr(qg, dg, bits: np.ndarray, profile: int = REF_PTX):
    q, d = as_batch(qg), as_batch(dg)
    offsets = np.zeros(d.num_graphs + 1, np.uint32)
    L = lib()
    total = L.orc_gmcr(ctypes.byref(_cg(q)), ctypes.byref(_cg(d)), _ptr(bits), profile, _ptr(offsets), None, 0)
    indices = np.zeros(max(total, 1), np.uint32)
    L.orc_gmcr(ctypes.byref(_cg(q)), ctypes.byref(_cg(d)), _ptr(bits), profile, _ptr(offsets), _ptr(indices), total)
    return offsets, indices[:total]


def join(qg, dg, bits, offsets, indices, profile: int = REF_PTX, find_first: bool = False, wg: int = 128):
    q, d = as_batch(qg), as_batch(dg)
    per = np.zeros(max(len(indices), 1), np.uint64)
    idx = np.ascontiguousarray(indices, np.uint32) if len(indices) else np.zeros(1, np.uint32)
    total = lib().orc_join(ctypes.byref(_cg(q)), ctypes.byref(_cg(d)), _ptr(bits), _ptr(offsets), _ptr(idx), profile,
                           int(find_first), wg, _ptr(per))
    if total == 2**64 - 1:
        raise ValueError("input outside the oracle's join domain")
    return int(total), per[: len(indices)]


def join_closed_form(qg, dg, bits, offsets, indices, find_first: bool = False):
    q, d = as_batch(qg), as_batch(dg)
    per = np.zeros(max(len(indices), 1), np.uint64)
    idx = np.ascontiguousarray(indices, np.uint32) if len(indices) else np.zeros(1, np.uint32)
    total = lib().orc_join_closed_form(ctypes.byref(_cg(q)), ctypes.byref(_cg(d)), _ptr(bits), _ptr(offsets), _ptr(idx),
                                       int(find_first), _ptr(per))
    return int(total), per[: len(indices)]



def join_wildcard(qg, dg, bits, offsets, indices, profile: int = REF_PTX, find_first: bool = True, wg: int = 128):
    """joinWildcardCandidates (isomorphism.hpp:435-560) on the final bitset and
    GMCR: returns (total, per-slot counts)."""
    q, d = as_batch(qg), as_batch(dg)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
    idx = np.ascontiguousarray(indices, dtype=np.uint32)
    per = np.zeros(max(int(offsets[-1]), 1), np.uint64)
    qel = np.ascontiguousarray(q.edge_labels, dtype=np.uint8)
    del_ = np.ascontiguousarray(d.edge_labels, dtype=np.uint8)
    total = lib().orc_join_wildcard(ctypes.byref(_cg(q)), _ptr(qel), ctypes.byref(_cg(d)), _ptr(del_), _ptr(bits), _ptr(offsets),
                                    _ptr(idx), profile, int(bool(find_first)), wg, _ptr(per))
    if total == 2**64 - 1:
        raise ValueError("outside the oracle's domain")
    return int(total), per[: int(offsets[-1])]

def run_pipeline(qg, dg, iterations: int, profile: int = REF_PTX, find_first: bool = False, wg: int = 128,
                 keep: bool = False, skip_join: bool = False, digests: bool = False):
    """The driver's stage order (library/src/sigmo.cpp:98-160): data then query
    signatures, label filter, R x (refine data sigs, refine query sigs, refine
    candidates), GMCR, join.  keep=True records signatures / bitsets of every
    iteration; digests=True records only the bitset digest after the filter
    and after every refinement (out["digests"], R + 1 values) — the form for
    full-size batches whose bitsets take gigabytes."""
    q, d = as_batch(qg), as_batch(dg)
    sd = generate_signatures(d)
    sq = generate_signatures(q)
    bits = filter_candidates(q, d)
    out = {"bitsets": [], "sig_data": [], "sig_query": [], "digests": []}

    def record():
        if keep:
            out["bitsets"].append(bits.copy())
            out["sig_data"].append(sd.copy())
            out["sig_query"].append(sq.copy())
        if digests:
            out["digests"].append(digest_fast(bits))

    record()
    rd, rq = new_reach(d.total_nodes, profile), new_reach(q.total_nodes, profile)
    for r in range(1, iterations + 1):
        refine_signatures(d, r, profile, sd, rd)
        refine_signatures(q, r, profile, sq, rq)
        refine_candidates(q, d, sq, sd, bits)
        record()
    out["bits"] = bits
    if skip_join:
        return out
    offsets, indices = gmcr(q, d, bits, profile)
    total, per = join(q, d, bits, offsets, indices, profile, find_first, wg)
    out.update(offsets=offsets, indices=indices, total=total, per_pair=per)
    return out


# ---- digest matching the library's sigmo_candidates_digest ------------------
_M = (1 << 64) - 1


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def digest(bits: np.ndarray) -> int:
    """sum_q mix64(h_q + q*K2), h_q = sum_w mix64(word ^ (w*K1)) mod 2^64."""
    K1, K2 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xC2B2AE3D27D4EB4F)
    if bits.size == 0:
        return 0
    with np.errstate(over="ignore"):
        w = np.arange(bits.shape[1], dtype=np.uint64) * K1
        h = _mix64(bits.astype(np.uint64) ^ w[None, :]).sum(axis=1, dtype=np.uint64)
        qv = np.arange(bits.shape[0], dtype=np.uint64) * K2
        return int(_mix64(h + qv).sum(dtype=np.uint64))


def digest_fast(bits: np.ndarray) -> int:
    """digest() computed by the oracle library (OpenMP), for large bitsets."""
    if bits.size == 0:
        return 0
    b = np.ascontiguousarray(bits, dtype=np.uint32)
    return int(lib().orc_digest(_ptr(b), b.shape[0], b.shape[1]))
