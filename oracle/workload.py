"""Seeded synthetic inputs for the CPU side — TEST / BENCH INFRASTRUCTURE.

oracle/libsigmo_workload.so is the library's own seeded generator and batch
helpers (sigmo_b200/csrc/generator.cpp, host_graphs.cpp) compiled with g++
alone.  bench.py's reference arm makes its inputs here, so that arm maps the
oracle and this host library but never the product's CUDA library; the graphs
are identical to sigmo_b200.generate_molecules / generate_queries for the same
arguments (tests/test_abi_cpu.py checks that).  Batches come back as
oracle.Batch (numpy copies).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

from . import Batch

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libsigmo_workload.so"


class _HostGraphsC(ctypes.Structure):
    # sigmo_host_graphs (include/sigmo_b200.h)
    _fields_ = [
        ("num_graphs", ctypes.c_uint32),
        ("total_nodes", ctypes.c_uint64),
        ("total_edges", ctypes.c_uint64),
        ("graph_offsets", ctypes.c_void_p),
        ("row_offsets", ctypes.c_void_p),
        ("column_indices", ctypes.c_void_p),
        ("node_labels", ctypes.c_void_p),
        ("edge_labels", ctypes.c_void_p),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), str(LIB_PATH)], check=True)
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER(_HostGraphsC)
        u32, u64 = ctypes.c_uint32, ctypes.c_uint64
        L.sigmo_generate_molecules.argtypes = [ctypes.c_int, u32, u32, u32, ctypes.c_double, u64, P]
        L.sigmo_generate_queries.argtypes = [ctypes.c_int, u32, u32, u32, u32, u32, u64, P]
        L.sigmo_host_graphs_free.argtypes = [P]
        L.sigmo_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _copy_out(raw: _HostGraphsC) -> Batch:
    def arr(ptr, ct, dt, n):
        if n == 0 or not ptr:
            return np.zeros(n, dt)
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,)).copy()

    G, N, E = int(raw.num_graphs), int(raw.total_nodes), int(raw.total_edges)
    try:
        return Batch(arr(raw.graph_offsets, ctypes.c_uint32, np.uint32, G + 1),
                     arr(raw.row_offsets, ctypes.c_uint32, np.uint32, N + 1),
                     arr(raw.column_indices, ctypes.c_uint32, np.uint32, E),
                     arr(raw.node_labels, ctypes.c_uint8, np.uint8, N),
                     arr(raw.edge_labels, ctypes.c_uint8, np.uint8, E))
    finally:
        lib().sigmo_host_graphs_free(ctypes.byref(raw))


def _check(rc: int):
    if rc != 0:
        raise RuntimeError(f"workload generator: {lib().sigmo_last_error().decode()} (status {rc})")


def generate_molecules(count: int, min_atoms: int = 10, max_atoms: int = 40, seed: int = 1, kind: int = 0,
                       median: float = 22.0) -> Batch:
    raw = _HostGraphsC()
    _check(lib().sigmo_generate_molecules(kind, count, min_atoms, max_atoms, median, seed, ctypes.byref(raw)))
    return _copy_out(raw)


def generate_queries(count: int, min_atoms: int = 4, max_atoms: int = 12, seed: int = 2, kind: int = 0,
                     skew_lo: int = 0, skew_hi: int = 0) -> Batch:
    raw = _HostGraphsC()
    _check(lib().sigmo_generate_queries(kind, count, min_atoms, max_atoms, skew_lo, skew_hi, seed, ctypes.byref(raw)))
    return _copy_out(raw)


def slice_graphs(b: Batch, first: int, count: int) -> Batch:
    """Graphs [first, first + count) of a batch with ids re-based to 0 (the
    same batch sigmo_host_graphs_slice returns)."""
    first = max(0, min(first, b.num_graphs))
    count = max(0, min(count, b.num_graphs - first))
    v0, v1 = int(b.graph_offsets[first]), int(b.graph_offsets[first + count])
    e0, e1 = int(b.row_offsets[v0]), int(b.row_offsets[v1])
    return Batch((b.graph_offsets[first:first + count + 1] - np.uint32(v0)).astype(np.uint32),
                 (b.row_offsets[v0:v1 + 1] - np.uint32(e0)).astype(np.uint32),
                 (b.column_indices[e0:e1] - np.uint32(v0)).astype(np.uint32),
                 b.node_labels[v0:v1].copy(), b.edge_labels[e0:e1].copy())


def format_text(b: Batch) -> str:
    """The batch in the reference's text format, one graph per line
    (sigmo_format_graphs; scripts/smile2graph.py:173-180 writes the same)."""
    arrs = [np.ascontiguousarray(b.graph_offsets, np.uint32), np.ascontiguousarray(b.row_offsets, np.uint32),
            np.ascontiguousarray(b.column_indices, np.uint32), np.ascontiguousarray(b.node_labels, np.uint8),
            np.ascontiguousarray(b.edge_labels, np.uint8)]
    raw = _HostGraphsC(b.num_graphs, b.total_nodes, b.total_edges, *[a.ctypes.data for a in arrs])
    L = lib()
    L.sigmo_format_graphs.argtypes = [ctypes.POINTER(_HostGraphsC), ctypes.c_char_p, ctypes.POINTER(ctypes.c_size_t)]
    n = ctypes.c_size_t(0)
    _check(L.sigmo_format_graphs(ctypes.byref(raw), None, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    _check(L.sigmo_format_graphs(ctypes.byref(raw), buf, ctypes.byref(n)))
    return buf.raw[: n.value].decode()
