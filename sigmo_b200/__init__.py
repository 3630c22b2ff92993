"""sigmo_b200: B200-native (sm_100a) SIGMo hot path behind a C ABI.

This Python layer mirrors the reference's C++ host API (namespace sigmo,
library/include/*.hpp) over ctypes bindings of libsigmo_b200.so:

  io.loadCSRGraphsFromFile / io.loadCSRGraphsFromLines      io.hpp:46-55
  createDeviceCSRGraph / destroyDeviceCSRGraph              graph.hpp:255-322
  candidates.Candidates                                      candidates.hpp:14-204
  signature.Signature (PowerGraph, 4-bit counters)           signature.hpp:20-391
  isomorphism.filter.filterCandidates / refineCandidates     isomorphism.hpp:22-127
  isomorphism.mapping.GMCR                                   gmcr.hpp:16-131
  isomorphism.join.joinCandidates                            isomorphism.hpp:270-381

`sycl::queue` becomes `Queue` (a CUDA stream plus options).  Every call runs
on the GPU; there is no CPU fallback: if the library is missing or no GPU is
present the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from types import SimpleNamespace

import numpy as np

from . import _lib as _L
from ._lib import SigmoError, check, lib

REF_PTX, REF_X86, EXACT = 0, 1, 2
PROFILE_NAMES = {"ref-ptx": REF_PTX, "ref-x86": REF_X86, "exact": EXACT}
SCOPE_DATA, SCOPE_QUERY = 0, 1

__all__ = [
    "SigmoError", "HostGraphs", "Queue", "DeviceBatchedCSRGraph", "createDeviceCSRGraph", "destroyDeviceCSRGraph",
    "io", "candidates", "signature", "isomorphism", "generate_molecules", "generate_queries", "match_batched",
    "Server", "REF_PTX", "EXACT",
]


def library_path() -> Path:
    return _L.LIB_PATH


# ---- host graphs ---------------------------------------------------------------
class HostGraphs:
    """A batch of graphs on the host in the batched CSR layout with global ids
    (what createDeviceCSRGraph builds before copying, graph.hpp:255-294).
    Owned by the library; the numpy views stay valid while this object lives."""

    def __init__(self, raw: _L.HostGraphsC):
        self._raw = raw

    def __del__(self):
        try:
            lib().sigmo_host_graphs_free(ctypes.byref(self._raw))
        except Exception:
            pass

    def _view(self, name, dtype, n):
        ptr = getattr(self._raw, name)
        if n == 0 or not ptr:
            return np.zeros(0, dtype)
        ct = {np.uint32: ctypes.c_uint32, np.uint8: ctypes.c_uint8}[dtype]
        arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,))
        arr.flags.writeable = False
        return arr

    @property
    def num_graphs(self) -> int:
        return int(self._raw.num_graphs)

    @property
    def total_nodes(self) -> int:
        return int(self._raw.total_nodes)

    @property
    def total_edges(self) -> int:
        return int(self._raw.total_edges)

    @property
    def graph_offsets(self):
        return self._view("graph_offsets", np.uint32, self.num_graphs + 1)

    @property
    def row_offsets(self):
        return self._view("row_offsets", np.uint32, self.total_nodes + 1)

    @property
    def column_indices(self):
        return self._view("column_indices", np.uint32, self.total_edges)

    @property
    def node_labels(self):
        return self._view("node_labels", np.uint8, self.total_nodes)

    @property
    def edge_labels(self):
        return self._view("edge_labels", np.uint8, self.total_edges)

    def __len__(self):
        return self.num_graphs

    def sizes(self) -> np.ndarray:
        return np.diff(self.graph_offsets.astype(np.int64))

    def slice(self, first: int, count: int) -> "HostGraphs":
        out = _L.HostGraphsC()
        check(lib().sigmo_host_graphs_slice(ctypes.byref(self._raw), first, count, ctypes.byref(out)))
        return HostGraphs(out)

    def concat(self, other: "HostGraphs") -> "HostGraphs":
        out = _L.HostGraphsC()
        check(lib().sigmo_host_graphs_concat(ctypes.byref(self._raw), ctypes.byref(other._raw), ctypes.byref(out)))
        return HostGraphs(out)

    def to_text(self) -> str:
        n = ctypes.c_size_t(0)
        check(lib().sigmo_format_graphs(ctypes.byref(self._raw), None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        check(lib().sigmo_format_graphs(ctypes.byref(self._raw), buf, ctypes.byref(n)))
        return buf.raw[: n.value].decode()

    def save(self, path) -> None:
        """Binary batch file (sigmo_graphs_save)."""
        check(lib().sigmo_graphs_save(ctypes.byref(self._raw), str(path).encode()))

    @staticmethod
    def load(path) -> "HostGraphs":
        out = _L.HostGraphsC()
        check(lib().sigmo_graphs_load(str(path).encode(), ctypes.byref(out)))
        return HostGraphs(out)

    def local_arrays(self):
        """The batch as per-graph CSRs back to back with local ids (the input
        of createDeviceCSRGraphFromLocal): node counts, directed-edge counts,
        each graph's n+1 row pointers from 0, local neighbour ids."""
        goff = self.graph_offsets.astype(np.int64)
        roff = self.row_offsets.astype(np.int64)
        n = np.diff(goff)
        e = roff[goff[1:]] - roff[goff[:-1]]
        # row pointers: graph g contributes roff[goff[g] .. goff[g+1]] - roff[goff[g]]
        idx = np.concatenate([np.arange(a, b + 1) for a, b in zip(goff[:-1], goff[1:])]) if len(n) else np.zeros(0, np.int64)
        base = np.repeat(roff[goff[:-1]], n + 1)
        rows = (roff[idx] - base).astype(np.uint32)
        gof_edge = np.repeat(goff[:-1], e)
        cols = (self.column_indices.astype(np.int64) - gof_edge).astype(np.uint32)
        return n.astype(np.uint32), e.astype(np.uint32), rows, cols

    @staticmethod
    def from_text(text: str) -> "HostGraphs":
        data = text.encode()
        out = _L.HostGraphsC()
        check(lib().sigmo_parse_graphs(data, len(data), ctypes.byref(out)))
        return HostGraphs(out)


def _load_lines(lines) -> HostGraphs:
    return HostGraphs.from_text("\n".join(lines))


def _load_file(path) -> HostGraphs:
    return HostGraphs.from_text(Path(path).read_text())


io = SimpleNamespace(loadCSRGraphsFromFile=_load_file, loadCSRGraphsFromLines=_load_lines, parse=HostGraphs.from_text)


def generate_molecules(count: int, min_atoms: int = 10, max_atoms: int = 40, seed: int = 1, kind: int = 0,
                       median: float = 22.0) -> HostGraphs:
    out = _L.HostGraphsC()
    check(lib().sigmo_generate_molecules(kind, count, min_atoms, max_atoms, median, seed, ctypes.byref(out)))
    return HostGraphs(out)


def generate_queries(count: int, min_atoms: int = 4, max_atoms: int = 12, seed: int = 2, kind: int = 0,
                     skew_lo: int = 0, skew_hi: int = 0) -> HostGraphs:
    out = _L.HostGraphsC()
    check(lib().sigmo_generate_queries(kind, count, min_atoms, max_atoms, skew_lo, skew_hi, seed, ctypes.byref(out)))
    return HostGraphs(out)


# ---- queue --------------------------------------------------------------------------
class BatchedEvent:
    """utils::BatchedEvent (utils.hpp:127-161): device time of a stage."""

    def __init__(self, queue: "Queue"):
        self._ms = None
        self._queue = queue
        v = ctypes.c_double(0)
        check(lib().sigmo_queue_last_stage_ms(queue._h, ctypes.byref(v)))
        self._ms = v.value

    def wait(self):
        self._queue.wait()

    def getProfilingInfo(self) -> float:
        """Seconds of device time (the reference returns duration<double>)."""
        return self._ms / 1e3


class Queue:
    """sycl::queue replacement: a CUDA stream on one device plus the options
    of device::DeviceOptions (device.hpp:17-21) and the semantics profile."""

    def __init__(self, device: int = 0, profile="ref-ptx", join_work_group_size: int = 128,
                 filter_work_group_size: int = 512):
        if isinstance(profile, str):
            profile = PROFILE_NAMES[profile]
        opts = _L.OptionsC(int(profile), join_work_group_size, filter_work_group_size)
        h = ctypes.c_void_p()
        check(lib().sigmo_queue_create(device, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self.profile = int(profile)
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().sigmo_queue_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def wait(self):
        check(lib().sigmo_queue_wait(self._h))

    wait_and_throw = wait

    @property
    def stream(self) -> int:
        p = ctypes.c_void_p()
        check(lib().sigmo_queue_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def set_tuning(self, **fields):
        """Join launch shape (sigmo_tuning); unspecified fields keep their value."""
        t = _L.TuningC()
        check(lib().sigmo_queue_get_tuning(self._h, ctypes.byref(t)))
        for k, v in fields.items():
            setattr(t, k, int(v))
        check(lib().sigmo_queue_set_tuning(self._h, ctypes.byref(t)))

    def get_tuning(self) -> dict:
        t = _L.TuningC()
        check(lib().sigmo_queue_get_tuning(self._h, ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in _L.TuningC._fields_}

    def set_join_budget(self, steps: int):
        """Step budget of the join kernels (sigmo_queue_set_join_budget): the
        most DFS levels one lane may leave per launch, 0 for no limit; a join
        that runs out raises SigmoError with code SIGMO_ERR_TIMEOUT (7)."""
        check(lib().sigmo_queue_set_join_budget(self._h, int(steps)))

    def join_budget(self) -> int:
        v = ctypes.c_uint64()
        check(lib().sigmo_queue_get_join_budget(self._h, ctypes.byref(v)))
        return v.value

    def launch_count(self) -> int:
        v = ctypes.c_uint64()
        check(lib().sigmo_queue_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def device_info(self):
        mem = ctypes.c_uint64()
        name = ctypes.create_string_buffer(256)
        check(lib().sigmo_queue_device_info(self._h, ctypes.byref(mem), name, 256))
        return mem.value, name.value.decode()


# ---- device graphs -------------------------------------------------------------------
class DeviceBatchedCSRGraph:
    """DeviceBatchedCSRGraph (graph.hpp:62-112) held on the device."""

    def __init__(self, queue: Queue, handle):
        self._queue = queue
        self._h = handle
        ng, tn, te, mx = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        check(lib().sigmo_graph_info(handle, ctypes.byref(ng), ctypes.byref(tn), ctypes.byref(te), ctypes.byref(mx)))
        self.num_graphs, self.total_nodes, self.total_edges, self.max_graph_nodes = ng.value, tn.value, te.value, mx.value

    def destroy(self):
        if getattr(self, "_h", None):
            lib().sigmo_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def set_vertex_base(self, base: int) -> None:
        """This batch is a shard whose vertex 0 has global id `base`
        (sigmo_graph_set_vertex_base)."""
        check(lib().sigmo_graph_set_vertex_base(self._h, base))

    def alloc_size(self) -> int:
        v = ctypes.c_uint64()
        check(lib().sigmo_graph_alloc_size(self._h, ctypes.byref(v)))
        return v.value


def createDeviceCSRGraph(queue: Queue, graphs: HostGraphs) -> DeviceBatchedCSRGraph:
    h = ctypes.c_void_p()
    check(lib().sigmo_graph_create(queue._h, ctypes.byref(graphs._raw), ctypes.byref(h)))
    return DeviceBatchedCSRGraph(queue, h)


def createDeviceCSRGraphFromLocal(queue: Queue, graphs: HostGraphs) -> DeviceBatchedCSRGraph:
    """createDeviceCSRGraph with the concatenation on the device
    (sigmo_graph_create_from_local), from the batch's per-graph local arrays."""
    n, e, rows, cols = graphs.local_arrays()
    nl = np.ascontiguousarray(graphs.node_labels)
    el = np.ascontiguousarray(graphs.edge_labels)
    h = ctypes.c_void_p()
    check(lib().sigmo_graph_create_from_local(queue._h, graphs.num_graphs, n.ctypes.data, e.ctypes.data, rows.ctypes.data,
                                              cols.ctypes.data, nl.ctypes.data, el.ctypes.data, ctypes.byref(h)))
    return DeviceBatchedCSRGraph(queue, h)


def createDeviceCSRGraphFromDevice(queue: Queue, num_graphs: int, total_nodes: int, total_edges: int, graph_offsets: int,
                                   row_offsets: int, column_indices: int, node_labels: int,
                                   edge_labels: int) -> DeviceBatchedCSRGraph:
    """Wrap five device-resident arrays (raw device pointers) without copying."""
    h = ctypes.c_void_p()
    check(lib().sigmo_graph_create_device(queue._h, num_graphs, total_nodes, total_edges, graph_offsets, row_offsets,
                                          column_indices, node_labels, edge_labels, ctypes.byref(h)))
    return DeviceBatchedCSRGraph(queue, h)


def destroyDeviceCSRGraph(graph: DeviceBatchedCSRGraph, queue: Queue | None = None):
    graph.destroy()


def getDeviceGraphAllocSize(graph: DeviceBatchedCSRGraph) -> int:
    return graph.alloc_size()


# ---- candidates ------------------------------------------------------------------------
class Candidates:
    """candidates::Candidates (candidates.hpp:14-204): query-vertex-major bit
    matrix, zero-filled at construction."""

    def __init__(self, queue: Queue, source_nodes: int, target_nodes: int):
        h = ctypes.c_void_p()
        check(lib().sigmo_candidates_create(queue._h, source_nodes, target_nodes, ctypes.byref(h)))
        self._h, self._queue = h, queue
        self.source_nodes, self.target_nodes = source_nodes, target_nodes
        self.single_node_size = (target_nodes + 31) // 32

    def close(self):
        if getattr(self, "_h", None):
            lib().sigmo_candidates_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def getHostCandidates(self, row0: int = 0, rows: int | None = None) -> np.ndarray:
        """Dense [rows][single_node_size] uint32 copy (candidates.hpp:185-190)."""
        if rows is None:
            rows = self.source_nodes - row0
        out = np.zeros((rows, self.single_node_size), np.uint32)
        check(lib().sigmo_candidates_download(self._h, row0, rows, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def getCandidatesCounts(self) -> np.ndarray:
        out = np.zeros(self.source_nodes, np.uint32)
        check(lib().sigmo_candidates_row_counts(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def getCandidatesCount(self, source_node: int) -> int:
        """getCandidatesCount(source) (candidates.hpp:77-81)."""
        return int(np.unpackbits(self.getHostCandidates(source_node, 1).view(np.uint8)).sum())

    def getAllocationSize(self) -> int:
        v = ctypes.c_uint64()
        check(lib().sigmo_candidates_alloc_size(self._h, ctypes.byref(v)))
        return v.value

    def digest(self) -> int:
        v = ctypes.c_uint64()
        check(lib().sigmo_candidates_digest(self._h, ctypes.byref(v)))
        return v.value


# ---- signatures --------------------------------------------------------------------------
class Signature:
    """signature::Signature<PowerGraph, 4> (signature.hpp:20-391)."""

    def __init__(self, queue: Queue, data_nodes: int, query_nodes: int):
        h = ctypes.c_void_p()
        check(lib().sigmo_signature_create(queue._h, data_nodes, query_nodes, ctypes.byref(h)))
        self._h, self._queue = h, queue
        self.data_nodes, self.query_nodes = data_nodes, query_nodes

    def close(self):
        if getattr(self, "_h", None):
            lib().sigmo_signature_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _gen(self, g, scope):
        check(lib().sigmo_signature_generate(self._h, g._h, scope))
        return BatchedEvent(self._queue)

    def _ref(self, g, scope, view):
        check(lib().sigmo_signature_refine(self._h, g._h, scope, view))
        return BatchedEvent(self._queue)

    def generateDataSignatures(self, g):
        return self._gen(g, SCOPE_DATA)

    def generateQuerySignatures(self, g):
        return self._gen(g, SCOPE_QUERY)

    def refineDataSignatures(self, g, view_size: int = 1):
        return self._ref(g, SCOPE_DATA, view_size)

    def refineQuerySignatures(self, g, view_size: int = 1):
        return self._ref(g, SCOPE_QUERY, view_size)

    def _download(self, scope, n):
        out = np.zeros(n, np.uint64)
        check(lib().sigmo_signature_download(self._h, scope, out.ctypes.data_as(ctypes.c_void_p), n))
        return out

    def getDataSignatures(self) -> np.ndarray:
        return self._download(SCOPE_DATA, self.data_nodes)

    def getQuerySignatures(self) -> np.ndarray:
        return self._download(SCOPE_QUERY, self.query_nodes)

    @staticmethod
    def getMaxLabels() -> int:
        return 16


# ---- filter / mapping / join ----------------------------------------------------------------
def filterCandidates(queue: Queue, query_graph, data_graph, signatures: Signature, candidates: Candidates):
    check(lib().sigmo_filter_candidates(queue._h, query_graph._h, data_graph._h, signatures._h, candidates._h))
    return BatchedEvent(queue)


def refineCandidates(queue: Queue, query_graph, data_graph, signatures: Signature, candidates: Candidates):
    check(lib().sigmo_refine_candidates(queue._h, query_graph._h, data_graph._h, signatures._h, candidates._h))
    return BatchedEvent(queue)


class GMCR:
    """isomorphism::mapping::GMCR (gmcr.hpp:16-131)."""

    def __init__(self, queue: Queue):
        h = ctypes.c_void_p()
        check(lib().sigmo_gmcr_create(queue._h, ctypes.byref(h)))
        self._h, self._queue = h, queue
        self._num_data_graphs = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().sigmo_gmcr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def generateGMCR(self, query_graphs, data_graphs, candidates: Candidates):
        check(lib().sigmo_gmcr_generate(self._h, query_graphs._h, data_graphs._h, candidates._h))
        self._num_data_graphs = data_graphs.num_graphs
        return BatchedEvent(self._queue)

    @property
    def total_query_indices(self) -> int:
        v = ctypes.c_uint64()
        check(lib().sigmo_gmcr_total(self._h, ctypes.byref(v)))
        return v.value

    def getGMCR(self):
        """(data_graph_offsets, query_graph_indices) on the host."""
        off = np.zeros(self._num_data_graphs + 1, np.uint32)
        tot = self.total_query_indices
        idx = np.zeros(max(tot, 1), np.uint32)
        check(lib().sigmo_gmcr_download(self._h, off.ctypes.data_as(ctypes.c_void_p), len(off),
                                        idx.ctypes.data_as(ctypes.c_void_p), len(idx)))
        return off, idx[:tot]

    def getPairCounts(self) -> np.ndarray:
        """Per-slot match counts of the last join / batched match on this GMCR."""
        tot = self.total_query_indices
        out = np.zeros(max(tot, 1), np.uint64)
        check(lib().sigmo_match_download_counts(self._h, out.ctypes.data_as(ctypes.c_void_p), len(out)))
        return out[:tot]


def joinCandidates(queue: Queue, query_graphs, data_graphs, candidates: Candidates, gmcr: GMCR, num_matches,
                   find_first: bool = True, per_pair: bool = False):
    """isomorphism::join::joinCandidates (isomorphism.hpp:270-381).
    num_matches: a one-element numpy uint64 array (the reference's USM
    counter), incremented by the number of matches."""
    acc = ctypes.c_uint64(int(num_matches[0]))
    pp = None
    if per_pair:
        pp = np.zeros(max(gmcr.total_query_indices, 1), np.uint64)
    check(lib().sigmo_join_candidates(queue._h, query_graphs._h, data_graphs._h, candidates._h, gmcr._h,
                                      ctypes.byref(acc), int(bool(find_first)),
                                      pp.ctypes.data_as(ctypes.c_void_p) if pp is not None else None))
    num_matches[0] = acc.value
    ev = BatchedEvent(queue)
    if per_pair:
        return ev, pp[: gmcr.total_query_indices]
    return ev


def joinWildcardCandidates(queue: Queue, query_graphs, data_graphs, candidates: Candidates, gmcr: GMCR, num_matches,
                           find_first: bool = True, per_pair: bool = False):
    """isomorphism::join::joinWildcardCandidates (isomorphism.hpp:435-560):
    max-candidate root, the root's candidates split over a sub-group's lanes,
    bond labels checked.  Same arguments and result as joinCandidates."""
    acc = ctypes.c_uint64(int(num_matches[0]))
    pp = np.zeros(max(gmcr.total_query_indices, 1), np.uint64) if per_pair else None
    check(lib().sigmo_join_wildcard_candidates(queue._h, query_graphs._h, data_graphs._h, candidates._h, gmcr._h,
                                               ctypes.byref(acc), int(bool(find_first)),
                                               pp.ctypes.data_as(ctypes.c_void_p) if pp is not None else None))
    num_matches[0] = acc.value
    ev = BatchedEvent(queue)
    if per_pair:
        return ev, pp[: gmcr.total_query_indices]
    return ev


MATCH_MATERIALIZE_BITSET = 1


MATCH_CUDA_GRAPH = 2


def match_batched(queue: Queue, query_graphs, data_graphs, iterations: int, find_first: bool,
                  candidates: Candidates | None, gmcr: GMCR, materialize: bool = False, graph: bool = False) -> dict:
    """The batched form: signatures for all iterations, candidate planes,
    GMCR and the persistent join in one call (same GMCR and counts as the
    stage calls).  With materialize=True the final candidate bitset is also
    written into `candidates`.  With graph=True the batch is captured into a
    CUDA graph on the first call and replayed by later calls with the same
    graphs (SIGMO_MATCH_CUDA_GRAPH)."""
    res = _L.MatchResultC()
    flags = (MATCH_MATERIALIZE_BITSET if materialize else 0) | (MATCH_CUDA_GRAPH if graph else 0)
    check(lib().sigmo_match_batched(queue._h, query_graphs._h, data_graphs._h, iterations, int(bool(find_first)), flags,
                                    candidates._h if candidates is not None else None, gmcr._h, ctypes.byref(res)))
    gmcr._num_data_graphs = data_graphs.num_graphs
    return {f: getattr(res, f) for f, _ in _L.MatchResultC._fields_}


def autotune(queue: Queue, query_graphs, data_graphs, iterations: int, find_first: bool, reps: int = 3) -> dict:
    """Searches the join launch shape on these graphs (sigmo_autotune), keeps
    the fastest on the queue and returns it with the median join times."""
    t = _L.TuningC()
    best, default = ctypes.c_double(), ctypes.c_double()
    check(lib().sigmo_autotune(queue._h, query_graphs._h, data_graphs._h, iterations, int(bool(find_first)), reps,
                               ctypes.byref(t), ctypes.byref(best), ctypes.byref(default)))
    out = {f: getattr(t, f) for f, _ in _L.TuningC._fields_}
    out.update(ms_join=best.value, ms_join_default=default.value)
    return out


# ---- sharding ---------------------------------------------------------------------
def shard_plan(graphs: HostGraphs, shards: int, weight=None, min_first: int = 256):
    """Contiguous ranges of data graphs, one per shard, balanced by `weight`
    per graph (default: vertices).  The first shard ends at or after global
    vertex `min_first`, so every later shard starts at a global id the
    sharded semantics allow.  Returns [(first_graph, count, vertex_base)]."""
    sizes = graphs.sizes()
    w = sizes.astype(np.float64) if weight is None else np.asarray(weight, np.float64)
    goff = graphs.graph_offsets.astype(np.int64)
    G = len(sizes)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    bounds = [0]
    for s in range(1, shards):
        b = int(np.searchsorted(cum, cum[-1] * s / shards))
        b = max(b, bounds[-1])
        if s == 1:
            b = max(b, int(np.searchsorted(goff, min_first)))  # first shard covers vertex min_first
        bounds.append(min(b, G))
    bounds.append(G)
    return [(bounds[i], bounds[i + 1] - bounds[i], int(goff[bounds[i]])) for i in range(shards)]


def createDeviceShard(queue: Queue, graphs: HostGraphs, first: int, count: int) -> DeviceBatchedCSRGraph:
    """Graphs [first, first+count) of a batch on the device, keeping the
    global ids of the whole batch for the semantics (vertex base)."""
    part = graphs.slice(first, count)
    dg = createDeviceCSRGraph(queue, part)
    base = int(graphs.graph_offsets[first]) if count else 0
    if base:
        dg.set_vertex_base(base)
    return dg


# ---- serving loop -----------------------------------------------------------------
REQUEST_PAIRS = 1


class Server:
    """A resident molecule database answering query requests with continuous
    batching (sigmo_server_*).  `submit` queues a request and returns a ticket
    at once; `wait` blocks for its result.  Each request's per-pair results
    are those it gets alone."""

    def __init__(self, database: HostGraphs, device: int = 0, profile="ref-ptx", iterations: int = 6,
                 find_first: bool = True, max_inflight: int = 2, max_batch_queries: int = 64, memory_budget: int = 0,
                 batch_window_us: int = 0, join_work_group_size: int = 128, join_step_budget: int = 0):
        if isinstance(profile, str):
            profile = PROFILE_NAMES[profile]
        opts = _L.OptionsC(int(profile), join_work_group_size, 512)
        so = _L.ServerOptionsC()
        lib().sigmo_server_default_options(ctypes.byref(so))
        so.iterations, so.find_first, so.max_inflight = iterations, int(bool(find_first)), max_inflight
        so.max_batch_queries, so.memory_budget, so.batch_window_us = max_batch_queries, memory_budget, batch_window_us
        so.join_step_budget = join_step_budget
        h = ctypes.c_void_p()
        check(lib().sigmo_server_create(device, ctypes.byref(database._raw), ctypes.byref(opts), ctypes.byref(so),
                                        ctypes.byref(h)))
        self._h = h
        self.num_molecules = database.num_graphs

    def submit(self, queries: HostGraphs, pairs: bool = False) -> int:
        t = ctypes.c_uint64()
        check(lib().sigmo_server_submit(self._h, ctypes.byref(queries._raw), REQUEST_PAIRS if pairs else 0, ctypes.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> dict:
        r = _L.RequestResultC()
        check(lib().sigmo_server_wait(self._h, ticket, timeout_ms, ctypes.byref(r)))
        return {f: getattr(r, f) for f, _ in _L.RequestResultC._fields_}

    def query_totals(self, ticket: int, num_queries: int):
        matched = np.zeros(num_queries, np.uint64)
        total = np.zeros(num_queries, np.uint64)
        check(lib().sigmo_server_query_totals(self._h, ticket, matched.ctypes.data, total.ctypes.data, num_queries))
        return matched, total

    def pairs(self, ticket: int):
        """(query index within the request, molecule, count) of every matched pair."""
        n = ctypes.c_uint64()
        check(lib().sigmo_server_pairs(self._h, ticket, None, None, None, 0, ctypes.byref(n)))
        q = np.zeros(n.value, np.uint32)
        g = np.zeros(n.value, np.uint32)
        c = np.zeros(n.value, np.uint64)
        check(lib().sigmo_server_pairs(self._h, ticket, q.ctypes.data, g.ctypes.data, c.ctypes.data, n.value, ctypes.byref(n)))
        return q, g, c

    def release(self, ticket: int):
        check(lib().sigmo_server_release(self._h, ticket))

    def stats(self) -> dict:
        st = _L.ServerStatsC()
        check(lib().sigmo_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _L.ServerStatsC._fields_}

    def close(self):
        if getattr(self, "_h", None):
            check(lib().sigmo_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


candidates = SimpleNamespace(Candidates=Candidates)
signature = SimpleNamespace(Signature=Signature)
isomorphism = SimpleNamespace(
    filter=SimpleNamespace(filterCandidates=filterCandidates, refineCandidates=refineCandidates),
    mapping=SimpleNamespace(GMCR=GMCR),
    join=SimpleNamespace(joinCandidates=joinCandidates, joinWildcardCandidates=joinWildcardCandidates),
)
