"""The allocation-free GMCR entry point (sigmo_gmcr_generate_noalloc).

Callers that cannot allocate device memory while the mapping runs (a fixed
arena owned by another allocator, a request path where cudaMalloc/cudaFree are
forbidden after start-up) pass their own output buffers; the entry point keeps
its intermediates in a static device array.  This test compares it, through
the C ABI, with the allocating sigmo_gmcr_generate on two calls in a row, and
checks that a batch larger than the static scratch is refused.

The file sorts last so that a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import sigmo_b200 as sb
from sigmo_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _filtered(queue, qh, dh, R):
    qg, dg = sb.createDeviceCSRGraph(queue, qh), sb.createDeviceCSRGraph(queue, dh)
    cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
    sig = sb.Signature(queue, dg.total_nodes, qg.total_nodes)
    sig.generateDataSignatures(dg)
    sig.generateQuerySignatures(qg)
    sb.filterCandidates(queue, qg, dg, sig, cand)
    for r in range(1, R + 1):
        sig.refineDataSignatures(dg, r)
        sig.refineQuerySignatures(qg, r)
        sb.refineCandidates(queue, qg, dg, sig, cand)
    queue.wait()
    return qg, dg, cand, sig


def _noalloc(queue, qg, dg, cand, d_off, d_idx, capacity):
    total = ctypes.c_uint64(0)
    rc = L.lib().sigmo_gmcr_generate_noalloc(queue._h, qg._h, dg._h, cand._h, ctypes.c_void_p(d_off),
                                             ctypes.c_void_p(d_idx), capacity, ctypes.byref(total))
    return rc, total.value


def test_noalloc_gmcr_matches_allocating_entry_point():
    import torch

    dh = sb.generate_molecules(2500, 10, 40, seed=515)
    qh = sb.generate_queries(40, 3, 10, seed=516)
    queue = sb.Queue(0)
    qg, dg, cand, _sig = _filtered(queue, qh, dh, 3)
    gm = sb.GMCR(queue)
    gm.generateGMCR(qg, dg, cand)
    off_ref, idx_ref = gm.getGMCR()
    assert len(idx_ref) > 0

    # the caller owns the output buffers (allocated here, not by the entry point)
    capacity = len(idx_ref) + 64
    d_off = torch.empty(dg.num_graphs + 1, dtype=torch.int32, device="cuda")
    d_idx = torch.empty(capacity, dtype=torch.int32, device="cuda")
    for call in range(2):
        d_off.fill_(-1)
        d_idx.fill_(-1)
        torch.cuda.synchronize()  # the library's stream does not order with torch's
        rc, total = _noalloc(queue, qg, dg, cand, d_off.data_ptr(), d_idx.data_ptr(), capacity)
        assert rc == 0, L.last_error()
        queue.wait()
        assert total == len(idx_ref), f"call {call}"
        assert np.array_equal(d_off.cpu().numpy().view(np.uint32), off_ref), f"call {call}"
        got = d_idx.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[:total], idx_ref), f"call {call}"
        assert (got[total:] == np.uint32(0xFFFFFFFF)).all(), f"call {call} wrote past the admitted pairs"

    # an index buffer that is too small is reported with the needed size
    rc, total = _noalloc(queue, qg, dg, cand, d_off.data_ptr(), d_idx.data_ptr(), 1)
    assert rc == 1 and total == len(idx_ref)


def test_noalloc_gmcr_refuses_batches_beyond_its_scratch():
    import torch

    # 300,000 one-vertex data graphs x 1,000 one-vertex queries: the
    # non-empty matrix alone needs 1,000 x 9,375 x 4 bytes > 32 MiB.
    dh = sb.io.parse("n#1 l#1 0 8 e#0\n" * 300_000)
    qh = sb.io.parse("n#1 l#1 0 8 e#0\n" * 1_000)
    queue = sb.Queue(0)
    qg, dg = sb.createDeviceCSRGraph(queue, qh), sb.createDeviceCSRGraph(queue, dh)
    cand = sb.Candidates(queue, qg.total_nodes, dg.total_nodes)
    d_off = torch.empty(dg.num_graphs + 1, dtype=torch.int32, device="cuda")
    d_idx = torch.empty(16, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(queue, qg, dg, cand, d_off.data_ptr(), d_idx.data_ptr(), 16)
    assert rc == 4  # SIGMO_ERR_DOMAIN
    assert "static scratch" in L.last_error()
