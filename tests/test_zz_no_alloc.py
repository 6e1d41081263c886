"""gpupr_solve_reduced_noalloc: the solve for callers that cannot allocate
device memory during the call (their own allocator owns the device heap, or
they must stay out of the CUDA allocator mid-pipeline).  Its scratch is a
static device array in the library, so it must give exactly what the
allocating gpupr_solve_reduced gives, call after call, while the array keeps
the previous call's contents.

Collected last on purpose (file name), so a failure here never hides the
results of the other GPU tests; it also passes run alone in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import cached_graph
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _graph(kind, seed, size):
    g = cached_graph(kind, seed, size)
    return orc.build(g["vertices"], g["tets"], g["neighbors"], g["labels"], g["fill_T"])


def _upload(b):
    nbr = torch.from_numpy(np.ascontiguousarray(b["nbr"])).cuda()
    res = torch.from_numpy(np.ascontiguousarray(b["res"]).view(np.int32)).cuda()
    term = torch.from_numpy(np.ascontiguousarray(b["term"])).cuda()
    return nbr, res, term


def _noalloc(nbr, res, term, part, **kw):
    import gpupr_capi

    st = gpupr_capi.CutStats()
    L = gpupr_capi.lib()
    rc = L.gpupr_solve_reduced_noalloc(
        int(nbr.shape[0]), ctypes.c_void_p(nbr.data_ptr()), ctypes.c_void_p(res.data_ptr()),
        ctypes.c_void_p(term.data_ptr()), ctypes.c_void_p(part.data_ptr()),
        kw.get("period", 1024), kw.get("max_rounds", 2000000), kw.get("local_steps", 8),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(st))
    return rc, st


def test_noalloc_matches_allocating_solve_twice(built):
    """Two calls in a row: a larger graph, then a smaller, different one, so the
    second call runs over the first call's leftover heights, queues, reverse
    slots and pair sums in the shared array.  Each result must equal the
    allocating gpupr_solve_reduced and the BK oracle, and once the array is
    committed (gpupr_noalloc_prepare) no call changes the device's free memory."""
    import gpupr_capi

    L = gpupr_capi.lib()
    nbytes = ctypes.c_uint64(0)
    assert L.gpupr_noalloc_prepare(ctypes.byref(nbytes)) == 0, L.gpupr_last_error()
    assert 40 << 20 <= nbytes.value <= 48 << 20
    graphs = [_graph("lattice", 3, 300_000), _graph("box", 5, 120_000)]
    assert len(graphs[1]["nbr"]) < len(graphs[0]["nbr"])
    for b in graphs:
        n = len(b["nbr"])
        assert n <= 1 << 20
        # the existing, allocating entry point
        nbr0, res0, term0 = _upload(b)
        part0, st0, _ = gpupr_capi.solve_reduced(nbr0, res0, term0)
        nbr, res, term = _upload(b)
        part = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc, st = _noalloc(nbr, res, term, part)
        torch.cuda.synchronize()
        assert rc == 0, L.gpupr_last_error()
        assert torch.cuda.mem_get_info()[0] == free_before
        assert st.raw_flow == st0["raw_flow"]
        assert np.array_equal(part.cpu().numpy(), part0)
        f_bk, _, _, p_bk = orc.maxflow_bk(b["nbr"], b["res"], b["term"])
        assert st.raw_flow == f_bk and np.array_equal(part.cpu().numpy(), p_bk)


def test_noalloc_rejects_oversized_graph(built):
    import gpupr_capi

    n = (1 << 20) + 1
    nbr = torch.full((n, 4), -1, dtype=torch.int32, device="cuda")
    res = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    term = torch.zeros(n, dtype=torch.int32, device="cuda")
    part = torch.zeros(n, dtype=torch.uint8, device="cuda")
    rc, _ = _noalloc(nbr, res, term, part)
    assert rc == 1
    assert b"static scratch limit" in gpupr_capi.lib().gpupr_last_error()
