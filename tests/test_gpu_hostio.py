"""Host <-> device copies of the boundary: the topology upload that replaces
wtivo.py:284-309 (topology_to_cuda_chunked) and the staged copies of host
vertices/labels in and labels out.  Results must equal numpy's own
conversion (np.ascontiguousarray(a, dtype=np.int32)) and the all-device cut."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cached_graph, to_cuda

pytestmark = pytest.mark.gpu


def _layouts(rng, n):
    a32 = rng.integers(-(2**31), 2**31 - 1, size=(n, 4), dtype=np.int64).astype(np.int32)
    a64 = rng.integers(-(2**40), 2**40, size=(n, 4), dtype=np.int64)   # narrowed like astype
    return {
        "c_int32": a32,
        "fortran_int32": np.asfortranarray(a32),
        "c_int64_wide": a64,
        "fortran_int64": np.asfortranarray(a64),
        "row_slice": np.concatenate([a32, a32])[::2],
        "uint32": a32.view(np.uint32),
        "reversed_rows": a32[::-1],
        "int16": a32.astype(np.int16),
    }


@pytest.mark.parametrize("n", [0, 1, 1000, 3_000_001])
def test_topology_upload_matches_numpy(built, n):
    import torch

    import gpupr_capi
    import wtivo_gpupr

    rng = np.random.default_rng(n)
    for name, a in _layouts(rng, n).items():
        want = np.ascontiguousarray(a, dtype=np.int32)
        t = wtivo_gpupr.topology_to_cuda_chunked(a, name)
        assert t.is_cuda and t.dtype == torch.int32 and tuple(t.shape) == (n, 4) and t.is_contiguous()
        assert np.array_equal(t.cpu().numpy(), want), name
        if a.dtype.itemsize in (4, 8) and a.dtype.kind in "iu":
            out = torch.full((n, 4), -7, dtype=torch.int32, device="cuda")
            gpupr_capi.upload_topology(a, out)
            assert np.array_equal(out.cpu().numpy(), want), name


def test_host_and_device_arrays_give_the_same_cut(built):
    """~3M tets: vertices (>1 MiB), labels and the returned labels go through
    the staged host copies; the cut must equal the all-device call."""
    import torch

    import gpupr_capi
    import wtivo_gpupr

    g = cached_graph("lattice", 11, 3_000_000)
    tets, nbrs, V, L = to_cuda(g["tets"], g["neighbors"], g["vertices"], g["labels"])
    dev_out, dev_st = gpupr_capi.graph_cut(V, tets, nbrs, L, 10.0)
    host_out, host_st = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], 10.0)
    assert isinstance(host_out, np.ndarray)
    assert np.array_equal(host_out, dev_out.cpu().numpy())
    assert host_st["adjusted_flow"] == dev_st["adjusted_flow"]
    # the drop-in call with a module-uploaded topology
    t2 = wtivo_gpupr.topology_to_cuda_chunked(g["tets"], "tets")
    n2 = wtivo_gpupr.topology_to_cuda_chunked(np.asfortranarray(g["neighbors"]), "neighbors")
    r = wtivo_gpupr.graph_cut_fast(g["vertices"], t2, n2, g["labels"], 10.0)
    assert np.array_equal(r[0], host_out) and r[1] == host_st["adjusted_flow"]
    torch.cuda.synchronize()
