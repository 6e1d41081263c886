"""Edge-degree watertight audit on the GPU (replaces is_watertight,
native/core/wtivo_core.cpp:402-464): bad edge groups equal to the oracle's
sort-and-count restatement and to an independent numpy count, for host and
device faces, on defect cases, cut surfaces and a multi-million-face mesh."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import cached_graph, to_cuda
from oracle import oracle as orc
from test_oracle import _numpy_bad_groups, audit_cases

pytestmark = pytest.mark.gpu


def test_audit_defect_cases(built):
    import gpupr_capi
    import wtivo_gpupr

    for name, (F, want) in audit_cases().items():
        ref = orc.edge_audit(F)
        bad, nbytes = gpupr_capi.edge_audit(F)
        assert bad == ref, name
        assert nbytes > 0
        dev_bad, _ = gpupr_capi.edge_audit(torch.from_numpy(np.ascontiguousarray(F, np.int32)).cuda())
        assert dev_bad == ref, name
        wt, b, sec, nb = wtivo_gpupr.is_watertight(F, 16)
        assert (wt, b) == (ref == 0, ref) and sec >= 0 and nb == nbytes, name


def test_audit_errors(built):
    import gpupr_capi
    import wtivo_gpupr

    with pytest.raises(gpupr_capi.GpuprError, match="negative vertex index"):
        gpupr_capi.edge_audit(np.array([[0, 1, 2], [0, -3, 1]], np.int32))
    with pytest.raises(RuntimeError, match="negative vertex index"):
        wtivo_gpupr.is_watertight(np.array([[0, 1, -1]], np.int32))
    # the context stays usable
    assert gpupr_capi.edge_audit(np.array([[0, 1, 2]], np.int32))[0] == 3


@pytest.mark.parametrize("kind,seed,size", [("proxy", 0, 20_000), ("lattice", 2, 80_000),
                                            ("box", 4, 60_000)])
def test_audit_of_cut_surfaces(built, kind, seed, size):
    """The path's own output: the cut surface, audited on the device."""
    import gpupr_capi
    import wtivo_gpupr

    g = cached_graph(kind, seed, size)
    lab, _ = orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    V, F = wtivo_gpupr.surface_extraction_topology_cuda(lab, g["vertices"], tets, nbrs)
    ref = orc.edge_audit(F)
    assert ref == _numpy_bad_groups(F)
    assert gpupr_capi.edge_audit(F)[0] == ref
    assert wtivo_gpupr.is_watertight(torch.from_numpy(F).cuda())[1] == ref


def test_audit_large_mesh(built):
    """A closed 5.2M-face sphere has no bad edge; dropping faces in patches
    gives the numpy count exactly."""
    import gpupr_capi
    import synth

    V, F = synth.icosphere(9)
    assert gpupr_capi.edge_audit(F)[0] == 0
    rng = np.random.default_rng(3)
    Fh = synth.delete_faces(F, 0.01, rng)
    assert gpupr_capi.edge_audit(torch.from_numpy(np.ascontiguousarray(Fh)).cuda())[0] == \
        _numpy_bad_groups(Fh)
