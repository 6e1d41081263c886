"""Tet-centroid labels from a sparse UDF brick grid on the GPU (replaces
SparseUDF.sample_tet_labels, native/vdb/wtivo_vdb.cpp:1519-1584): labels
and samples bit-identical to the oracle's restatement for every placement
of the inputs, through the C ABI and the module's BrickUDF."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from test_oracle import label_case

pytestmark = pytest.mark.gpu


def _dev_grid(grid):
    g = dict(grid)
    g["table"] = torch.from_numpy(np.ascontiguousarray(grid["table"]).reshape(-1)).cuda()
    g["values"] = torch.from_numpy(np.ascontiguousarray(grid["values"]).reshape(-1)).cuda()
    return g


@pytest.mark.parametrize("bmin,bmax,padding", [((0, 0, 0), (1, 1, 1), 0.0),
                                               ((-0.1, 0.0, 0.05), (1.2, 1.0, 0.95), 0.0),
                                               ((0, 0, 0), (1, 1, 1), 0.03)])
def test_labels_match_oracle(built, bmin, bmax, padding):
    import gpupr_capi

    V, F, grid, TV, T = label_case(60, seed=2)
    thr = 1.0 / 128 - 1e-4
    want, ws = orc.sample_tet_labels(grid, TV, T, bmin, bmax, padding, thr)
    for g in (grid, _dev_grid(grid)):
        lab, s = gpupr_capi.sample_tet_labels(g, TV, T, bmin, bmax, padding, thr)
        assert np.array_equal(lab, want)
        assert np.array_equal(s.view(np.uint32), ws.view(np.uint32))
    lab, s = gpupr_capi.sample_tet_labels(_dev_grid(grid), torch.from_numpy(TV).cuda(),
                                          torch.from_numpy(T).cuda(), bmin, bmax, padding, thr,
                                          device_out=True)
    assert np.array_equal(lab.cpu().numpy(), want)
    assert np.array_equal(s.cpu().numpy().view(np.uint32), ws.view(np.uint32))
    assert 0 < int(want.sum()) < len(want)


def test_brick_udf_module(built):
    import wtivo_gpupr

    V, F, grid, TV, T = label_case(50, seed=4)
    thr = 1.0 / 128 - 1e-4
    want, _ = orc.sample_tet_labels(grid, TV, T, (0, 0, 0), (1, 1, 1), 0.0, thr)
    udf = wtivo_gpupr.BrickUDF(grid["values"], grid["table"], grid["origin"], grid["voxel_size"],
                               float(grid["background"]))
    lab, sec = udf.sample_tet_labels(TV, T, np.zeros(3), np.ones(3), 0.0, thr, 16)
    assert lab.dtype == np.uint8 and np.array_equal(lab, want) and sec >= 0
    lab2, _ = udf.sample_tet_labels(TV, torch.from_numpy(T).cuda(), np.zeros(3), np.ones(3), 0.0, thr)
    assert np.array_equal(lab2, want)
    assert udf.stats()["bricks"] == grid["values"].shape[0]
    with pytest.raises(RuntimeError, match="SparseUDF.sample_tet_labels: tet_vertices must be float64 Nx3"):
        udf.sample_tet_labels(TV[:, :2], T, np.zeros(3), np.ones(3), 0.0, thr)
    with pytest.raises(RuntimeError, match="SparseUDF.sample_tet_labels: tets must be int32 Mx4"):
        udf.sample_tet_labels(TV, T[:, :3], np.zeros(3), np.ones(3), 0.0, thr)
    with pytest.raises(RuntimeError, match="SparseUDF.sample_tet_labels: bbox must have length 3"):
        udf.sample_tet_labels(TV, T, np.zeros(2), np.ones(3), 0.0, thr)
    with pytest.raises(RuntimeError, match="SparseUDF.sample_tet_labels: degenerate bbox"):
        udf.sample_tet_labels(TV, T, np.zeros(3), np.array([1.0, 0.0, 1.0]), 0.0, thr)
    bad = T.copy()
    bad[7, 1] = -1
    with pytest.raises(RuntimeError, match="SparseUDF.sample_tet_labels: tet index out of range"):
        udf.sample_tet_labels(TV, bad, np.zeros(3), np.ones(3), 0.0, thr)
    # the context stays usable after the error
    assert np.array_equal(udf.sample_tet_labels(TV, T, np.zeros(3), np.ones(3), 0.0, thr)[0], want)


def test_outside_and_inactive_bricks_read_background(built):
    import gpupr_capi

    V, F, grid, TV, T = label_case(30, seed=1)
    g = dict(grid)
    tab = grid["table"].copy()
    tab[tab.shape[0] // 2:] = -1                 # half the bricks inactive
    g["table"] = tab
    # a query box twice as large maps half the centroids outside the grid
    want, ws = orc.sample_tet_labels(g, TV, T, (0, 0, 0), (2, 2, 2), 0.0, 0.004)
    lab, s = gpupr_capi.sample_tet_labels(g, TV, T, (0, 0, 0), (2, 2, 2), 0.0, 0.004)
    assert np.array_equal(lab, want) and np.array_equal(s, ws)
    assert np.any(ws == grid["background"])
