"""Autotuner: picks the persistent engine's blocks per SM and relabel work
factor for a graph's size class; later cuts use the entry, and the cut is
the same whatever the choice."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import cached_graph, to_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_autotune_then_cut(built):
    import gpupr_capi

    g = cached_graph("lattice", 3, 300_000)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    gpupr_capi.set_tune_table([])
    base, st0 = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"])
    e = gpupr_capi.autotune(g["vertices"], tets, nbrs, g["labels"], g["fill_T"], reps=2)
    k = int(st0["free_n"]).bit_length() - 1
    assert e["size_class"] == k
    assert e["blocks_per_sm"] in (1, 2, 3, 4) and e["work_relabel_factor"] in (0.25, 0.5, 1.0, 2.0)
    assert 0 < e["solve_ms"] <= e["default_ms"] * 1.5
    assert [t["size_class"] for t in gpupr_capi.tune_table()] == [k]
    out, st = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"])
    assert np.array_equal(out, base) and st["adjusted_flow"] == st0["adjusted_flow"]
    assert st["solve_blocks_per_sm"] == e["blocks_per_sm"]
    assert st["relabel_work_factor"] == e["work_relabel_factor"]
    assert (st["chain_hops"], st["chain_max_active"]) == (e["chain_hops"], e["chain_max_active"])
    # explicit options still win over the table
    _, st2 = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"],
                                  opts=gpupr_capi.options(blocks_per_sm=3, work_relabel_factor=0.25))
    assert st2["solve_blocks_per_sm"] == 3 and st2["relabel_work_factor"] == 0.25
    gpupr_capi.set_tune_table([])
    _, st3 = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"])
    assert st3["solve_blocks_per_sm"] == st0["solve_blocks_per_sm"]


def test_batch_autotune_keeps_cuts_and_fills_its_bucket(built):
    """The batch tuner times the segmented solve of one batch and keeps an
    entry for the batch's size bucket; a batch cut with that entry gives every
    graph its own cut."""
    import gpupr_capi

    graphs = [cached_graph("proxy", 0, 20_000), cached_graph("box", 4, 60_000),
              cached_graph("torus", 5, 60_000), cached_graph("lattice", 2, 80_000)]
    toff, voff, V, T, Nb, L = gpupr_capi.pack_batch(graphs)
    t, n = torch.from_numpy(T).cuda(), torch.from_numpy(Nb).cuda()
    old = gpupr_capi.batch_tune_table()
    try:
        e = gpupr_capi.autotune_batch(toff, voff, V, t, n, L, 10.0, reps=1)
        assert e["blocks_per_sm"] >= 1 and e["solve_ms"] > 0 and e["solve_ms"] <= e["default_ms"] * 1.5
        assert any(x["size_class"] == e["size_class"] for x in gpupr_capi.batch_tune_table())
        out, items, st = gpupr_capi.graph_cut_batch(toff, voff, V, t, n, L, 10.0)
        assert st["solve_blocks_per_sm"] == e["blocks_per_sm"] and st["chain_hops"] == e["chain_hops"]
        for k, g in enumerate(graphs):
            lab, ost = orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)
            assert np.array_equal(out[int(toff[k]):int(toff[k + 1])], lab), k
            assert items[k]["adjusted_flow"] == ost["adjusted_flow"]
    finally:
        gpupr_capi.set_batch_tune_table(old)
