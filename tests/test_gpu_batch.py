"""Batched cuts: a batch of independent graphs solved as one must give every
graph exactly its own cut (labels and max flow) as if cut alone."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import cached_graph
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _graphs():
    gs = [cached_graph("proxy", 0, 20_000), cached_graph("lattice", 2, 80_000),
          cached_graph("box", 4, 60_000), cached_graph("torus", 5, 60_000),
          cached_graph("proxy", 1, 60_000)]
    return gs


def _run_batch(graphs, **kw):
    import gpupr_capi

    toff, voff, V, T, Nb, L = gpupr_capi.pack_batch(graphs)
    t = torch.from_numpy(T).cuda()
    n = torch.from_numpy(Nb).cuda()
    return toff, gpupr_capi.graph_cut_batch(toff, voff, V, t, n, L, 10.0, **kw)


@pytest.mark.parametrize("engine,bottom_up,tail,tiles", [(1, 0, 0, 0), (2, 0, 0, 0), (2, 1, 0, 0),
                                                         (2, 0, 1024, 0), (2, 0, 0, 1), (2, 0, 0, -1)])
def test_batch_equals_individual_cuts(built, engine, bottom_up, tail, tiles):
    import gpupr_capi

    graphs = _graphs()
    toff, (out, items, st) = _run_batch(graphs, opts=gpupr_capi.options(
        engine=engine, bfs_bottom_up=bottom_up, bfs_bottom_up_ratio=1e9 if bottom_up else 0.0,
        bfs_tail_max=tail, relabel_tiles=tiles))
    assert len(items) == len(graphs)
    for k, g in enumerate(graphs):
        lab, ost = orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)
        assert np.array_equal(out[int(toff[k]):int(toff[k + 1])], lab), k
        assert items[k]["adjusted_flow"] == ost["adjusted_flow"], k
        assert items[k]["raw_flow"] == ost["raw_flow"], k
        assert items[k]["free_n"] == ost["free_n"] and items[k]["n_tets"] == len(g["tets"])
    assert st["adjusted_flow"] == sum(i["adjusted_flow"] for i in items)


def test_batch_edge_cases(built):
    import gpupr_capi

    g0 = cached_graph("proxy", 0, 20_000)
    empty = dict(vertices=np.zeros((0, 3)), tets=np.zeros((0, 4), np.int32),
                 neighbors=np.zeros((0, 4), np.int32), labels=np.zeros(0, np.uint8))
    fixed = dict(g0)
    fixed["labels"] = np.zeros_like(g0["labels"])       # every tet a fixed source
    toff, (out, items, st) = _run_batch([empty, g0, fixed, empty])
    lab, ost = orc.graph_cut(g0["vertices"], g0["tets"], g0["neighbors"], g0["labels"], 10.0)
    assert items[0]["n_tets"] == 0 and items[0]["adjusted_flow"] == 0
    assert np.array_equal(out[int(toff[1]):int(toff[2])], lab)
    assert items[1]["adjusted_flow"] == ost["adjusted_flow"]
    assert items[2]["free_n"] == 0 and items[2]["adjusted_flow"] == 0
    assert np.array_equal(out[int(toff[2]):int(toff[3])], fixed["labels"])
    # a local neighbor id outside its own graph is rejected, not aliased
    bad = dict(g0)
    bad["neighbors"] = g0["neighbors"].copy()
    i = int(np.nonzero((bad["neighbors"] >= 0).all(1))[0][0])
    bad["neighbors"][i, 0] = len(g0["tets"]) + 5
    with pytest.raises(gpupr_capi.GpuprError, match="neighbor out of range"):
        _run_batch([g0, bad])


def test_batch_device_resident_and_repeatable(built):
    import gpupr_capi

    graphs = _graphs()[:3]
    toff, voff, V, T, Nb, L = gpupr_capi.pack_batch(graphs)
    t, n, v, l = (torch.from_numpy(x).cuda() for x in (T, Nb, V, L))
    o1, it1, _ = gpupr_capi.graph_cut_batch(toff, voff, v, t, n, l, 10.0)
    o2, it2, _ = gpupr_capi.graph_cut_batch(toff, voff, V, t, n, L, 10.0)
    assert np.array_equal(o1.cpu().numpy(), o2) and it1 == it2


def test_batch_retires_finished_graphs(built):
    """Graphs of very different size finish at different relabels: the small
    ones retire while the large one still runs, and every graph keeps exactly
    its own cut (its labels from the relabel at which it retired)."""
    import gpupr_capi

    graphs = [cached_graph("lattice", 2, 80_000)] + [cached_graph("proxy", s, 6_000) for s in range(6)] + \
             [cached_graph("lattice", 3, 300_000)]
    # a relabel every 16 discharge rounds: the small graphs finish after a few
    # relabels while the large one needs many more
    toff, (out, items, st) = _run_batch(graphs, opts=gpupr_capi.options(engine=2, global_relabel_period=16,
                                                                        chain_hops=1))
    assert st["engine"] == 2 and st["global_relabels"] > 2 and st["graphs_retired"] >= 1
    for k, g in enumerate(graphs):
        lab, ost = orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)
        assert np.array_equal(out[int(toff[k]):int(toff[k + 1])], lab), k
        assert items[k]["adjusted_flow"] == ost["adjusted_flow"], k
