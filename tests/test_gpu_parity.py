"""GPU parity: the CUDA path against the CPU oracle on the same seeded inputs.

Integer capacities make every comparison exact: labels, flows and all build
arrays must be identical (no tolerance)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import cached_graph, to_cuda
from gpu_helpers import cut_capacity, np_, residual_consistent
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CASES = [("proxy", 0, 20_000), ("proxy", 1, 60_000), ("lattice", 2, 80_000),
         ("lattice", 3, 300_000), ("box", 4, 60_000), ("torus", 5, 60_000)]


@pytest.fixture(scope="module")
def gp(built):
    import wtivo_gpupr

    return wtivo_gpupr


@pytest.mark.parametrize("kind,seed,size", CASES)
def test_graph_cut_fast_matches_oracle(gp, kind, seed, size):
    g = cached_graph(kind, seed, size)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    r = gp.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], g["fill_T"])
    lab, st = orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], g["fill_T"])
    assert len(r) == 18
    assert np.array_equal(np.asarray(r[0]), lab)
    assert int(r[1]) == st["adjusted_flow"] and int(r[2]) == st["raw_flow"]
    assert (int(r[5]), int(r[6]), int(r[7]), int(r[8]), int(r[9])) == (
        st["full_E"], st["free_E"], st["fixed_source"], st["fixed_sink"], st["terminal_edges"])
    assert int(r[10]) == 16 and int(r[15]) == 8
    assert int(r[13]) == len(g["tets"]) * 4 + st["free_n"] * 4


@pytest.mark.parametrize("kind,seed,size", CASES[:3])
def test_build_is_byte_identical(built, kind, seed, size):
    import gpupr_capi

    g = cached_graph(kind, seed, size)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    d = gpupr_capi.build_reduced(g["vertices"], tets, nbrs, g["labels"], g["fill_T"])
    o = orc.build(g["vertices"], g["tets"], g["neighbors"], g["labels"], g["fill_T"])
    assert np.array_equal(d["full_to_free"], o["full_to_free"])
    assert np.array_equal(d["free_old"], o["free_old"])
    assert np.array_equal(d["nbr"], o["nbr"])
    assert np.array_equal(d["res"], o["res"])
    assert np.array_equal(d["term"], o["term"])
    rev = orc.reverse_slots(o["nbr"])
    packed = np.zeros(len(rev), np.uint8)
    for k in range(4):
        packed |= (np.where(rev[:, k] == 255, 0, rev[:, k]) << (2 * k)).astype(np.uint8)
    assert np.array_equal(d["rev"], packed)
    for k in ("free_n", "fixed_source", "fixed_sink", "full_refs", "free_refs", "terminal_edges",
              "terminal_base_flow"):
        key = "free_n" if k == "free_n" else k
        assert d["info"][k] == o["info"][key], k


@pytest.mark.parametrize("kind,seed,size", CASES[1:4])
def test_solver_invariants(built, kind, seed, size):
    import gpupr_capi

    g = cached_graph(kind, seed, size)
    o = orc.build(g["vertices"], g["tets"], g["neighbors"], g["labels"], g["fill_T"])
    f_bk, _, _, p_bk = orc.maxflow_bk(o["nbr"], o["res"], o["term"])
    nbr, res, term = to_cuda(o["nbr"], o["res"].view(np.int32), o["term"])
    cap0, term0 = res.clone(), term.clone()
    part, st, exc = gpupr_capi.solve_reduced(nbr, res, term, want_excess=True)
    assert st["raw_flow"] == f_bk
    assert np.array_equal(part, p_bk)
    # feasibility: residuals non-negative and pairwise conserved
    assert int((res < 0).sum()) == 0            # residuals stay below 2^31 here
    assert residual_consistent(nbr, cap0, res)
    # preflow conservation: sum of initial excess = sink flow + remaining excess
    assert int(term0.clamp_min(0).long().sum()) == st["raw_flow"] + int(exc.sum())
    assert int(exc.min()) >= 0
    # no node with excess reaches the sink; sink arcs only lost capacity
    p = torch.from_numpy(part).cuda()
    assert int(((exc > 0) & (p == 1)).sum()) == 0
    assert bool(torch.all((term0 >= 0) | ((term >= term0) & (term <= 0))))
    # max-flow min-cut certificate on the original capacities
    assert cut_capacity(nbr, cap0, term0, p) == st["raw_flow"]


@pytest.mark.parametrize("opt", [dict(local_steps=1), dict(local_steps=32),
                                 dict(global_relabel_period=0), dict(global_relabel_period=16),
                                 dict(blocks_per_sm=1, round_batch=3, bfs_batch=2),
                                 dict(work_relabel_factor=0.05), dict(engine=1), dict(engine=2),
                                 dict(engine=2, blocks_per_sm=1), dict(engine=2, local_steps=1),
                                 dict(engine=2, global_relabel_period=-1, work_relabel_factor=0.1),
                                 dict(chain_hops=1), dict(chain_hops=2), dict(chain_hops=64),
                                 dict(chain_hops=64, local_steps=1, blocks_per_sm=1),
                                 dict(bfs_block_levels=1, bfs_chain_hops=1), dict(bfs_block_levels=1, bfs_chain_hops=16),
                                 dict(bfs_tail_max=1024), dict(bfs_tail_max=8, blocks_per_sm=1),
                                 dict(discharge_warp_aggregate=1),
                                 dict(bfs_block_levels=1, bfs_chain_max_frontier=1 << 30),
                                 dict(bfs_block_levels=1, bfs_chain_max_frontier=1 << 30, bfs_chain_hops=8),
                                 dict(discharge_warp_aggregate=1, chain_hops=1, local_steps=32),
                                 dict(bfs_tail_max=1024, bfs_block_levels=1, bfs_chain_hops=1, work_relabel_factor=0.05),
                                 dict(bfs_bottom_up=1), dict(bfs_bottom_up=1, bfs_bottom_up_ratio=64.0),
                                 dict(bfs_bottom_up=1, bfs_bottom_up_ratio=1e9, blocks_per_sm=1),
                                 dict(bfs_bottom_up=1, bfs_bottom_up_ratio=1e9, work_relabel_factor=0.05),
                                 dict(relabel_tiles=1), dict(relabel_tiles=-1),
                                 dict(relabel_tiles=1, blocks_per_sm=1),
                                 dict(relabel_tiles=1, work_relabel_factor=0.05),
                                 dict(relabel_tiles=1, discharge_warp_aggregate=1),
                                 dict(relabel_tiles=1, bfs_bottom_up=1, bfs_tail_max=1024),
                                 dict(relabel_tiles=1, engine=1),
                                 dict(bfs_block_levels=1), dict(bfs_block_levels=4), dict(bfs_block_levels=2, blocks_per_sm=1),
                                 dict(bfs_block_levels=16, work_relabel_factor=0.05),
                                 dict(bfs_in_arc_masks=1), dict(bfs_in_arc_masks=-1),
                                 dict(bfs_in_arc_masks=1, bfs_block_levels=1),
                                 dict(bfs_in_arc_masks=1, bfs_bottom_up=1, bfs_bottom_up_ratio=1e9)])
def test_options_do_not_change_the_cut(built, opt):
    import gpupr_capi

    g = cached_graph("lattice", 3, 300_000)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    base, st0 = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"])
    out, st = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"],
                                   opts=gpupr_capi.options(**opt))
    assert np.array_equal(out, base)
    assert st["adjusted_flow"] == st0["adjusted_flow"]


def test_step_histograms_add_up(built):
    """The persistent engine's per-class counters cover every discharge round
    and BFS step of a solve, and their times fit inside the solve; with the
    bottom-up switch forced on, the default (block sub-level) BFS steps hand
    over to bottom-up steps, and the cut stays the same."""
    import gpupr_capi

    g = cached_graph("lattice", 3, 300_000)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    base, st = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"])
    assert int(st["engine"]) == 2
    assert sum(st["discharge_rounds_by_active"]) == int(st["rounds"])
    assert sum(st["bfs_steps_by_frontier"]) + int(st["bottom_up_steps"]) >= 1
    assert 0.0 < sum(st["discharge_ms_by_active"]) <= st["solve_device_ms"]
    assert sum(st["bfs_ms_by_frontier"]) <= st["solve_device_ms"]
    out, st2 = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], g["fill_T"],
                                    opts=gpupr_capi.options(bfs_bottom_up=1, bfs_bottom_up_ratio=64.0))
    assert int(st2["bottom_up_steps"]) > 0
    assert np.array_equal(out, base) and st2["adjusted_flow"] == st["adjusted_flow"]


def test_device_resident_inputs(built):
    import gpupr_capi

    g = cached_graph("proxy", 1, 60_000)
    tets, nbrs, V, L = to_cuda(g["tets"], g["neighbors"], g["vertices"], g["labels"])
    out, st = gpupr_capi.graph_cut(V, tets, nbrs, L, 10.0)
    ref, st2 = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], 10.0)
    assert np.array_equal(np_(out), ref) and st["adjusted_flow"] == st2["adjusted_flow"]


@pytest.mark.parametrize("seed,delaunay", [(0, True), (1, False)])
def test_raw_integer_graph(built, seed, delaunay):
    import gpupr_capi
    import synth

    g = synth.config4(seed, n_points=30_000, use_delaunay=delaunay)
    src = g["src"].astype(np.int64)
    snk = g["snk"].astype(np.int64)
    term = (src - snk).astype(np.int32)
    base = int(np.minimum(src, snk).sum())
    f_bk, _, _, p_bk = orc.maxflow_bk(g["nbr"], g["cap"], term)
    nbr, cap, s, k = to_cuda(g["nbr"], g["cap"].view(np.int32), g["src"].view(np.int32),
                             g["snk"].view(np.int32))
    flow, part, st = gpupr_capi.solve_ell(nbr, cap, s, k)
    assert flow == f_bk + base
    assert np.array_equal(np_(part), p_bk)


def test_surface_matches_oracle(gp):
    g = cached_graph("proxy", 1, 60_000)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    lab = np.asarray(gp.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], 10.0)[0])
    V, F = gp.surface_extraction_topology_cuda(lab, g["vertices"], tets, nbrs)
    V2, F2 = orc.surface(lab, g["vertices"], g["tets"], g["neighbors"])
    assert F.dtype == np.int32 and V.dtype == np.float64
    assert np.array_equal(F, F2) and np.array_equal(V, V2)


def test_all_fixed_returns_16_tuple_and_empty(gp):
    g = cached_graph("proxy", 0, 20_000)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    zero = np.zeros(len(g["labels"]), np.uint8)
    r = gp.graph_cut_fast(g["vertices"], tets, nbrs, zero, 10.0)
    assert len(r) == 16 and np.array_equal(np.asarray(r[0]), zero)
    assert int(r[7]) == len(zero) and int(r[8]) == 0
    e = torch.zeros((0, 4), dtype=torch.int32, device="cuda")
    r = gp.graph_cut_fast(g["vertices"], e, e, np.zeros(0, np.uint8), 10.0)
    assert len(r) == 16 and len(r[0]) == 0


def test_reference_errors(gp):
    g = cached_graph("proxy", 0, 20_000)
    V, T, Nb, L = g["vertices"], g["tets"], g["neighbors"], g["labels"]
    bad = Nb.copy()
    bad[5, 0] = len(bad) + 10
    with pytest.raises(RuntimeError, match="neighbor out of range"):
        gp.graph_cut_fast(V, *to_cuda(T, bad), L, 10.0)
    odd = Nb.copy()
    i = int(np.nonzero((odd >= 0).all(1))[0][0])
    odd[i, 0] = -1
    with pytest.raises(RuntimeError, match="neighbor reference count not even"):
        gp.graph_cut_fast(V, *to_cuda(T, odd), L, 10.0)
    with pytest.raises(RuntimeError, match="invalid graph reduction/capacity state"):
        gp.graph_cut_fast(V * 1e4, *to_cuda(T, Nb), L, 10.0)
    asym = Nb.copy()
    free = np.nonzero((L != 0) & (Nb >= 0).all(1))[0]
    a, b = int(free[0]), int(free[1])
    j = int(asym[a, 0])
    asym[a, 0] = b if b != j else int(free[2])     # keeps the count even, breaks symmetry
    with pytest.raises(RuntimeError):
        gp.graph_cut_fast(V, *to_cuda(T, asym), L, 10.0)
    with pytest.raises(RuntimeError, match="max macro rounds exceeded"):
        gp.graph_cut_fast(V, *to_cuda(T, Nb), L, 10.0, 16, 1024, 1, 8)
    with pytest.raises(RuntimeError, match="tets/neighbors must be int32"):
        gp.graph_cut_fast(V, *[t.long() for t in to_cuda(T, Nb)], L, 10.0)
    # the context stays usable after every error
    r = gp.graph_cut_fast(V, *to_cuda(T, Nb), L, 10.0)
    lab, st = orc.graph_cut(V, T, Nb, L, 10.0)
    assert np.array_equal(np.asarray(r[0]), lab)


def test_bounded_wait_returns_timeout(built):
    import gpupr_capi

    rc = gpupr_capi.bounded_wait_selftest(100_000)
    assert rc == 12          # GPUPR_ERR_TIMEOUT, no fault, no hang
    torch.cuda.synchronize()
    x = torch.ones(4, device="cuda") * 2
    assert float(x.sum()) == 8.0


def test_repeatable(gp):
    g = cached_graph("lattice", 3, 300_000)
    tets, nbrs = to_cuda(g["tets"], g["neighbors"])
    a = gp.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], 10.0)
    b = gp.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], 10.0)
    assert np.array_equal(np.asarray(a[0]), np.asarray(b[0])) and int(a[1]) == int(b[1])
