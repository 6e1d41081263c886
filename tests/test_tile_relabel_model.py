"""A host model of the persistent engine's tiled relabels (tile_relabel and
the tile-step loop of k_solve_persistent in csrc/push_relabel.cu), checked
against a plain level-synchronous BFS.

The device code processes a step's queued tiles in parallel, one block per
tile.  The model processes them one after another in a random order, and
each label it reads from another tile is, at random, either the value at the
start of the step or the latest one, which covers what a block can see while
other blocks write.  What it pins down is the design argument the kernel
relies on:

* the labels end as the exact BFS distances (reachability included) for any
  tile size, processing order and staleness of the labels read across tiles;
* a tile enters a step's queue at most once (the stamps), so a queue never
  holds more than the number of tiles;
* the seeds' tiles are the only tiles queued at the start; in the first step
  every labelled node announces its label to the other tiles (a seed's label
  is set before the step, so it never "goes down" there).
"""
from __future__ import annotations

import numpy as np
import pytest

from test_bfs_step_model import UNVIS, bfs_distances, grid_graph, reverse_residual


def tiled_relabel(nbr, res, seeds, tile, rng):
    n = len(nbr)
    h = np.where(seeds, 1, UNVIS).astype(np.uint64)
    ntiles = (n + tile - 1) // tile
    stamp = np.zeros(ntiles, np.int64)
    step = 1
    queue = []
    for t in sorted({int(v) // tile for v in np.nonzero(seeds)[0]}):
        stamp[t] = step
        queue.append(t)
    steps = 0
    while queue:
        steps += 1
        assert len(queue) == len(set(queue)) <= ntiles
        snap = h.copy()
        nxt = []
        for t in rng.permutation(queue):
            b, e = int(t) * tile, min(n, (int(t) + 1) * tile)
            h0 = h[b:e].copy()
            lab = h0.copy()
            low = np.zeros(e - b, bool)
            # arcs into other tiles: their label now or at the start of the step
            for j, u in enumerate(range(b, e)):
                for k in range(4):
                    v = nbr[u, k]
                    if v < 0 or res[u, k] == 0 or b <= v < e:
                        continue
                    hv = h[v] if rng.random() < 0.5 else snap[v]
                    if hv != UNVIS and hv + 1 < lab[j]:
                        lab[j] = hv + 1
                        low[j] = True
            # the BFS inside the tile, in worklist rounds from the nodes that
            # went down (in the first step: from every labelled node); the
            # tile was at a fixpoint after its last processing
            work = [j for j in range(e - b) if low[j] or (steps == 1 and lab[j] != UNVIS)]
            while work:
                nxt_work = []
                for j in rng.permutation(work):
                    u = b + int(j)
                    if lab[j] == UNVIS:
                        continue
                    for k in range(4):
                        w = nbr[u, k]
                        if w < 0 or not (b <= w < e) or reverse_residual(nbr, res, u, k) == 0:
                            continue
                        if lab[w - b] > lab[j] + 1:
                            lab[w - b] = lab[j] + 1
                            low[w - b] = True
                            nxt_work.append(w - b)
                work = nxt_work
            # write back the labels that went down; queue the tiles that read
            # them (in the first step every label is new: the seeds' too)
            for j, u in enumerate(range(b, e)):
                if not low[j] and not (steps == 1 and lab[j] != UNVIS):
                    continue
                h[u] = lab[j]
                for k in range(4):
                    w = nbr[u, k]
                    if w < 0 or b <= w < e or reverse_residual(nbr, res, u, k) == 0:
                        continue
                    if h[w] > lab[j] + 1:
                        tw = int(w) // tile
                        if stamp[tw] < step + 1:
                            stamp[tw] = step + 1
                            nxt.append(tw)
        queue = nxt
        step += 1
    return h, steps


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("tile", [1, 7, 32, 64, 1000])
def test_tiled_relabel_gives_exact_distances(seed, tile):
    rng = np.random.default_rng(seed)
    w, hgt = int(rng.integers(8, 30)), int(rng.integers(8, 30))
    nbr, res, seeds = grid_graph(rng, w, hgt)
    want = bfs_distances(nbr, res, seeds)
    got, steps = tiled_relabel(nbr, res, seeds, tile, rng)
    assert np.array_equal(got, want)
    assert steps <= len(nbr) + 1


def test_one_tile_is_one_step():
    rng = np.random.default_rng(11)
    nbr, res, seeds = grid_graph(rng, 20, 20)
    got, steps = tiled_relabel(nbr, res, seeds, 400, rng)
    assert np.array_equal(got, bfs_distances(nbr, res, seeds))
    assert steps == 1


def test_unreached_tiles_keep_unvisited_labels():
    rng = np.random.default_rng(5)
    nbr, res, seeds = grid_graph(rng, 16, 16, p_res=0.0)   # no residual arcs at all
    got, _ = tiled_relabel(nbr, res, seeds, 8, rng)
    assert np.array_equal(got, np.where(seeds, 1, UNVIS).astype(np.uint64))
