"""A host model of the persistent engine's BFS steps (bfs_step_body, the
per-thread chains, and bfs_step_levels_body, the block sub-levels, in
csrc/push_relabel.cu), checked against a plain level-synchronous BFS.

The device code runs a step's queue entries in parallel; the model runs them
one after another in a random order each step, which covers the orders a
parallel step can produce at node granularity.  What it pins down is the
design argument the kernel relies on:

* reachability to the sink is exact whatever the hops, order or propagation
  (it decides the end of the solve and the partition);
* while lowered labels propagate, the labels converge to the BFS distances
  (every label a node ends with is expanded);
* a step queues at most 4 * hops * cnt entries, so the caller's condition
  4 * hops * cnt <= n keeps the queue inside its n entries, and without
  propagation every node is queued at most once per BFS.
"""
from __future__ import annotations

from collections import deque

import numpy as np
import pytest

UNVIS = np.iinfo(np.uint32).max


def grid_graph(rng, w, hgt, p_res=0.7, p_cut=0.1, p_sink=0.02):
    """A w x hgt grid in the 4-slot ELL layout (slot 0: x+1, 1: x-1, 2: y+1,
    3: y-1, -1 = no neighbour) with some edges removed, an independent
    residual per direction, and sink-adjacent seeds."""
    n = w * hgt
    nbr = -np.ones((n, 4), np.int64)
    for y in range(hgt):
        for x in range(w):
            u = y * w + x
            if x + 1 < w and rng.random() >= p_cut:
                nbr[u, 0], nbr[u + 1, 1] = u + 1, u
            if y + 1 < hgt and rng.random() >= p_cut:
                nbr[u, 2], nbr[u + w, 3] = u + w, u
    res = np.where(rng.random((n, 4)) < p_res, 1, 0) * (nbr >= 0)
    seeds = rng.random(n) < p_sink
    if not seeds.any():
        seeds[int(rng.integers(n))] = True
    return nbr, res, seeds


def reverse_residual(nbr, res, u, k):
    """Residual of the arc v -> u for v = nbr[u, k] (its reverse slot is k ^ 1)."""
    return res[nbr[u, k], k ^ 1]


def bfs_distances(nbr, res, seeds):
    """Level-synchronous backward BFS: label 1 at the seeds, +1 per arc v -> u."""
    n = len(nbr)
    h = np.full(n, UNVIS, np.uint64)
    q = deque()
    for s in np.nonzero(seeds)[0]:
        h[s] = 1
        q.append(int(s))
    while q:
        u = q.popleft()
        for k in range(4):
            v = nbr[u, k]
            if v >= 0 and h[v] == UNVIS and reverse_residual(nbr, res, u, k):
                h[v] = h[u] + 1
                q.append(int(v))
    return h


def model_bfs(nbr, res, seeds, rng, hops_max, chain_max):
    """The step loop of k_solve_persistent's relabel with bfs_step_body."""
    n = len(nbr)
    h = np.full(n, UNVIS, np.uint64)
    frontier = [int(s) for s in np.nonzero(seeds)[0]]
    h[frontier] = 1
    queued_once = np.zeros(n, np.int64)
    queued_once[frontier] += 1
    L, exact, steps, all_prop = 1, True, 0, True
    while frontier:
        cnt = len(frontier)
        hops = hops_max if (hops_max > 1 and cnt <= chain_max and 4 * hops_max * cnt <= n) else 1
        propagate = 4 * hops * cnt <= n
        all_prop = all_prop and propagate
        out = []
        order = rng.permutation(cnt)
        for i in order:
            u = frontier[i]
            hu = L if exact else int(h[u])
            hop = 1
            while hu < n:
                cand = hu + 1
                nxt = None
                for k in range(4):
                    v = nbr[u, k]
                    if v < 0 or not reverse_residual(nbr, res, u, k) or h[v] <= cand:
                        continue
                    old = int(h[v])
                    h[v] = cand                       # atomicMin, won
                    if old != UNVIS and not propagate:
                        continue
                    if old == UNVIS:
                        queued_once[v] += 1
                    if hop < hops and nxt is None:
                        nxt = int(v)
                    else:
                        out.append(int(v))
                if nxt is None:
                    break
                u, hu, hop = nxt, cand, hop + 1
        assert len(out) <= 4 * hops * cnt
        if propagate:
            assert len(out) <= n                      # the queue holds n entries
        if hops > 1:
            exact = False
        frontier = out
        L += 1
        steps += 1
    return h, steps, queued_once, all_prop


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("hops", [1, 4, 8])
def test_steps_reach_exactly_and_converge_to_distances(seed, hops):
    rng = np.random.default_rng(seed)
    nbr, res, seeds = grid_graph(rng, 40, 30)
    ref = bfs_distances(nbr, res, seeds)
    h, steps, once, all_prop = model_bfs(nbr, res, seeds, rng, hops, chain_max=len(nbr))
    assert all_prop                                   # every lowered label propagated
    assert np.array_equal(h != UNVIS, ref != UNVIS)   # reachability exact
    assert np.array_equal(h, ref)                     # labels are BFS distances
    assert once.max() <= 1                            # a first label happens once
    levels = int(ref[ref != UNVIS].max())
    if hops == 1:
        assert steps == levels                        # one step per level
    else:
        assert steps < levels                         # chained steps cover several levels


@pytest.mark.parametrize("seed", range(4))
def test_without_propagation_reachability_stays_exact(seed):
    # frontiers too wide for the queue bound (4 * hops * cnt > n) queue first
    # labels only: labels may stay above the distances, reachability may not
    rng = np.random.default_rng(100 + seed)
    nbr, res, seeds = grid_graph(rng, 24, 20, p_sink=0.3)
    ref = bfs_distances(nbr, res, seeds)
    h, _, once, all_prop = model_bfs(nbr, res, seeds, rng, 4, chain_max=len(nbr))
    assert not all_prop
    assert np.array_equal(h != UNVIS, ref != UNVIS)
    assert np.all(h[ref != UNVIS] >= ref[ref != UNVIS])   # path lengths, never below
    assert once.max() <= 1


def model_bfs_levels(nbr, res, seeds, rng, levels, blocks, half, threads=4):
    """The step loop of k_solve_persistent's relabel with bfs_step_levels_body:
    a step deals its frontier to `blocks` blocks of `threads` threads (one
    entry per thread per pass); each block expands its entries, then, for up
    to levels - 1 sub-levels, the nodes it staged itself (stage halves of
    `half` entries; a node that does not fit goes to the next step's queue);
    the last sub-level's stage goes to the next step's queue.  Blocks run one
    after another in a random order, nodes within a sub-level too."""
    n = len(nbr)
    h = np.full(n, UNVIS, np.uint64)
    frontier = [int(s) for s in np.nonzero(seeds)[0]]
    h[frontier] = 1
    queued_once = np.zeros(n, np.int64)
    queued_once[frontier] += 1
    steps, all_prop = 0, True
    while frontier:
        cnt = len(frontier)
        passes = -(-cnt // (blocks * threads))
        ex_max = cnt + (levels - 1) * half * blocks * passes
        propagate = 4 * ex_max <= n
        all_prop = all_prop and propagate
        out, expanded = [], 0

        def expand(u, stage):
            nonlocal expanded
            expanded += 1
            cand = int(h[u]) + 1
            for k in range(4):
                v = nbr[u, k]
                if v < 0 or not reverse_residual(nbr, res, u, k) or h[v] <= cand:
                    continue
                old = int(h[v])
                h[v] = cand                           # atomicMin, won
                if old != UNVIS and not propagate:
                    continue
                if old == UNVIS:
                    queued_once[v] += 1
                if len(stage) < half:
                    stage.append(int(v))
                else:
                    out.append(int(v))                # the stage half is full

        for p in range(passes):
            for b in rng.permutation(blocks):
                lo = (p * blocks + b) * threads
                cur = []
                for i in rng.permutation(range(lo, min(lo + threads, cnt))) if lo < cnt else []:
                    expand(frontier[i], cur)
                for _ in range(levels - 1):
                    if not cur:
                        break
                    nxt = []
                    for u in rng.permutation(cur):
                        expand(int(u), nxt)
                    cur = nxt
                out.extend(cur)
        assert expanded <= ex_max
        assert len(out) <= 4 * ex_max
        if propagate:
            assert len(out) <= n                      # the queue holds n entries
        frontier = out
        steps += 1
    return h, steps, queued_once, all_prop


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("levels,half", [(2, 8), (4, 16), (16, 8), (16, 4)])
def test_block_sublevels_reach_exactly_and_converge(seed, levels, half):
    # sizes where every step's worst case fits the queue, so lowered labels propagate
    rng = np.random.default_rng(200 + seed)
    nbr, res, seeds = grid_graph(rng, 80, 60)
    ref = bfs_distances(nbr, res, seeds)
    h, steps, once, all_prop = model_bfs_levels(nbr, res, seeds, rng, levels, blocks=3, half=half,
                                                threads=64)
    assert np.array_equal(h != UNVIS, ref != UNVIS)   # reachability exact in every case
    assert np.all(h[ref != UNVIS] >= ref[ref != UNVIS])
    if all_prop or levels <= 4:                       # (the small cases always propagate here)
        assert all_prop
        assert np.array_equal(h, ref)                 # lowered labels propagated: distances
    assert once.max() <= 1
    assert steps < int(ref[ref != UNVIS].max())       # sub-levels cover several levels a step


@pytest.mark.parametrize("seed", range(4))
def test_block_sublevels_without_propagation_stay_exact(seed):
    rng = np.random.default_rng(300 + seed)
    nbr, res, seeds = grid_graph(rng, 24, 20, p_sink=0.3)
    ref = bfs_distances(nbr, res, seeds)
    h, _, once, all_prop = model_bfs_levels(nbr, res, seeds, rng, 16, blocks=8, half=64)
    assert not all_prop
    assert np.array_equal(h != UNVIS, ref != UNVIS)
    assert np.all(h[ref != UNVIS] >= ref[ref != UNVIS])
    assert once.max() <= 1
