"""Edge cases of the capacity formula and the solver, GPU against the oracle
(labels, flows and build counts identical): degenerate tets with zero-area
faces, capacities just below the 2^30 limit, fill_T in (-1, 0) where
capacities truncate towards zero, and a graph whose free part falls apart
into many components."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cached_graph, to_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _same_cut(V, T, Nb, L, fill):
    import wtivo_gpupr

    r = wtivo_gpupr.graph_cut_fast(V, *to_cuda(T, Nb), L, fill)
    lab, st = orc.graph_cut(V, T, Nb, L, fill)
    assert np.array_equal(np.asarray(r[0]), lab)
    assert int(r[1]) == st["adjusted_flow"] and int(r[2]) == st["raw_flow"]
    for i, k in ((5, "full_E"), (6, "free_E"), (7, "fixed_source"), (8, "fixed_sink"), (9, "terminal_edges")):
        assert int(r[i]) == st[k], k
    return st


def test_degenerate_tets(built):
    g = cached_graph("lattice", 5, 120_000)
    V = g["vertices"].copy()
    rng = np.random.default_rng(0)
    # collapse 5% of the vertices onto a neighbouring vertex of one of their
    # tets: faces through both become zero-area (capacity 0)
    for t in rng.choice(len(g["tets"]), size=len(V) // 20, replace=False):
        a, b = g["tets"][t, 0], g["tets"][t, 1]
        V[a] = V[b]
    st = _same_cut(V, g["tets"], g["neighbors"], g["labels"], 10.0)
    assert st["free_n"] > 0


def test_capacities_near_the_limit(built):
    g = cached_graph("lattice", 6, 60_000)
    o = orc.build(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)
    top = max(int(o["res"].max()), int(np.abs(o["term"]).max()), 1)
    # capacities scale with the square of the coordinates
    s = float(np.sqrt(0.9 * (2 ** 30) / top))
    V = g["vertices"] * s
    o2 = orc.build(V, g["tets"], g["neighbors"], g["labels"], 10.0)
    assert int(o2["res"].max()) > 2 ** 29
    _same_cut(V, g["tets"], g["neighbors"], g["labels"], 10.0)


@pytest.mark.parametrize("fill", [-0.5, -0.999, 0.0])
def test_fill_between_minus_one_and_zero(built, fill):
    g = cached_graph("box", 4, 60_000)
    _same_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], fill)


def test_many_components(built):
    """Labelling every third lattice layer fixed cuts the free part into
    slabs that share no arc."""
    g = cached_graph("lattice", 7, 90_000)
    L = g["labels"].copy()
    c = g["vertices"][g["tets"]].mean(1)
    z = c[:, 2]
    band = ((z - z.min()) / (np.ptp(z) + 1e-12) * 9).astype(int) % 3 == 0
    L[band] = 0
    _same_cut(g["vertices"], g["tets"], g["neighbors"], L, 10.0)
