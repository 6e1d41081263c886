"""Seeded input generators: CelloCut slot convention and determinism."""
from __future__ import annotations

import numpy as np
import pytest

import synth

LUT = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])


def check_slots(T, Nb):
    for fi in range(4):
        i = np.nonzero(Nb[:, fi] >= 0)[0]
        j = Nb[i, fi]
        rows = Nb[j]
        k = np.argmax(rows == i[:, None], axis=1)
        assert np.all(rows[np.arange(len(i)), k] == i), "asymmetric adjacency"
        fa = np.sort(T[i][:, LUT[fi]], axis=1)
        fb = np.sort(T[j][np.arange(len(j))[:, None], LUT[k]], axis=1)
        assert np.array_equal(fa, fb), "slot does not share the LUT face"


def test_lattice_slots_and_hull():
    V, T, Nb = synth.lattice_cells((5, 4, 3), (0, 0, 0), (1, 1, 1), seed=3)
    assert T.shape == (360, 4)
    check_slots(T, Nb)
    # hull faces = boundary of the box: 2 triangles per boundary square
    assert int((Nb < 0).sum()) == 2 * 2 * (5 * 4 + 4 * 3 + 5 * 3)


def test_delaunay_slot_map():
    P = np.random.default_rng(0).random((2000, 3))
    T, Nb = synth.delaunay_cells(P)
    check_slots(T, Nb)


def test_determinism():
    a = synth.config1(7, n_points=5000)
    b = synth.config1(7, n_points=5000)
    for k in ("vertices", "tets", "neighbors", "labels"):
        assert np.array_equal(a[k], b[k])
    V1, T1, N1 = synth.lattice_cells((6, 6, 6), (0, 0, 0), (1, 1, 1), seed=11)
    V2, T2, N2 = synth.lattice_cells((6, 6, 6), (0, 0, 0), (1, 1, 1), seed=11)
    assert np.array_equal(V1, V2) and np.array_equal(T1, T2) and np.array_equal(N1, N2)


def test_udf_labels_band():
    mv, mf = synth.icosphere(2, 0.3, (0.5, 0.5, 0.5))
    V, T, Nb = synth.lattice_cells((20, 20, 20), (0, 0, 0), (1, 1, 1), jitter=0.0)
    lab = synth.udf_labels(V, T, mv, mf, 0.04)
    c = V[T].mean(1)
    r = np.linalg.norm(c - 0.5, axis=1)
    assert np.all(lab[np.abs(r - 0.3) < 0.02] == 0)
    assert np.all(lab[np.abs(r - 0.3) > 0.1] == 1)


def test_raw_graph_symmetric():
    g = synth.config4(0, n_points=3000)
    nbr, cap = g["nbr"], g["cap"]
    i = np.repeat(np.arange(len(nbr)), 4).reshape(-1, 4)
    m = nbr >= 0
    rev = synth._reverse_slots_np(nbr)
    back = cap[np.where(m, nbr, 0), np.where(m, rev, 0)]
    assert np.array_equal(np.where(m, cap, 0), np.where(m, back, 0))


def _raw_graph_numpy(P, tets, nbrs, noise):
    """Plain numpy restatement of synth_raw_graph (the check)."""
    lut = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])
    area = np.empty(tets.shape, np.float64)
    for fi in range(4):
        a, b, c = (P[tets[:, lut[fi, k]]] for k in range(3))
        area[:, fi] = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
    valid = nbrs >= 0
    rev = synth._reverse_slots_np(nbrs)
    j = np.where(valid, nbrs, 0)
    other = area[j, np.where(valid, rev, 0)]
    face = np.where(np.arange(len(tets))[:, None] <= j, area, other)
    cap = np.where(valid, np.rint(1e4 * face / area[valid].mean()), 0)
    d = np.linalg.norm(P[tets].mean(1) - 0.5, axis=1) - 0.3 + noise
    return cap, np.rint(100 * np.maximum(0, -d)), np.rint(100 * np.maximum(0, d))


@pytest.mark.parametrize("delaunay", [False, True])
def test_raw_graph_matches_numpy_restatement(delaunay):
    rng = np.random.default_rng(7)
    if delaunay:
        P = rng.random((4000, 3))
        T, Nb = synth.delaunay_cells(P)
    else:
        P, T, Nb = synth.lattice_cells((12, 12, 12), (0, 0, 0), (1, 1, 1), seed=3)
    g = synth.raw_graph_from_cells(P, T, Nb, np.random.default_rng(1))
    noise = np.random.default_rng(1).normal(scale=0.02, size=len(T))
    cap, src, snk = _raw_graph_numpy(P, T, Nb, noise)
    # the mean is summed in another order, so a value at a .5 boundary may round apart
    assert np.abs(g["cap"].astype(np.int64) - cap).max() <= 1
    assert (g["cap"] != cap).mean() < 1e-3
    assert np.abs(g["src"].astype(np.int64) - src).max() <= 1
    assert np.abs(g["snk"].astype(np.int64) - snk).max() <= 1


def test_morton_order_keeps_the_triangulation():
    P = np.random.default_rng(3).random((3000, 3))
    from scipy.spatial import Delaunay

    d = Delaunay(P)
    T0 = d.simplices.astype(np.int32)
    T, Nb = synth.delaunay_cells(P)
    assert sorted(map(tuple, np.sort(T0, 1))) == sorted(map(tuple, np.sort(T, 1)))
    m = Nb >= 0
    rev = synth._reverse_slots_np(Nb)
    assert np.all(Nb[np.where(m, Nb, 0), np.where(m, rev, 0)][m] == np.nonzero(m)[0])
    # slot fi is the tet opposite local vertex 3 - fi: the shared face has the other 3 vertices
    i, k = np.nonzero(m)
    j = Nb[i, k]
    for a, b, kk in zip(i[:500], j[:500], k[:500]):
        face = set(T[a]) - {T[a][3 - kk]}
        assert face <= set(T[b])
    # spatially coherent: neighbour ids lie closer to a cell's own id than in
    # Qhull's order (what the solver's node-ordered passes and caches see)
    N0 = d.neighbors[:, ::-1]

    def spread(nb):
        a, kk = np.nonzero(nb >= 0)
        return np.mean(np.abs(a - nb[a, kk]))

    assert spread(Nb) < 0.5 * spread(N0)
