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
