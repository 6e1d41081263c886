"""The CPU oracle (the checker) against independent solvers and restatements.

Pins: scipy.sparse.csgraph.maximum_flow and networkx's Boykov-Kolmogorov on
the same reduced graphs; a numpy restatement of the capacity formula
(native/gpupr/wtivo_gpupr_bindings.cpp:65-98); the reference's error texts.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import maximum_flow

from conftest import cached_graph
from oracle import oracle as orc


def scipy_flow(nbr, res, term):
    F = len(nbr)
    s, t = F, F + 1
    v = np.repeat(np.arange(F), 4)
    u = nbr.reshape(-1)
    c = res.reshape(-1).astype(np.int64)
    m = u >= 0
    pos, neg = term > 0, term < 0
    rows = np.concatenate([v[m], np.full(pos.sum(), s), np.nonzero(neg)[0]])
    cols = np.concatenate([u[m], np.nonzero(pos)[0], np.full(neg.sum(), t)])
    caps = np.concatenate([c[m], term[pos], -term[neg].astype(np.int64)]).astype(np.int32)
    G = sp.csr_matrix((caps, (rows, cols)), shape=(F + 2, F + 2))
    return int(maximum_flow(G, s, t).flow_value)


GRAPHS = [("proxy", 0, 20_000), ("proxy", 1, 40_000), ("lattice", 2, 60_000),
          ("box", 3, 30_000), ("torus", 4, 30_000)]


@pytest.mark.parametrize("kind,seed,size", GRAPHS)
def test_bk_matches_scipy_and_pr(kind, seed, size):
    g = cached_graph(kind, seed, size)
    b = orc.build(g["vertices"], g["tets"], g["neighbors"], g["labels"], g["fill_T"])
    f_bk, r_bk, t_bk, p_bk = orc.maxflow_bk(b["nbr"], b["res"], b["term"])
    f_pr, r_pr, t_pr, e_pr, p_pr, rounds, rel = orc.maxflow_pr(b["nbr"], b["res"], b["term"])
    assert f_bk == f_pr == scipy_flow(b["nbr"], b["res"], b["term"])
    # the minimal sink side is unique across maximum flows
    assert np.array_equal(p_bk, p_pr)
    # preflow conservation: initial excess = flow into the sink + what is left
    assert int(np.maximum(b["term"], 0).sum()) == f_pr + int(e_pr.sum())
    # no node holding excess reaches the sink
    assert not np.any((e_pr > 0) & (p_pr == 1))


def test_bk_matches_networkx_tiny():
    nx = pytest.importorskip("networkx")
    g = cached_graph("proxy", 5, 3_000)
    b = orc.build(g["vertices"], g["tets"], g["neighbors"], g["labels"], g["fill_T"])
    nbr, res, term = b["nbr"], b["res"], b["term"]
    G = nx.DiGraph()
    F = len(nbr)
    for v in range(F):
        for k in range(4):
            if nbr[v, k] >= 0:
                G.add_edge(v, int(nbr[v, k]), capacity=int(res[v, k]))
        if term[v] > 0:
            G.add_edge("s", v, capacity=int(term[v]))
        elif term[v] < 0:
            G.add_edge(v, "t", capacity=int(-term[v]))
    from networkx.algorithms.flow import boykov_kolmogorov
    R = boykov_kolmogorov(G, "s", "t")
    f, *_ = orc.maxflow_bk(nbr, res, term)
    assert f == R.graph["flow_value"]


def numpy_capacity(V, tets, labels, nbrs, fill_T):
    """Vectorised restatement of capacity_exact_formula (bindings.cpp:65-98)
    for every (tet, slot) with a neighbor; -1 where the slot is empty."""
    lut = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])
    out = np.full(tets.shape, -1, np.int64)
    for fi in range(4):
        p0, p1, p2 = (V[tets[:, lut[fi, k]]] for k in range(3))
        x1, y1, z1 = (p1[:, i] - p0[:, i] for i in range(3))
        x2, y2, z2 = (p2[:, i] - p0[:, i] for i in range(3))
        cx = y1 * z2 - z1 * y2
        cy = z1 * x2 - x1 * z2
        cz = x1 * y2 - y1 * x2
        area = (5.0e6 * np.sqrt(cx * cx + cy * cy + cz * cz)).astype(np.float32).astype(np.float64)
        j = nbrs[:, fi]
        ok = j >= 0
        lj = labels[np.where(ok, j, 0)]
        pen = np.where(labels != lj, area, area * (1.0 + fill_T))
        out[:, fi] = np.where(ok, np.trunc(pen).astype(np.int64), -1)
    return out


@pytest.mark.parametrize("kind,seed,size", GRAPHS[:3])
def test_build_capacities_match_numpy(kind, seed, size):
    g = cached_graph(kind, seed, size)
    b = orc.build(g["vertices"], g["tets"], g["neighbors"], g["labels"], g["fill_T"])
    caps = numpy_capacity(g["vertices"], g["tets"], g["labels"], g["neighbors"], g["fill_T"])
    old = b["free_old"]
    f2f = b["full_to_free"]
    m = f2f[g["neighbors"][old]]                     # class of each neighbor
    own = caps[old]
    want_res = np.where(m >= 0, own, 0).astype(np.uint32)
    assert np.array_equal(b["res"], want_res)
    assert np.array_equal(b["nbr"], np.where(m >= 0, m, -1))
    src = np.where(m == -2, own, 0).sum(1)
    snk = np.where(m == -3, own, 0).sum(1)
    assert np.array_equal(b["term"], (src - snk).astype(np.int32))
    assert b["info"]["terminal_base_flow"] == int(np.minimum(src, snk).sum())
    # compaction: rank order of free tets
    assert np.all(np.diff(old.astype(np.int64)) > 0)


def test_classification_counts():
    g = cached_graph("proxy", 0, 20_000)
    f2f, old, info = orc.classify(g["neighbors"], g["labels"])
    lab = g["labels"]
    ext = (g["neighbors"] < 0).any(1)
    assert info.fixed_source == int((lab == 0).sum())
    assert info.fixed_sink == int(((lab != 0) & ext).sum())
    assert info.free_n == int(((lab != 0) & ~ext).sum())
    assert info.full_refs == int((g["neighbors"] >= 0).sum())


def test_reference_error_texts():
    g = cached_graph("proxy", 0, 20_000)
    bad = g["neighbors"].copy()
    bad[5, 0] = len(bad) + 10
    with pytest.raises(RuntimeError, match="neighbor out of range"):
        orc.build(g["vertices"], g["tets"], bad, g["labels"], 10.0)
    odd = g["neighbors"].copy()
    i = int(np.nonzero((odd >= 0).all(1))[0][0])
    odd[i, 0] = -1
    with pytest.raises(RuntimeError, match="neighbor reference count not even"):
        orc.build(g["vertices"], g["tets"], odd, g["labels"], 10.0)
    big = g["vertices"] * 1e4          # areas beyond the 30-bit capacity range
    with pytest.raises(RuntimeError, match="invalid graph reduction/capacity state"):
        orc.build(big, g["tets"], g["neighbors"], g["labels"], 10.0)
    tets = g["tets"].copy()
    free = np.nonzero((g["labels"] != 0) & (g["neighbors"] >= 0).all(1))[0]
    tets[free[0], 1] = len(g["vertices"]) + 3
    with pytest.raises(RuntimeError, match="invalid graph reduction/capacity state"):
        orc.build(g["vertices"], tets, g["neighbors"], g["labels"], 10.0)


def test_capacity_edge_semantics():
    V = np.array([[0, 0, 0], [1e-3, 0, 0], [0, 1e-3, 0], [0, 0, 1e-3]], np.float64)
    t = np.array([0, 1, 2, 3], np.int32)
    # 5e6 * 1e-6 = 5 -> float 5.0 -> 5 ; same labels multiply by 1+fill
    assert orc.capacity(V, t, 0, 1, 0, 10.0) == 5
    assert orc.capacity(V, t, 0, 1, 1, 10.0) == 55
    # pen in (-1, 0) truncates to 0 and passes; <= -1 fails
    assert orc.capacity(V, t, 0, 1, 1, -1.1) == 0
    with pytest.raises(RuntimeError):
        orc.capacity(V, t, 0, 1, 1, -1.5)


def numpy_surface(labels, V, tets, nbrs):
    lut = [[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]
    opp = [3, 2, 1, 0]
    raw = []
    for i in np.nonzero(labels == 0)[0]:
        for fi in range(4):
            j = nbrs[i, fi]
            if not (j < 0 or labels[j] != 0):
                continue
            a, b, c = sorted(int(tets[i, k]) for k in lut[fi])
            d = int(tets[i, opp[fi]])
            v0, v1, v2, vp = V[a], V[b], V[c], V[d]
            e1, e2 = v1 - v0, v2 - v0
            cx = e1[1] * e2[2] - e1[2] * e2[1]
            cy = e1[2] * e2[0] - e1[0] * e2[2]
            cz = e1[0] * e2[1] - e1[1] * e2[0]
            p = vp - v0
            vol = cx * p[0] + cy * p[1] + cz * p[2]
            raw.append((a, b, c) if vol < 0 else (a, c, b))
    raw = np.asarray(raw, np.int64).reshape(-1, 3)
    used = np.unique(raw)
    remap = np.full(len(V), -1, np.int64)
    remap[used] = np.arange(len(used))
    return V[used], remap[raw].astype(np.int32)


def test_surface_oracle_matches_numpy():
    g = cached_graph("proxy", 0, 20_000)
    labels, _ = orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)
    V1, F1 = orc.surface(labels, g["vertices"], g["tets"], g["neighbors"])
    V2, F2 = numpy_surface(labels, g["vertices"], g["tets"], g["neighbors"])
    assert np.array_equal(F1, F2)
    assert np.array_equal(V1, V2)
    # every edge of the cut surface is shared by an even number of faces
    e = np.sort(np.concatenate([F1[:, [0, 1]], F1[:, [1, 2]], F1[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert np.all(cnt % 2 == 0)


def _numpy_bad_groups(F):
    """Independent count for the audit: distinct undirected edges whose
    multiplicity is not 2 (numpy unique over packed edge keys)."""
    F = np.asarray(F, np.int64)
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    key = (np.minimum(e[:, 0], e[:, 1]) << 32) | np.maximum(e[:, 0], e[:, 1])
    _, cnt = np.unique(key, return_counts=True)
    return int((cnt != 2).sum())


def audit_cases():
    """Meshes with known edge defects (wtivo_core.cpp:402-464 semantics)."""
    import synth

    rng = np.random.default_rng(7)
    V, F = synth.icosphere(3)
    tet = np.array([[0, 1, 2], [0, 3, 1], [1, 3, 2], [2, 3, 0]], np.int32)
    soup = rng.integers(0, 50, size=(400, 3)).astype(np.int32)
    # the reference's own known-answer case (scripts/verify_install.py:38-41):
    # a tetrahedron shell, every edge of degree 2, so watertight with 0 bad groups
    ref_shell = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    return {
        "reference_install_check_tetra_shell": (ref_shell, 0),
        "closed_icosphere": (F, 0),
        "closed_tetrahedron": (tet, 0),
        "one_face_missing": (F[1:], 3),
        "duplicated_face": (np.concatenate([F, F[:1]]), 3),
        "fin_on_an_edge": (np.concatenate([tet, [[0, 1, 4]]]).astype(np.int32), 3),
        "holed": (synth.holed_icosphere(3, subdiv=3, frac=0.05)[1], None),
        "soup": (soup, None),
        "degenerate_face": (np.array([[0, 0, 1]], np.int32), None),
    }


def test_edge_audit_oracle_matches_numpy():
    for name, (F, want) in audit_cases().items():
        got = orc.edge_audit(F)
        assert got == _numpy_bad_groups(F), name
        if want is not None:
            assert got == want, name
    assert orc.edge_audit(np.zeros((0, 3), np.int32)) == 0
    with pytest.raises(RuntimeError, match="negative vertex index"):
        orc.edge_audit(np.array([[0, 1, -1]], np.int32))


def label_case(n_cubes=40, seed=0, h=1.0 / 128):
    """A sphere-mesh UDF brick grid in the unit query box and a jittered
    lattice of tets over it (the label sampler's inputs)."""
    import synth

    V, F = synth.icosphere(4, 0.3, (0.5, 0.5, 0.5))
    grid = synth.brick_udf(V, F, h, 3.0)
    TV, T, _ = synth.lattice_cells((n_cubes,) * 3, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), seed=seed)
    return V, F, grid, TV, T


def test_label_sampler_oracle_is_the_box_sampler():
    """On a field linear in the voxel index the box sampler is exact; on a
    mesh UDF the sample tracks the exact distance within a voxel."""
    import synth

    V, F, grid, TV, T = label_case()
    lin = dict(grid)
    tab = grid["table"]
    idx = np.argwhere(tab >= 0)
    vals = np.empty_like(grid["values"])
    l = np.arange(8)
    for b, (bx, by, bz) in zip(tab[tuple(idx.T)], idx):
        i = grid["origin"][0] + 8 * bx + l[:, None, None]
        j = grid["origin"][1] + 8 * by + l[None, :, None]
        k = grid["origin"][2] + 8 * bz + l[None, None, :]
        vals[b] = (0.001 * i + 0.002 * j + 0.003 * k).astype(np.float32)
    lin["values"] = vals
    lab, s = orc.sample_tet_labels(lin, TV, T, (0, 0, 0), (1, 1, 1), 0.0, 0.5)
    c = TV[T].mean(1) / grid["voxel_size"]
    # lattice cells fully inside active bricks: every sampled voxel is active
    full = np.zeros(len(T), bool)
    fi = np.floor(c).astype(np.int64) - grid["origin"]
    for d in range(8):
        o = np.array([(d >> 2) & 1, (d >> 1) & 1, d & 1])
        b = (fi + o) >> 3
        okb = np.all((b >= 0) & (b < np.array(tab.shape)), 1)
        act = np.zeros(len(T), bool)
        act[okb] = tab[tuple(b[okb].T)] >= 0
        full = act if d == 0 else (full & act)
    want = 0.001 * c[:, 0] + 0.002 * c[:, 1] + 0.003 * c[:, 2]
    assert full.sum() > 1000
    assert np.allclose(s[full], want[full], rtol=0, atol=2e-5)
    # mesh UDF: sample vs exact centroid distance near the surface
    lab, s = orc.sample_tet_labels(grid, TV, T, (0, 0, 0), (1, 1, 1), 0.0, 1.0 / 128 - 1e-4)
    near = s < grid["background"] * 0.6
    exact0 = synth.udf_labels(TV, T, V, F, 1.0 / 128 - 1e-4)
    assert near.sum() > 1000
    # the sampled field interpolates exact voxel distances: labels agree
    # everywhere except within a voxel of the threshold
    agree = (lab == exact0).mean()
    assert agree > 0.97
    assert set(np.unique(lab)) == {0, 1}


def test_label_sampler_oracle_errors():
    V, F, grid, TV, T = label_case(4)
    with pytest.raises(RuntimeError, match="degenerate bbox"):
        orc.sample_tet_labels(grid, TV, T, (0, 0, 0), (1, 0, 1), 0.0, 0.01)
    bad = T.copy()
    bad[3, 2] = len(TV)
    with pytest.raises(RuntimeError, match="tet index out of range"):
        orc.sample_tet_labels(grid, TV, bad, (0, 0, 0), (1, 1, 1), 0.0, 0.01)
