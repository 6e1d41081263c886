"""Seeded synthetic cell graphs for the graph-cut path.

The reference builds its cut graph from a mesh through OpenVDB (unsigned
distance field, FaithC point proxy), CGAL (Delaunay tets + neighbor export,
``native/core/wtivo_core.cpp:72-165``) and a centroid label query
(``native/vdb/wtivo_vdb.cpp:1519-1584``).  None of those libraries exists in
this image and no benchmark mesh ships with the reference, so the inputs here
are generated from seeds:

* meshes: holed icosphere, torus-knot tube with dropped patches, duplicated
  inner shell and vertex noise, rounded box with a missing face;
* point proxy: area-weighted surface samples pushed +-EPS along the normal
  (a stand-in for FaithC's iso=EPS anchors);
* tetrahedralization: scipy's Qhull Delaunay for proxy-sized clouds (the
  Qhull neighbor of simplex i opposite vertex k lands in CelloCut slot 3-k,
  the same {3,2,1,0} map as wtivo_core.cpp:138), or the seeded Kuhn lattice
  of ``synth.c`` where Qhull would take too long (80M tets);
* labels: exact point-to-triangle distance of each tet centroid, label 0 iff
  <= threshold, in the reference's query coordinates.

Everything returned is what ``graph_cut_fast`` consumes: ``vertices``
float64 [Nv,3], ``tets`` int32 [N,4], ``neighbors`` int32 [N,4], ``labels``
uint8 [N].
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libsynth.so"


def build_library(force: bool = False) -> Path:
    src = HERE / "synth.c"
    if not force and LIB_PATH.exists() and LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB_PATH
    tmp = LIB_PATH.with_suffix(".so.tmp")
    base = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-o", str(tmp), str(src), "-lm"]
    try:  # OpenMP only speeds generation up; results do not depend on it
        subprocess.check_call(base + ["-fopenmp"], stderr=subprocess.DEVNULL)
    except subprocess.CalledProcessError:
        subprocess.check_call(base)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def _L():
    global _lib
    if _lib is None:
        build_library()
        L = ctypes.CDLL(str(LIB_PATH))
        p = ctypes.c_void_p
        L.synth_lattice.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, p, p,
                                    ctypes.c_double, ctypes.c_uint64, p, p, p, p]
        L.synth_lattice.restype = ctypes.c_int64
        L.synth_brick_udf.argtypes = [p, ctypes.c_int64, p, ctypes.c_int64, ctypes.c_double,
                                      ctypes.c_double, p, p, ctypes.c_int, p, p, p]
        L.synth_udf_labels.argtypes = [p, ctypes.c_int64, p, ctypes.c_int64, p, p, p,
                                       ctypes.c_int64, p, ctypes.c_int64, p, p,
                                       ctypes.c_double, p]
        L.synth_udf_labels.restype = ctypes.c_int
        L.synth_raw_graph.argtypes = [p, p, p, ctypes.c_int64, p, ctypes.c_double, p, p, p, p]
        L.synth_raw_graph.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------
# meshes
# --------------------------------------------------------------------------
def icosphere(subdiv: int = 5, radius: float = 0.4, center=(0.0, 0.0, 0.0)):
    """Icosahedron subdivided ``subdiv`` times (20*4^subdiv faces)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
         (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = np.asarray(V, np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.asarray(F, np.int64)
    for _ in range(subdiv):
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (len(V) + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (len(V) + 1), uniq % (len(V) + 1)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = (inv + len(V)).reshape(3, -1).T  # midpoints of edges 01,12,20
        V = np.concatenate([V, mid])
        f0, f1, f2 = F[:, 0], F[:, 1], F[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1),
                            np.stack([f2, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return V * radius + np.asarray(center, np.float64), F.astype(np.int32)


def delete_faces(F, frac: float, rng: np.random.Generator):
    """Drop ``frac`` of the faces at seeded random positions."""
    keep = np.ones(len(F), bool)
    k = int(round(frac * len(F)))
    if k:
        keep[rng.choice(len(F), size=k, replace=False)] = False
    return F[keep]


def torus_knot_tube(p: int = 3, q: int = 5, R: float = 0.3, r: float = 0.12,
                    tube: float = 0.05, n_faces: int = 2_000_000):
    """Closed tube of radius ``tube`` around a (p,q) torus knot; about
    ``n_faces`` triangles.  Returns (V, F, (nu, nv))."""
    # aspect: keep quads roughly square along the curve
    s = np.linspace(0.0, 2.0 * np.pi, 4097)
    c = _knot(s, p, q, R, r)
    length = float(np.sum(np.linalg.norm(np.diff(c, axis=0), axis=1)))
    quads = n_faces // 2
    nv = max(8, int(round(math.sqrt(quads * 2.0 * np.pi * tube / length))))
    nu = max(16, quads // nv)
    u = np.arange(nu) * (2.0 * np.pi / nu)
    C = _knot(u, p, q, R, r)
    T = _knot(u + 1e-4, p, q, R, r) - _knot(u - 1e-4, p, q, R, r)
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    # rotation-minimising frame by projection transport
    ref = np.array([0.0, 0.0, 1.0])
    N = np.empty_like(T)
    n0 = ref - T[0] * np.dot(ref, T[0])
    N[0] = n0 / np.linalg.norm(n0)
    for i in range(1, nu):
        n = N[i - 1] - T[i] * np.dot(N[i - 1], T[i])
        N[i] = n / np.linalg.norm(n)
    B = np.cross(T, N)
    v = np.arange(nv) * (2.0 * np.pi / nv)
    P = (C[:, None, :] + tube * (np.cos(v)[None, :, None] * N[:, None, :]
                                 + np.sin(v)[None, :, None] * B[:, None, :]))
    V = P.reshape(-1, 3)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = i * nv + j
    b = ((i + 1) % nu) * nv + j
    cc = ((i + 1) % nu) * nv + (j + 1) % nv
    d = i * nv + (j + 1) % nv
    F = np.concatenate([np.stack([a, b, cc], -1).reshape(-1, 3),
                        np.stack([a, cc, d], -1).reshape(-1, 3)])
    return V, F.astype(np.int32), (nu, nv)


def _knot(t, p, q, R, r):
    rr = R + r * np.cos(q * t)
    return np.stack([rr * np.cos(p * t), rr * np.sin(p * t), r * np.sin(q * t)], -1)


def drop_patches(V, F, frac: float, rng: np.random.Generator, patch_faces: int = 64):
    """Drop about ``frac`` of the faces in compact patches around seeded
    centers (face centroids within a radius of a center)."""
    from scipy.spatial import cKDTree

    cen = V[F].mean(axis=1)
    target = int(round(frac * len(F)))
    if target == 0:
        return F
    area = 0.5 * np.linalg.norm(np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]]), axis=1)
    rad = math.sqrt(patch_faces * float(area.mean()) / math.pi)
    tree = cKDTree(cen)
    keep = np.ones(len(F), bool)
    dropped = 0
    while dropped < target:
        c = cen[rng.integers(len(F))]
        idx = np.asarray(tree.query_ball_point(c, rad), dtype=np.int64)
        if idx.size:
            dropped += int(np.count_nonzero(keep[idx]))
            keep[idx] = False
    return F[keep]


def offset_shell(V, F, d: float):
    """Copy of the mesh moved by ``d`` along its (area-weighted) vertex
    normals, with flipped orientation (a duplicated inner shell)."""
    n = np.zeros_like(V)
    fn = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    for k in range(3):
        np.add.at(n, F[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return V + d * n, F[:, ::-1].copy()


def rounded_box(half=(0.3, 0.25, 0.2), radius: float = 0.05, n: int = 48):
    """Rounded box: a cube-sphere grid pushed onto the rounded-box surface.
    Returns (V, F, face_id) with face_id in 0..5 for each triangle."""
    g = np.linspace(-1.0, 1.0, n + 1)
    A, Bm = np.meshgrid(g, g, indexing="ij")
    Vs, Fs, ids = [], [], []
    base = 0
    for axis in range(3):
        for sign in (-1.0, 1.0):
            P = np.zeros((n + 1, n + 1, 3))
            o = [k for k in range(3) if k != axis]
            P[..., axis] = sign
            P[..., o[0]] = A
            P[..., o[1]] = Bm
            Vs.append(P.reshape(-1, 3))
            i = np.arange(n)[:, None]
            j = np.arange(n)[None, :]
            a = base + i * (n + 1) + j
            b = a + (n + 1)
            c = b + 1
            d = a + 1
            f = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3),
                                np.stack([a, c, d], -1).reshape(-1, 3)])
            if sign < 0:
                f = f[:, ::-1]
            Fs.append(f)
            ids.append(np.full(len(f), axis * 2 + (sign > 0), np.int8))
            base += (n + 1) * (n + 1)
    U = np.concatenate(Vs)
    F = np.concatenate(Fs).astype(np.int32)
    h = np.asarray(half, np.float64)
    inner = h - radius
    X = U * h
    core = np.clip(X, -inner, inner)
    dvec = X - core
    nrm = np.linalg.norm(dvec, axis=1, keepdims=True)
    dvec = np.where(nrm > 1e-15, dvec / np.maximum(nrm, 1e-15) * radius, dvec)
    return core + dvec, F, np.concatenate(ids)


# --------------------------------------------------------------------------
# point proxy + tetrahedralizations
# --------------------------------------------------------------------------
def proxy_points(V, F, n: int, eps: float, rng: np.random.Generator):
    """``n`` area-weighted surface samples pushed +-eps along the face
    normal, with 10% tangential jitter of eps."""
    e1 = V[F[:, 1]] - V[F[:, 0]]
    e2 = V[F[:, 2]] - V[F[:, 0]]
    fn = np.cross(e1, e2)
    area = 0.5 * np.linalg.norm(fn, axis=1)
    fn /= np.maximum(2.0 * area[:, None], 1e-30)
    f = rng.choice(len(F), size=n, p=area / area.sum())
    r1 = np.sqrt(rng.random(n))
    r2 = rng.random(n)
    P = (V[F[f, 0]] * (1 - r1)[:, None] + V[F[f, 1]] * (r1 * (1 - r2))[:, None]
         + V[F[f, 2]] * (r1 * r2)[:, None])
    side = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    P += fn[f] * (side * eps)[:, None]
    P += rng.normal(scale=0.1 * eps, size=P.shape)
    return P


def delaunay_cells(points, spatial_order: bool = True):
    """Qhull Delaunay -> (tets int32 [N,4], neighbors int32 [N,4]) in the
    CelloCut slot convention (slot fi = tet opposite local vertex 3-fi).
    With spatial_order the cells are renumbered in Morton order of their
    centroids: CGAL inserts a point set in spatially sorted order, so its
    cells come out spatially coherent, while Qhull's do not."""
    from scipy.spatial import Delaunay
    P = np.asarray(points, np.float64)
    d = Delaunay(P)
    tets = np.ascontiguousarray(d.simplices.astype(np.int32))
    nbrs = np.ascontiguousarray(d.neighbors[:, ::-1].astype(np.int32))
    del d
    if spatial_order:
        tets, nbrs = morton_order_cells(P, tets, nbrs)
    return tets, nbrs


def morton_order_cells(P, tets, nbrs, bits: int = 10):
    """Cells renumbered by the Morton code of their centroids (stable)."""
    cen = P[tets].mean(axis=1)
    lo = cen.min(0)
    span = np.maximum(cen.max(0) - lo, 1e-300)
    q = np.clip(((cen - lo) / span * ((1 << bits) - 1)).astype(np.int64), 0, (1 << bits) - 1)
    code = np.zeros(len(tets), np.int64)
    for b in range(bits):
        for a in range(3):
            code |= ((q[:, a] >> b) & 1) << (3 * b + a)
    order = np.argsort(code, kind="stable")
    inv = np.empty(len(tets), np.int64)
    inv[order] = np.arange(len(tets))
    t2 = np.ascontiguousarray(tets[order])
    n2 = nbrs[order]
    n2 = np.where(n2 >= 0, inv[np.maximum(n2, 0)], -1).astype(np.int32)
    return t2, np.ascontiguousarray(n2)


def lattice_cells(shape, lo, hi, jitter: float = 0.15, seed: int = 0):
    """Jittered Kuhn lattice over the box [lo, hi] with ``shape`` cubes:
    (V float64, tets int32, neighbors int32); 6 tets per cube."""
    nx, ny, nz = (int(s) for s in shape)
    lo = np.asarray(lo, np.float64)
    h = (np.asarray(hi, np.float64) - lo) / np.array([nx, ny, nz], np.float64)
    N = 6 * nx * ny * nz
    V = np.empty(((nx + 1) * (ny + 1) * (nz + 1), 3), np.float64)
    tets = np.empty((N, 4), np.int32)
    nbrs = np.empty((N, 4), np.int32)
    scratch = np.empty(nx * ny * nz, np.int32)
    got = _L().synth_lattice(nx, ny, nz, _ptr(lo), _ptr(h), float(jitter),
                             int(seed) & 0xFFFFFFFFFFFFFFFF, _ptr(V), _ptr(tets), _ptr(nbrs),
                             _ptr(scratch))
    if got != N:
        raise ValueError("lattice too large or empty")
    return V, tets, nbrs


def udf_labels(V, tets, mesh_V, mesh_F, threshold: float, centroid_map=None, mesh_map=None):
    """labels[i] = 0 iff dist(centroid_i, mesh) <= threshold.  Optional
    per-axis affine maps (scale[3], offset[3]) for centroids and mesh."""
    V = np.ascontiguousarray(V, np.float64)
    tets = np.ascontiguousarray(tets, np.int32)
    MV = np.ascontiguousarray(mesh_V, np.float64)
    MF = np.ascontiguousarray(mesh_F, np.int32)
    cs, co = (np.ones(3), np.zeros(3)) if centroid_map is None else centroid_map
    ms, mo = (np.ones(3), np.zeros(3)) if mesh_map is None else mesh_map
    cs, co, ms, mo = (np.ascontiguousarray(x, np.float64) for x in (cs, co, ms, mo))
    out = np.empty(len(tets), np.uint8)
    rc = _L().synth_udf_labels(_ptr(V), len(V), _ptr(tets), len(tets), _ptr(cs), _ptr(co),
                               _ptr(MV), len(MV), _ptr(MF), len(MF), _ptr(ms), _ptr(mo),
                               float(threshold), _ptr(out))
    if rc != 0:
        raise MemoryError("udf_labels failed")
    return out


def brick_udf(mesh_V, mesh_F, voxel_size: float, band_voxels: float = 3.0):
    """Narrow-band unsigned distance field of a triangle mesh on a brick grid
    (8^3 voxels per brick), the input of the tet-centroid label sampler; a
    stand-in for OpenVDB meshToUnsignedDistanceField with a linear transform
    of ``voxel_size`` (voxel (i,j,k) at world (i,j,k)*voxel_size, exact
    distances below band_voxels*voxel_size, background band_voxels*voxel_size
    elsewhere).  Returns dict(voxel_size, origin (voxel index of the first
    brick's first voxel), dims (bricks), background, table int32[dims]
    (brick number or -1), values float32[bricks, 8, 8, 8] (z fastest))."""
    MV = np.ascontiguousarray(mesh_V, np.float64)
    MF = np.ascontiguousarray(mesh_F, np.int32)
    h = float(voxel_size)
    band = float(band_voxels) * h
    lo = np.floor((MV.min(0) - band) / h).astype(np.int64) - 1
    hi = np.ceil((MV.max(0) + band) / h).astype(np.int64) + 1
    bmin3 = np.ascontiguousarray(lo >> 3, np.int32)
    dims = np.ascontiguousarray((hi >> 3) - (lo >> 3) + 1, np.int32)
    mask = np.zeros(int(np.prod(dims.astype(np.int64))), np.uint8)
    L = _L()
    if L.synth_brick_udf(_ptr(MV), len(MV), _ptr(MF), len(MF), h, band, _ptr(bmin3), _ptr(dims), 0,
                         _ptr(mask), None, None) != 0:
        raise ValueError("brick_udf: voxel outside the brick box")
    table = np.full(mask.shape, -1, np.int32)
    act = np.nonzero(mask)[0]
    table[act] = np.arange(len(act), dtype=np.int32)
    values = np.full((max(len(act), 1), 8, 8, 8), np.float32(band), np.float32)
    if L.synth_brick_udf(_ptr(MV), len(MV), _ptr(MF), len(MF), h, band, _ptr(bmin3), _ptr(dims), 1,
                         None, _ptr(table), _ptr(values)) != 0:
        raise ValueError("brick_udf: voxel outside the brick box")
    return dict(voxel_size=h, origin=(bmin3.astype(np.int64) * 8).astype(np.int32), dims=dims,
                background=np.float32(band), table=table.reshape(tuple(dims)), values=values[:len(act)])


# --------------------------------------------------------------------------
# workload configurations
# --------------------------------------------------------------------------
class CellGraph(dict):
    """vertices, tets, neighbors, labels (+ metadata)."""

    @property
    def n_tets(self):
        return int(self["tets"].shape[0])


def _reference_maps(mesh_V, eps):
    """The reference normalises the mesh into [eps, 1-eps]^3 per axis for the
    field (wtivo.py:195-197) but queries tet centroids with zero padding
    (wtivo.py:91-93, wtivo_vdb.cpp:1567-1569): query = (c-bmin)/span."""
    bmin = mesh_V.min(0)
    span = mesh_V.max(0) - bmin
    scale = 1.0 - 2.0 * eps
    mesh_map = (scale / span, eps - bmin * scale / span)
    centroid_map = (1.0 / span, -bmin / span)
    return mesh_map, centroid_map


def proxy_delaunay_graph(mesh_V, mesh_F, n_points: int, res: int, seed: int):
    """Reference-shaped cell graph: point proxy at EPS=1/res around the mesh,
    Qhull Delaunay, centroid labels at threshold EPS-1e-4 (wtivo.py:88-92)."""
    rng = np.random.default_rng(seed)
    eps = 1.0 / res
    mesh_map, centroid_map = _reference_maps(mesh_V, eps)
    # points live in field space around the normalised mesh, mapped back
    NV = mesh_V * mesh_map[0] + mesh_map[1]
    P = proxy_points(NV, mesh_F, n_points, eps, rng)
    P = (P - mesh_map[1]) / mesh_map[0]
    tets, nbrs = delaunay_cells(P)
    labels = udf_labels(P, tets, mesh_V, mesh_F, eps - 1.0e-4, centroid_map=centroid_map,
                        mesh_map=mesh_map)
    return CellGraph(vertices=P, tets=tets, neighbors=nbrs, labels=labels,
                     kind="proxy-delaunay", eps=eps)


def lattice_graph(mesh_V, mesh_F, n_tets: int, seed: int, margin: float = 0.06,
                  band_cells: float = 0.8, jitter: float = 0.15):
    """Kuhn-lattice cell graph of about ``n_tets`` tets over the mesh bbox
    (plus ``margin`` of its span on each side), labelled by the exact UDF at
    ``band_cells`` lattice spacings."""
    lo = mesh_V.min(0)
    hi = mesh_V.max(0)
    pad = margin * (hi - lo).max()
    lo = lo - pad
    hi = hi + pad
    ext = hi - lo
    cubes = n_tets / 6.0
    hcell = (float(np.prod(ext)) / cubes) ** (1.0 / 3.0)
    shape = np.maximum(1, np.round(ext / hcell)).astype(int)
    V, tets, nbrs = lattice_cells(shape, lo, hi, jitter=jitter, seed=seed)
    hmean = float(np.mean(ext / shape))
    labels = udf_labels(V, tets, mesh_V, mesh_F, band_cells * hmean)
    return CellGraph(vertices=V, tets=tets, neighbors=nbrs, labels=labels, kind="kuhn-lattice",
                     shape=tuple(int(s) for s in shape), threshold=band_cells * hmean)


def holed_icosphere(seed: int, subdiv: int = 5, frac: float = 0.05):
    rng = np.random.default_rng(seed)
    V, F = icosphere(subdiv, 0.4)
    return V, delete_faces(F, frac, rng)


def defective_torus_knot(seed: int, n_faces: int = 2_000_000):
    """(3,5) torus-knot tube r=0.05, 2% faces dropped in patches, inner shell
    offset 0.002, Gaussian vertex noise sigma=1e-4."""
    rng = np.random.default_rng(seed)
    V, F, _ = torus_knot_tube(3, 5, 0.3, 0.12, 0.05, n_faces // 2)
    F = drop_patches(V, F, 0.02, rng)
    Vi, Fi = offset_shell(V, F, -0.002)
    allV = np.concatenate([V, Vi])
    allF = np.concatenate([F, Fi + len(V)])
    allV = allV + rng.normal(scale=1e-4, size=allV.shape)
    return allV, allF.astype(np.int32)


def holed_torus(seed: int, R: float = 0.3, r: float = 0.1, nu: int = 192, nv: int = 64,
                frac: float = 0.03):
    rng = np.random.default_rng(seed)
    u = np.arange(nu) * (2 * np.pi / nu)
    v = np.arange(nv) * (2 * np.pi / nv)
    U, W = np.meshgrid(u, v, indexing="ij")
    V = np.stack([(R + r * np.cos(W)) * np.cos(U), (R + r * np.cos(W)) * np.sin(U),
                  r * np.sin(W)], -1).reshape(-1, 3)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = i * nv + j
    b = ((i + 1) % nu) * nv + j
    c = ((i + 1) % nu) * nv + (j + 1) % nv
    d = i * nv + (j + 1) % nv
    F = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3),
                        np.stack([a, c, d], -1).reshape(-1, 3)]).astype(np.int32)
    return V, drop_patches(V, F, frac, rng, patch_faces=16)


def open_rounded_box(seed: int):
    rng = np.random.default_rng(seed)
    V, F, ids = rounded_box()
    missing = int(rng.integers(6))
    return V, F[ids != missing]


def config1(seed: int = 0, n_points: int = 500_000):
    """Plain single cut: holed icosphere (r=0.4, subdiv 5, 5% faces deleted),
    500k-point proxy at res 256, Qhull Delaunay (~3.3M tets), lambda 10."""
    mv, mf = holed_icosphere(seed)
    g = proxy_delaunay_graph(mv, mf, n_points, 256, seed + 1)
    g["fill_T"] = 10.0
    g["name"] = f"icosphere-holed-{n_points}pt"
    return g


def config2(seed: int = 0, n_tets: int = 80_000_000, n_faces: int = 2_000_000):
    """Benchmark-scale cut: defective (3,5) torus-knot tube (~2M faces);
    Kuhn lattice of ~80M tets standing in for the 12M-point Delaunay."""
    mv, mf = defective_torus_knot(seed, n_faces)
    g = lattice_graph(mv, mf, n_tets, seed + 1)
    g["fill_T"] = 10.0
    g["name"] = f"torusknot-lattice-{g.n_tets}"
    g["mesh_V"], g["mesh_F"] = mv, mf
    return g


def batch_mesh(kind: int, seed: int):
    if kind == 0:
        return holed_icosphere(seed, subdiv=4, frac=0.05)
    if kind == 1:
        return holed_torus(seed)
    return open_rounded_box(seed)


def config3_sizes(seed: int = 0, count: int = 64, lo: float = 5e4, hi: float = 4e6):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).astype(np.int64)


def config3_graph(i: int, n_tets: int, seed: int = 0):
    """One graph of the uneven batch: mesh kind i%3, lattice of ~n_tets."""
    mv, mf = batch_mesh(i % 3, seed * 1000 + i)
    g = lattice_graph(mv, mf, int(n_tets), seed * 1000 + i + 7)
    g["fill_T"] = 10.0
    return g


def config4(seed: int = 0, n_points: int = 2_000_000, use_delaunay: bool = True,
            nlink_scale: float = 1e4):
    """Integer-capacity raw graph: uniform points in [0,1]^3, n-link
    round(nlink_scale*area/mean_area) (symmetric per face; 1e4 in the
    workload), t-links from a noisy sphere SDF (c=0.5, r=0.3, sigma=0.02):
    src=round(100*max(0,-d')), snk=round(100*max(0,d')).  Returns
    dict(nbr, cap, src, snk)."""
    rng = np.random.default_rng(seed)
    if use_delaunay:
        P = rng.random((n_points, 3))
        tets, nbrs = delaunay_cells(P)
    else:
        m = max(2, int(round(n_points ** (1.0 / 3.0))) - 1)
        P, tets, nbrs = lattice_cells((m, m, m), (0, 0, 0), (1, 1, 1), seed=seed)
    return raw_graph_from_cells(P, tets, nbrs, rng, nlink_scale)


def raw_graph_from_cells(P, tets, nbrs, rng, nlink_scale: float = 1e4):
    """Integer n-links round(nlink_scale*area/mean_area), identical in both
    directions (each face's area is taken from its lower-id tet), and sphere
    SDF t-links with Gaussian noise (sigma 0.02) drawn from rng
    (synth_raw_graph in synth.c)."""
    P = np.ascontiguousarray(P, np.float64)
    tets = np.ascontiguousarray(tets, np.int32)
    nbrs = np.ascontiguousarray(nbrs, np.int32)
    N = len(tets)
    noise = np.ascontiguousarray(rng.normal(scale=0.02, size=N))
    scratch = np.empty((N, 4), np.float64)
    cap = np.empty((N, 4), np.uint32)
    src = np.empty(N, np.uint32)
    snk = np.empty(N, np.uint32)
    rc = _L().synth_raw_graph(_ptr(P), _ptr(tets), _ptr(nbrs), N, _ptr(noise), float(nlink_scale),
                              _ptr(scratch), _ptr(cap), _ptr(src), _ptr(snk))
    if rc != 0:
        raise ValueError("raw_graph_from_cells: asymmetric neighbours" if rc == -1 else "out of memory")
    return dict(nbr=nbrs, cap=cap, src=src, snk=snk, n_points=len(P))


def _reverse_slots_np(nbrs):
    N = len(nbrs)
    valid = nbrs >= 0
    j = np.where(valid, nbrs, 0)
    rows = nbrs[j]  # [N,4,4]
    me = np.arange(N)[:, None, None]
    hit = rows == me
    rev = np.argmax(hit, axis=2).astype(np.int8)
    return np.where(valid, rev, -1)
