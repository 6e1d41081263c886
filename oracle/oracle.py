"""ctypes front end of the CPU oracle (``wtivo_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker that the CUDA product is compared
against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` import this module; the product never does.

Every function restates reference semantics from
``native/gpupr/wtivo_gpupr_bindings.cpp`` and
``native/gpupr/gpu_push_relabel_fast.cu`` (see ``wtivo_oracle.h``), and raises
the same exception text the reference raises for the same failure.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

# Reference error text for each oracle status (bindings.cpp:172,177,188,197,
# 297,318; gpu_push_relabel_fast.cu:254,292,492).
_ERRORS = {
    1: (RuntimeError, "invalid argument"),
    2: (RuntimeError, "neighbor out of range"),
    3: (RuntimeError, "neighbor reference count not even"),
    4: (RuntimeError, "invalid graph reduction/capacity state"),
    5: (RuntimeError, "free reference count not even"),
    6: (RuntimeError, ">INT32_MAX reduced nodes unsupported"),
    7: (RuntimeError, "device invariant failed: missing reverse slot"),
    8: (MemoryError, "oracle out of host memory"),
    9: (RuntimeError, "GPUPr-FAST-v6.30 max macro rounds exceeded"),
    10: (RuntimeError, "device invariant failed: no residual out-arc"),
    11: (RuntimeError, "negative vertex index"),
    12: (RuntimeError, "SparseUDF.sample_tet_labels: degenerate bbox"),
    13: (RuntimeError, "SparseUDF.sample_tet_labels: tet index out of range"),
}


class BuildInfo(ctypes.Structure):
    _fields_ = [
        ("n_full", ctypes.c_uint64),
        ("free_n", ctypes.c_uint64),
        ("fixed_source", ctypes.c_uint64),
        ("fixed_sink", ctypes.c_uint64),
        ("full_refs", ctypes.c_uint64),
        ("free_refs", ctypes.c_uint64),
        ("terminal_edges", ctypes.c_uint64),
        ("terminal_base_flow", ctypes.c_int64),
    ]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


def build_library(force: bool = False) -> Path:
    """Compile ``liboracle.so`` with strict IEEE doubles (no FMA contraction)."""
    src = HERE / "wtivo_oracle.c"
    if (not force and LIB_PATH.exists()
            and LIB_PATH.stat().st_mtime >= src.stat().st_mtime
            and LIB_PATH.stat().st_mtime >= (HERE / "wtivo_oracle.h").stat().st_mtime):
        return LIB_PATH
    tmp = LIB_PATH.with_suffix(".so.tmp")
    subprocess.check_call([
        "gcc", "-O2", "-std=c11", "-Wall", "-fPIC", "-shared",
        "-ffp-contract=off", "-fno-fast-math", "-o", str(tmp), str(src), "-lm",
    ])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_library()
        L = ctypes.CDLL(str(LIB_PATH))
        p = ctypes.c_void_p
        u64, i32, f64 = ctypes.c_uint64, ctypes.c_int, ctypes.c_double
        L.orc_capacity.argtypes = [p, u64, p, i32, ctypes.c_uint8, ctypes.c_uint8, f64, p]
        L.orc_classify.argtypes = [p, p, u64, p, p, p]
        L.orc_build.argtypes = [p, u64, p, p, p, u64, f64, p, p, p, p, p]
        L.orc_reverse_slots.argtypes = [ctypes.c_uint32, p, p]
        L.orc_maxflow_bk.argtypes = [ctypes.c_uint32, p, p, p, p, p]
        L.orc_maxflow_pr.argtypes = [ctypes.c_uint32, p, p, p, p, i32, i32, u64, p, p, p, p]
        L.orc_sink_reachable.argtypes = [ctypes.c_uint32, p, p, p, p]
        L.orc_graph_cut.argtypes = [p, u64, p, p, p, u64, f64, i32, p, p]
        L.orc_surface.argtypes = [p, p, u64, p, p, u64, p, p, p, p]
        L.orc_edge_audit.argtypes = [p, u64, p]
        L.orc_sample_tet_labels.argtypes = [p, p, u64, p, u64, p, p, f64, f64, p, p]
        for name in ("orc_capacity", "orc_classify", "orc_build", "orc_reverse_slots",
                     "orc_maxflow_bk", "orc_maxflow_pr", "orc_sink_reachable",
                     "orc_graph_cut", "orc_surface", "orc_edge_audit",
                     "orc_sample_tet_labels"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        exc, msg = _ERRORS.get(rc, (RuntimeError, f"oracle status {rc}"))
        raise exc(msg)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def capacity(V, tet4, fi, li, lj, fill_T) -> int:
    """One arc capacity (bindings.cpp:65-98)."""
    V = _c(V, np.float64)
    t = _c(tet4, np.int32).reshape(4)
    out = ctypes.c_int32(0)
    _check(lib().orc_capacity(_ptr(V), V.shape[0], _ptr(t), int(fi), int(li), int(lj),
                              float(fill_T), ctypes.byref(out)))
    return int(out.value)


def classify(nbrs, labels):
    """Classification + compaction (bindings.cpp:146-188)."""
    nbrs = _c(nbrs, np.int32)
    labels = _c(labels, np.uint8).reshape(-1)
    N = labels.shape[0]
    f2f = np.empty(N, np.int32)
    old = np.empty(max(N, 1), np.uint32)
    info = BuildInfo()
    _check(lib().orc_classify(_ptr(nbrs), _ptr(labels), N, _ptr(f2f), _ptr(old),
                              ctypes.byref(info)))
    return f2f, old[: info.free_n].copy(), info


def build(V, tets, nbrs, labels, fill_T):
    """Reduced ELL graph: returns dict(nbr[F,4], res[F,4], term[F],
    full_to_free[N], free_old[F], info)."""
    V = _c(V, np.float64)
    tets = _c(tets, np.int32)
    nbrs = _c(nbrs, np.int32)
    labels = _c(labels, np.uint8).reshape(-1)
    f2f, old, info = classify(nbrs, labels)
    F = int(info.free_n)
    nbr = np.full((max(F, 1), 4), -1, np.int32)
    res = np.zeros((max(F, 1), 4), np.uint32)
    term = np.zeros(max(F, 1), np.int32)
    _check(lib().orc_build(_ptr(V), V.shape[0], _ptr(tets), _ptr(nbrs), _ptr(labels),
                           labels.shape[0], float(fill_T), _ptr(f2f), ctypes.byref(info),
                           _ptr(nbr), _ptr(res), _ptr(term)))
    return dict(nbr=nbr[:F].copy(), res=res[:F].copy(), term=term[:F].copy(),
                full_to_free=f2f, free_old=old, info=info.as_dict())


def reverse_slots(nbr):
    nbr = _c(nbr, np.int32)
    F = nbr.shape[0]
    rev = np.empty((F, 4), np.uint8)
    _check(lib().orc_reverse_slots(F, _ptr(nbr), _ptr(rev)))
    return rev


def maxflow_bk(nbr, res, term):
    """Boykov-Kolmogorov max flow.  Returns (raw_flow, res_final, term_final,
    partition) with partition[v] = 1 iff v reaches the sink."""
    nbr = _c(nbr, np.int32)
    res = _c(res, np.uint32).copy()
    term = _c(term, np.int32).copy()
    F = nbr.shape[0]
    part = np.zeros(max(F, 1), np.uint8)
    flow = ctypes.c_int64(0)
    _check(lib().orc_maxflow_bk(F, _ptr(nbr), _ptr(res), _ptr(term), ctypes.byref(flow),
                                _ptr(part)))
    return int(flow.value), res, term, part[:F]


def maxflow_pr(nbr, res, term, local_steps=8, global_relabel_period=1024, max_rounds=0):
    """Sequential Phase-I push-relabel with the reference's rules.  Returns
    (raw_flow, res_final, term_final, excess, partition, rounds, relabels)."""
    nbr = _c(nbr, np.int32)
    res = _c(res, np.uint32).copy()
    term = _c(term, np.int32).copy()
    F = nbr.shape[0]
    exc = np.zeros(max(F, 1), np.int64)
    part = np.zeros(max(F, 1), np.uint8)
    flow = ctypes.c_int64(0)
    rounds = ctypes.c_uint64(0)
    rel = ctypes.c_uint64(0)
    _check(lib().orc_maxflow_pr(F, _ptr(nbr), _ptr(res), _ptr(term), _ptr(exc),
                                int(local_steps), int(global_relabel_period),
                                int(max_rounds), ctypes.byref(flow), _ptr(part),
                                ctypes.byref(rounds), ctypes.byref(rel)))
    return (int(flow.value), res, term, exc[:F], part[:F], int(rounds.value),
            int(rel.value))


def sink_reachable(nbr, res, term):
    nbr = _c(nbr, np.int32)
    res = _c(res, np.uint32)
    term = _c(term, np.int32)
    F = nbr.shape[0]
    part = np.zeros(max(F, 1), np.uint8)
    _check(lib().orc_sink_reachable(F, _ptr(nbr), _ptr(res), _ptr(term), _ptr(part)))
    return part[:F]


def graph_cut(V, tets, nbrs, labels, fill_T, solver: str = "bk"):
    """The whole graph_cut_fast path on the CPU.  Returns (labels_out, stats)
    with stats = dict(adjusted_flow, raw_flow, full_E, free_E, fixed_source,
    fixed_sink, terminal_edges, free_n)."""
    V = _c(V, np.float64)
    tets = _c(tets, np.int32)
    nbrs = _c(nbrs, np.int32)
    labels = _c(labels, np.uint8).reshape(-1)
    N = labels.shape[0]
    out = np.empty(max(N, 1), np.uint8)
    st = np.zeros(8, np.int64)
    _check(lib().orc_graph_cut(_ptr(V), V.shape[0], _ptr(tets), _ptr(nbrs), _ptr(labels), N,
                               float(fill_T), 0 if solver == "bk" else 1, _ptr(out), _ptr(st)))
    keys = ("adjusted_flow", "raw_flow", "full_E", "free_E", "fixed_source", "fixed_sink",
            "terminal_edges", "free_n")
    return out[:N], {k: int(v) for k, v in zip(keys, st)}


def surface(labels, V, tets, nbrs):
    """Cut-surface extraction (bindings.cpp:400-577): returns (verts[U,3] f64,
    faces[F,3] int32)."""
    labels = _c(labels, np.uint8).reshape(-1)
    V = _c(V, np.float64)
    tets = _c(tets, np.int32)
    nbrs = _c(nbrs, np.int32)
    nf = ctypes.c_uint64(0)
    nu = ctypes.c_uint64(0)
    L = lib()
    _check(L.orc_surface(_ptr(labels), _ptr(V), V.shape[0], _ptr(tets), _ptr(nbrs),
                         labels.shape[0], ctypes.byref(nf), ctypes.byref(nu), None, None))
    faces = np.empty((max(nf.value, 1), 3), np.int32)
    verts = np.empty((max(nu.value, 1), 3), np.float64)
    _check(L.orc_surface(_ptr(labels), _ptr(V), V.shape[0], _ptr(tets), _ptr(nbrs),
                         labels.shape[0], ctypes.byref(nf), ctypes.byref(nu), _ptr(faces),
                         _ptr(verts)))
    return verts[: nu.value], faces[: nf.value]


def edge_audit(faces):
    """Edge-degree watertight audit (wtivo_core.cpp:402-464): returns the
    number of bad edge groups (runs of equal undirected edges whose length
    is not 2)."""
    faces = _c(faces, np.int32).reshape(-1, 3)
    bad = ctypes.c_uint64(0)
    _check(lib().orc_edge_audit(_ptr(faces), faces.shape[0], ctypes.byref(bad)))
    return int(bad.value)


class BrickGrid(ctypes.Structure):
    _fields_ = [("voxel_size", ctypes.c_double), ("origin", ctypes.c_int32 * 3),
                ("dims", ctypes.c_int32 * 3), ("background", ctypes.c_float),
                ("table", ctypes.c_void_p), ("values", ctypes.c_void_p)]


def sample_tet_labels(grid, V, tets, bbox_min, bbox_max, padding, threshold):
    """Tet-centroid labels (wtivo_vdb.cpp:1519-1584) on a brick grid (dict
    as made by synth.brick_udf): returns (labels uint8[N], samples f32[N])."""
    table = _c(grid["table"], np.int32).reshape(-1)
    values = _c(grid["values"], np.float32).reshape(-1)
    g = BrickGrid(float(grid["voxel_size"]), (ctypes.c_int32 * 3)(*[int(x) for x in grid["origin"]]),
                  (ctypes.c_int32 * 3)(*[int(x) for x in grid["dims"]]), float(grid["background"]),
                  table.ctypes.data, values.ctypes.data)
    V = _c(V, np.float64)
    tets = _c(tets, np.int32)
    bmin = _c(bbox_min, np.float64)
    bmax = _c(bbox_max, np.float64)
    out = np.empty(max(len(tets), 1), np.uint8)
    udf = np.empty(max(len(tets), 1), np.float32)
    _check(lib().orc_sample_tet_labels(ctypes.byref(g), _ptr(V), V.shape[0], _ptr(tets), tets.shape[0],
                                       _ptr(bmin), _ptr(bmax), float(padding), float(threshold),
                                       _ptr(out), _ptr(udf)))
    return out[:len(tets)], udf[:len(tets)]
