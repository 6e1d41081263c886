"""ctypes front end of ``libwtivo_gpupr.so`` (the C ABI in include/wtivo_gpupr.h).

Device buffers are passed as torch CUDA tensors (their data_ptr) and host
buffers as numpy arrays; torch is only used for device memory and streams.
Every call raises ``GpuprError`` with the library's message on failure.
The CUDA library is required: loading fails loudly if it is missing.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libwtivo_gpupr.so"
HEADER = PKG.parent / "include" / "wtivo_gpupr.h"

STATS_FIELDS = [
    ("adjusted_flow", ctypes.c_int64), ("raw_flow", ctypes.c_int64),
    ("graph_bytes", ctypes.c_uint64), ("workspace_bytes", ctypes.c_uint64),
    ("full_E", ctypes.c_uint64), ("free_E", ctypes.c_uint64),
    ("fixed_source", ctypes.c_uint64), ("fixed_sink", ctypes.c_uint64),
    ("terminal_edges", ctypes.c_uint64), ("threads", ctypes.c_int64),
    ("rounds", ctypes.c_uint64), ("global_relabels", ctypes.c_uint64),
    ("map_bytes", ctypes.c_uint64), ("build_seconds", ctypes.c_double),
    ("local_steps", ctypes.c_int64), ("solve_seconds", ctypes.c_double),
    ("native_total_seconds", ctypes.c_double),
    ("free_n", ctypes.c_uint64), ("n_full", ctypes.c_uint64),
    ("final_relabel_seconds", ctypes.c_double), ("partition_seconds", ctypes.c_double),
    ("node_visits", ctypes.c_uint64), ("pushes", ctypes.c_uint64),
    ("bfs_visits", ctypes.c_uint64), ("bfs_levels", ctypes.c_uint64),
    ("kernel_launches", ctypes.c_uint64), ("solve_device_ms", ctypes.c_double),
    ("build_device_ms", ctypes.c_double), ("discharge_ms", ctypes.c_double),
    ("bfs_ms", ctypes.c_double), ("discharge_launches", ctypes.c_uint64),
    ("bfs_launches", ctypes.c_uint64), ("engine", ctypes.c_int64),
    ("solve_blocks_per_sm", ctypes.c_int64), ("relabel_work_factor", ctypes.c_double),
    ("chain_hops", ctypes.c_int64), ("chain_max_active", ctypes.c_int64),
    ("sweep_ms", ctypes.c_double), ("graphs_retired", ctypes.c_uint64),
    ("bottom_up_steps", ctypes.c_uint64),
    ("bfs_steps_by_frontier", ctypes.c_uint64 * 3), ("bfs_ms_by_frontier", ctypes.c_double * 3),
    ("bfs_tail_steps", ctypes.c_uint64), ("bfs_tail_levels", ctypes.c_uint64),
    ("relabel_tiles", ctypes.c_int64), ("tile_steps", ctypes.c_uint64),
    ("tile_procs", ctypes.c_uint64), ("tile_loads", ctypes.c_uint64),
    ("tile_writes", ctypes.c_uint64),
    ("discharge_rounds_by_active", ctypes.c_uint64 * 3),
    ("discharge_ms_by_active", ctypes.c_double * 3),
]


class CutStats(ctypes.Structure):
    _fields_ = STATS_FIELDS

    def as_dict(self):
        return {k: (list(v) if isinstance(v, ctypes.Array) else v)
                for k, v in ((k, getattr(self, k)) for k, _ in self._fields_)}


class SolveOptions(ctypes.Structure):
    _fields_ = [
        ("local_steps", ctypes.c_int32), ("global_relabel_period", ctypes.c_int32),
        ("max_rounds", ctypes.c_uint64), ("time_limit_seconds", ctypes.c_double),
        ("round_batch", ctypes.c_int32), ("bfs_batch", ctypes.c_int32),
        ("block_size", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
        ("work_relabel_factor", ctypes.c_double), ("engine", ctypes.c_int32),
        ("chain_hops", ctypes.c_int32), ("chain_max_active", ctypes.c_int32),
        ("bfs_bottom_up", ctypes.c_int32), ("bfs_bottom_up_ratio", ctypes.c_double),
        ("bfs_chain_hops", ctypes.c_int32), ("bfs_tail_max", ctypes.c_int32),
        ("discharge_warp_aggregate", ctypes.c_int32), ("bfs_chain_max_frontier", ctypes.c_int32),
        ("relabel_tiles", ctypes.c_int32), ("bfs_block_levels", ctypes.c_int32),
        ("bfs_in_arc_masks", ctypes.c_int32),
    ]


class BatchItem(ctypes.Structure):
    _fields_ = [("adjusted_flow", ctypes.c_int64), ("raw_flow", ctypes.c_int64),
                ("n_tets", ctypes.c_uint64), ("free_n", ctypes.c_uint64)]


class RequestResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int32), ("batch_size", ctypes.c_int32),
                ("adjusted_flow", ctypes.c_int64), ("raw_flow", ctypes.c_int64),
                ("n_tets", ctypes.c_uint64), ("free_n", ctypes.c_uint64),
                ("queue_ms", ctypes.c_double), ("upload_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("lane", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class GpuprError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


STATUS = {
    0: "GPUPR_OK", 1: "GPUPR_ERR_INVALID_ARGUMENT", 2: "GPUPR_ERR_NEIGHBOR_RANGE",
    3: "GPUPR_ERR_REFS_ODD", 4: "GPUPR_ERR_BUILD", 5: "GPUPR_ERR_FREE_REFS_ODD",
    6: "GPUPR_ERR_TOO_MANY_NODES", 7: "GPUPR_ERR_NO_REVERSE", 8: "GPUPR_ERR_OUT_OF_MEMORY",
    9: "GPUPR_ERR_MAX_ROUNDS", 10: "GPUPR_ERR_INVARIANT", 11: "GPUPR_ERR_CUDA",
    12: "GPUPR_ERR_TIMEOUT", 13: "GPUPR_ERR_TOO_MANY_TETS",
}

_lib = None


def header_functions():
    """Names of every function the public header declares."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(gpupr_[a-z_0-9]+)\s*\(",
                                 text, flags=re.M)))


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run build.py (no CPU fallback exists)")
        L = ctypes.CDLL(str(LIB_PATH))
        p, u64, i32, f64 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_double
        L.gpupr_status_string.restype = ctypes.c_char_p
        L.gpupr_status_string.argtypes = [ctypes.c_int]
        L.gpupr_last_error.restype = ctypes.c_char_p
        L.gpupr_last_error.argtypes = []
        L.gpupr_abi_version.restype = ctypes.c_int
        L.gpupr_graph_cut.argtypes = [p, u64, ctypes.c_int, p, p, u64, p, ctypes.c_int, f64, i32,
                                      i32, u64, i32, p, ctypes.c_int, p, p]
        L.gpupr_graph_cut_ex.argtypes = [p, u64, ctypes.c_int, p, p, u64, p, ctypes.c_int, f64,
                                         i32, p, p, ctypes.c_int, p, p]
        L.gpupr_build_reduced.argtypes = [p, u64, ctypes.c_int, p, p, u64, p, ctypes.c_int, f64,
                                          p, p, p, p, p, p, p, p]
        L.gpupr_solve_reduced.argtypes = [ctypes.c_uint32, p, p, p, p, i32, u64, i32, p, p, p]
        L.gpupr_solve_ell.argtypes = [ctypes.c_uint32, p, p, p, p, p, p, p, p, p]
        L.gpupr_surface_count.argtypes = [p, ctypes.c_int, p, u64, ctypes.c_int, p, p, u64, p, p, p]
        L.gpupr_surface_fetch.argtypes = [p, p, ctypes.c_int, p]
        L.gpupr_solve_reduced_noalloc.argtypes = [ctypes.c_uint32, p, p, p, p, i32, u64, i32, p, p]
        L.gpupr_noalloc_prepare.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
        L.gpupr_graph_cut_batch.argtypes = [ctypes.c_uint32, p, p, p, ctypes.c_int, p, p, p,
                                            ctypes.c_int, f64, p, p, ctypes.c_int, p, p, p]
        L.gpupr_server_create.argtypes = [ctypes.c_uint64, ctypes.c_uint32, p, ctypes.POINTER(p)]
        L.gpupr_server_create_lanes.argtypes = [ctypes.c_uint64, ctypes.c_uint32, p, ctypes.c_uint64,
                                                ctypes.POINTER(p)]
        L.gpupr_server_submit.argtypes = [p, p, ctypes.c_uint64, p, p, p, ctypes.c_uint64, f64,
                                          p, ctypes.POINTER(ctypes.c_uint64)]
        L.gpupr_server_wait.argtypes = [p, ctypes.c_uint64, f64, p]
        L.gpupr_server_destroy.argtypes = [p]
        L.gpupr_upload_topology.argtypes = [p, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64,
                                            ctypes.c_int32, p, p]
        L.gpupr_edge_audit.argtypes = [p, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                       ctypes.POINTER(ctypes.c_uint64), p]
        L.gpupr_sample_tet_labels.argtypes = [p, p, ctypes.c_uint64, ctypes.c_int, p, ctypes.c_uint64,
                                              ctypes.c_int, p, p, f64, f64, p, ctypes.c_int, p, p]
        L.gpupr_autotune.argtypes = [p, ctypes.c_uint64, ctypes.c_int, p, p, ctypes.c_uint64, p, ctypes.c_int,
                                     f64, ctypes.c_int32, ctypes.c_int32, p, p]
        L.gpupr_tune_table.argtypes = [p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
        L.gpupr_tune_table_set.argtypes = [p, ctypes.c_uint32]
        L.gpupr_autotune_batch.argtypes = [ctypes.c_uint32, p, p, p, ctypes.c_int, p, p, p, ctypes.c_int,
                                           f64, ctypes.c_int32, ctypes.c_int32, p, p]
        L.gpupr_batch_tune_table.argtypes = [p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
        L.gpupr_batch_tune_table_set.argtypes = [p, ctypes.c_uint32]
        L.gpupr_release_cached_memory.argtypes = []
        L.gpupr_selftest_bounded_wait.argtypes = [ctypes.c_uint32, p]
        for name in header_functions():
            fn = getattr(L, name)
            if name not in ("gpupr_status_string", "gpupr_last_error", "gpupr_abi_version"):
                fn.restype = ctypes.c_int
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        msg = lib().gpupr_last_error().decode() or lib().gpupr_status_string(rc).decode()
        raise GpuprError(rc, msg)


def _dp(t):
    """device pointer of a torch CUDA tensor"""
    return ctypes.c_void_p(t.data_ptr())


def _hp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _stream(torch, device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def options(**kw):
    o = SolveOptions()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def graph_cut(vertices, tets, nbrs, labels, fill_T, threads=16, global_relabel_period=1024,
              max_rounds=2000000, local_steps=8, opts=None, out=None):
    """gpupr_graph_cut(_ex).  ``tets``/``nbrs`` are CUDA int32 tensors.
    ``vertices``/``labels`` may be numpy arrays (host) or CUDA tensors.
    Returns (labels_out, stats dict); labels_out matches ``out`` placement
    (a new numpy array when out is None and labels are on the host)."""
    import torch

    v_dev = isinstance(vertices, torch.Tensor)
    l_dev = isinstance(labels, torch.Tensor)
    N = int(tets.shape[0])
    if out is None:
        out = torch.empty(N, dtype=torch.uint8, device=tets.device) if l_dev else np.empty(N, np.uint8)
    o_dev = isinstance(out, torch.Tensor)
    if v_dev:
        vp = _dp(vertices)
    else:
        vertices = np.ascontiguousarray(vertices, np.float64)
        vp = _hp(vertices)
    if not l_dev:
        labels = np.ascontiguousarray(labels, np.uint8)
    lp = _dp(labels) if l_dev else _hp(labels)
    op = _dp(out) if o_dev else _hp(out)
    st = CutStats()
    nv = int(vertices.shape[0])
    if opts is None:
        rc = lib().gpupr_graph_cut(vp, nv, int(v_dev), _dp(tets), _dp(nbrs), N, lp, int(l_dev),
                                   float(fill_T), int(threads), int(global_relabel_period),
                                   int(max_rounds), int(local_steps), op, int(o_dev),
                                   _stream(torch, tets.device), ctypes.byref(st))
    else:
        rc = lib().gpupr_graph_cut_ex(vp, nv, int(v_dev), _dp(tets), _dp(nbrs), N, lp, int(l_dev),
                                      float(fill_T), int(threads), ctypes.byref(opts), op,
                                      int(o_dev), _stream(torch, tets.device), ctypes.byref(st))
    check(rc)
    return out, st.as_dict()


def pack_batch(graphs):
    """Concatenate graphs (dicts with vertices/tets/neighbors/labels, local
    ids) -> (tet_offsets, vertex_offsets, vertices, tets, neighbors, labels)."""
    toff = np.zeros(len(graphs) + 1, np.uint64)
    voff = np.zeros(len(graphs) + 1, np.uint64)
    for k, g in enumerate(graphs):
        toff[k + 1] = toff[k] + len(g["tets"])
        voff[k + 1] = voff[k] + len(g["vertices"])
    V = np.ascontiguousarray(np.concatenate([g["vertices"] for g in graphs]), np.float64)
    T = np.ascontiguousarray(np.concatenate([g["tets"] for g in graphs]), np.int32)
    Nb = np.ascontiguousarray(np.concatenate([g["neighbors"] for g in graphs]), np.int32)
    L = np.ascontiguousarray(np.concatenate([g["labels"] for g in graphs]), np.uint8)
    return toff, voff, V, T, Nb, L


def graph_cut_batch(toff, voff, vertices, tets, nbrs, labels, fill_T, opts=None, out=None):
    """gpupr_graph_cut_batch.  tets/nbrs: CUDA int32 tensors (local ids,
    concatenated); vertices/labels numpy or CUDA.  Returns (labels_out,
    items list of dicts, stats dict)."""
    import torch

    G = len(toff) - 1
    toff = np.ascontiguousarray(toff, np.uint64)
    voff = np.ascontiguousarray(voff, np.uint64)
    v_dev = isinstance(vertices, torch.Tensor)
    l_dev = isinstance(labels, torch.Tensor)
    N = int(toff[-1])
    if out is None:
        out = torch.empty(N, dtype=torch.uint8, device=tets.device) if l_dev else np.empty(N, np.uint8)
    o_dev = isinstance(out, torch.Tensor)
    if not v_dev:
        vertices = np.ascontiguousarray(vertices, np.float64)
    if not l_dev:
        labels = np.ascontiguousarray(labels, np.uint8)
    items = (BatchItem * max(G, 1))()
    st = CutStats()
    check(lib().gpupr_graph_cut_batch(
        G, _hp(toff), _hp(voff), _dp(vertices) if v_dev else _hp(vertices), int(v_dev), _dp(tets),
        _dp(nbrs), _dp(labels) if l_dev else _hp(labels), int(l_dev), float(fill_T),
        ctypes.byref(opts) if opts is not None else None, _dp(out) if o_dev else _hp(out), int(o_dev),
        _stream(torch, tets.device), items, ctypes.byref(st)))
    return out, [{k: getattr(items[i], k) for k, _ in BatchItem._fields_} for i in range(G)], st.as_dict()


class Server:
    """Continuous-batching cut server (gpupr_server_*): submit() host graphs
    at any time, wait() for each result.  split_tets=None: the library's
    default two lanes (split at 2M tets); 0: one lane; else the split."""

    def __init__(self, hbm_budget_bytes=0, opts=None, max_batch=0, split_tets=None):
        import torch

        torch.cuda.init()
        lib()
        self._h = ctypes.c_void_p()
        o = ctypes.byref(opts) if opts is not None else None
        if split_tets is None:
            check(_lib.gpupr_server_create(int(hbm_budget_bytes), int(max_batch), o, ctypes.byref(self._h)))
        else:
            check(_lib.gpupr_server_create_lanes(int(hbm_budget_bytes), int(max_batch), o,
                                                 int(split_tets), ctypes.byref(self._h)))
        self._held = {}

    def submit(self, vertices, tets, nbrs, labels, fill_T=10.0):
        """Queue one cut; the arrays are held (the server reads them in
        place) until wait() returns for the request."""
        V = np.ascontiguousarray(vertices, np.float64)
        T = np.ascontiguousarray(tets, np.int32)
        Nb = np.ascontiguousarray(nbrs, np.int32)
        L = np.ascontiguousarray(labels, np.uint8)
        out = np.empty(max(len(L), 1), np.uint8)
        rid = ctypes.c_uint64(0)
        check(_lib.gpupr_server_submit(self._h, _hp(V), len(V), _hp(T), _hp(Nb), _hp(L), len(L),
                                       float(fill_T), _hp(out), ctypes.byref(rid)))
        self._held[rid.value] = (V, T, Nb, L, out)
        return rid.value

    def wait(self, rid, timeout_s=0.0):
        res = RequestResult()
        rc = _lib.gpupr_server_wait(self._h, ctypes.c_uint64(rid), float(timeout_s), ctypes.byref(res))
        if rc != 0 and res.id != rid:   # not finished (or unknown id): arrays stay held
            check(rc)
        held = self._held.pop(rid)
        check(rc)
        return held[4][:len(held[3])], {k: getattr(res, k) for k, _ in RequestResult._fields_}

    def close(self):
        if self._h:
            _lib.gpupr_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._held.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def build_reduced(vertices, tets, nbrs, labels, fill_T):
    """gpupr_build_reduced: the reduced graph copied back to the host."""
    import torch

    vertices = np.ascontiguousarray(vertices, np.float64)
    labels = np.ascontiguousarray(labels, np.uint8)
    N = int(tets.shape[0])
    f2f = np.empty(max(N, 1), np.int32)
    old = np.empty(max(N, 1), np.uint32)
    nbr = np.empty((max(N, 1), 4), np.int32)
    res = np.empty((max(N, 1), 4), np.uint32)
    term = np.empty(max(N, 1), np.int32)
    rev = np.empty(max(N, 1), np.uint8)
    info = np.zeros(8, np.int64)
    check(lib().gpupr_build_reduced(_hp(vertices), vertices.shape[0], 0, _dp(tets), _dp(nbrs), N,
                                    _hp(labels), 0, float(fill_T), _hp(f2f), _hp(old), _hp(nbr),
                                    _hp(res), _hp(term), _hp(rev), _hp(info),
                                    _stream(torch, tets.device)))
    F = int(info[0])
    keys = ("free_n", "fixed_source", "fixed_sink", "full_refs", "free_refs", "terminal_edges",
            "terminal_base_flow", "n_full")
    return dict(full_to_free=f2f[:N], free_old=old[:F], nbr=nbr[:F], res=res[:F], term=term[:F],
                rev=rev[:F], info={k: int(v) for k, v in zip(keys, info)})


def solve_reduced(nbr, res, term, local_steps=8, global_relabel_period=1024, max_rounds=2000000,
                  want_excess=False):
    """gpupr_solve_reduced on CUDA tensors nbr int32[n,4], res int32/uint32
    [n,4], term int32[n] (modified in place).  Returns (partition numpy,
    stats, excess tensor or None)."""
    import torch

    n = int(nbr.shape[0])
    part = np.zeros(max(n, 1), np.uint8)
    exc = torch.zeros(max(n, 1), dtype=torch.int64, device=nbr.device) if want_excess else None
    st = CutStats()
    check(lib().gpupr_solve_reduced(n, _dp(nbr), _dp(res), _dp(term), _hp(part),
                                    int(global_relabel_period), int(max_rounds), int(local_steps),
                                    _dp(exc) if exc is not None else None,
                                    _stream(torch, nbr.device), ctypes.byref(st)))
    return part[:n], st.as_dict(), exc


def noalloc_prepare():
    """gpupr_noalloc_prepare on the current device; returns the static
    scratch array's size in bytes."""
    nb = ctypes.c_uint64(0)
    check(lib().gpupr_noalloc_prepare(ctypes.byref(nb)))
    return int(nb.value)


def solve_reduced_noalloc(nbr, res, term, part, local_steps=8, global_relabel_period=1024,
                          max_rounds=2000000):
    """gpupr_solve_reduced_noalloc on CUDA tensors (res/term modified in place,
    the partition written to the uint8 CUDA tensor part).  Returns stats."""
    import torch

    st = CutStats()
    check(lib().gpupr_solve_reduced_noalloc(int(nbr.shape[0]), _dp(nbr), _dp(res), _dp(term), _dp(part),
                                            int(global_relabel_period), int(max_rounds),
                                            int(local_steps), _stream(torch, nbr.device),
                                            ctypes.byref(st)))
    return st.as_dict()


def solve_ell(nbr, cap, src, snk, opts=None):
    """gpupr_solve_ell on CUDA tensors.  Returns (max_flow, partition tensor,
    stats)."""
    import torch

    n = int(nbr.shape[0])
    part = torch.empty(max(n, 1), dtype=torch.uint8, device=nbr.device)
    flow = ctypes.c_int64(0)
    st = CutStats()
    check(lib().gpupr_solve_ell(n, _dp(nbr), _dp(cap), _dp(src), _dp(snk),
                                ctypes.byref(opts) if opts is not None else None,
                                ctypes.byref(flow), _dp(part), _stream(torch, nbr.device),
                                ctypes.byref(st)))
    return int(flow.value), part[:n], st.as_dict()


def surface(labels, vertices, tets, nbrs):
    """gpupr_surface_count + fetch with host labels/vertices -> (V, F)."""
    import torch

    labels = np.ascontiguousarray(labels, np.uint8)
    vertices = np.ascontiguousarray(vertices, np.float64)
    nf = ctypes.c_uint64(0)
    nu = ctypes.c_uint64(0)
    s = _stream(torch, tets.device)
    check(lib().gpupr_surface_count(_hp(labels), 0, _hp(vertices), vertices.shape[0], 0, _dp(tets),
                                    _dp(nbrs), int(tets.shape[0]), ctypes.byref(nf),
                                    ctypes.byref(nu), s))
    F = np.empty((max(nf.value, 1), 3), np.int32)
    V = np.empty((max(nu.value, 1), 3), np.float64)
    check(lib().gpupr_surface_fetch(_hp(F), _hp(V), 0, s))
    return V[: nu.value], F[: nf.value]


def bounded_wait_selftest(limit_us=200_000):
    import torch

    return lib().gpupr_selftest_bounded_wait(int(limit_us), _stream(torch))


def upload_topology(host, out):
    """gpupr_upload_topology: host Nx4 int32/int64 array (any strides) ->
    the contiguous int32 CUDA tensor ``out``."""
    import torch

    a = np.asarray(host)
    check(lib().gpupr_upload_topology(ctypes.c_void_p(a.ctypes.data), a.shape[0], a.strides[0],
                                      a.strides[1], a.itemsize, _dp(out), _stream(torch, out.device)))
    return out


def edge_audit(faces):
    """gpupr_edge_audit: faces numpy Fx3 (host) or CUDA int32 tensor.
    Returns (bad_groups, table_bytes)."""
    import torch

    bad = ctypes.c_uint64(0)
    nbytes = ctypes.c_uint64(0)
    if isinstance(faces, torch.Tensor):
        check(lib().gpupr_edge_audit(_dp(faces), faces.shape[0], 1, ctypes.byref(bad), ctypes.byref(nbytes),
                                     _stream(torch, faces.device)))
    else:
        f = np.ascontiguousarray(faces, np.int32).reshape(-1, 3)
        check(lib().gpupr_edge_audit(_hp(f), f.shape[0], 0, ctypes.byref(bad), ctypes.byref(nbytes),
                                     _stream(torch)))
    return int(bad.value), int(nbytes.value)


class BrickGrid(ctypes.Structure):
    _fields_ = [("voxel_size", ctypes.c_double), ("origin", ctypes.c_int32 * 3),
                ("dims", ctypes.c_int32 * 3), ("background", ctypes.c_float),
                ("on_device", ctypes.c_int32), ("table", ctypes.c_void_p), ("values", ctypes.c_void_p),
                ("n_bricks", ctypes.c_uint64)]


def sample_tet_labels(grid, vertices, tets, bbox_min, bbox_max, padding, threshold, device_out=False):
    """gpupr_sample_tet_labels.  grid: dict as made by synth.brick_udf (host
    arrays, or CUDA tensors for table/values).  vertices/tets: numpy or CUDA.
    Returns (labels, samples) (numpy, or CUDA tensors with device_out)."""
    import torch

    tab, val = grid["table"], grid["values"]
    g_dev = isinstance(tab, torch.Tensor)
    if not g_dev:
        tab = np.ascontiguousarray(tab, np.int32)
        val = np.ascontiguousarray(val, np.float32)
    g = BrickGrid(float(grid["voxel_size"]), (ctypes.c_int32 * 3)(*[int(x) for x in grid["origin"]]),
                  (ctypes.c_int32 * 3)(*[int(x) for x in grid["dims"]]), float(grid["background"]), int(g_dev),
                  _dp(tab) if g_dev else _hp(tab), _dp(val) if g_dev else _hp(val),
                  int((val.numel() if g_dev else val.size) // 512))
    v_dev = isinstance(vertices, torch.Tensor)
    t_dev = isinstance(tets, torch.Tensor)
    if not v_dev:
        vertices = np.ascontiguousarray(vertices, np.float64)
    if not t_dev:
        tets = np.ascontiguousarray(tets, np.int32)
    n = int(tets.shape[0])
    if device_out:
        dev = tets.device if t_dev else torch.device("cuda")
        lab = torch.empty(max(n, 1), dtype=torch.uint8, device=dev)
        udf = torch.empty(max(n, 1), dtype=torch.float32, device=dev)
    else:
        lab = np.empty(max(n, 1), np.uint8)
        udf = np.empty(max(n, 1), np.float32)
    bmin = np.ascontiguousarray(bbox_min, np.float64)
    bmax = np.ascontiguousarray(bbox_max, np.float64)
    check(lib().gpupr_sample_tet_labels(
        ctypes.byref(g), _dp(vertices) if v_dev else _hp(vertices), int(vertices.shape[0]), int(v_dev),
        _dp(tets) if t_dev else _hp(tets), n, int(t_dev), _hp(bmin), _hp(bmax), float(padding),
        float(threshold), _dp(lab) if device_out else _hp(lab), int(device_out),
        _dp(udf) if device_out else _hp(udf), _stream(torch, tets.device if t_dev else None)))
    return lab[:n], udf[:n]


class TuneEntry(ctypes.Structure):
    _fields_ = [("size_class", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("work_relabel_factor", ctypes.c_double), ("solve_ms", ctypes.c_double),
                ("default_ms", ctypes.c_double), ("chain_hops", ctypes.c_int32),
                ("chain_max_active", ctypes.c_int32)]


def autotune(vertices, tets, nbrs, labels, fill_T, local_steps=8, reps=3):
    """gpupr_autotune on one cut (tets/nbrs CUDA int32): returns the chosen
    entry of the graph's size class as a dict."""
    import torch

    v_dev = isinstance(vertices, torch.Tensor)
    l_dev = isinstance(labels, torch.Tensor)
    if not v_dev:
        vertices = np.ascontiguousarray(vertices, np.float64)
    if not l_dev:
        labels = np.ascontiguousarray(labels, np.uint8)
    e = TuneEntry()
    check(lib().gpupr_autotune(_dp(vertices) if v_dev else _hp(vertices), int(vertices.shape[0]), int(v_dev),
                               _dp(tets), _dp(nbrs), int(tets.shape[0]), _dp(labels) if l_dev else _hp(labels),
                               int(l_dev), float(fill_T), int(local_steps), int(reps), ctypes.byref(e),
                               _stream(torch, tets.device)))
    return {k: getattr(e, k) for k, _ in TuneEntry._fields_}


def autotune_batch(toff, voff, vertices, tets, nbrs, labels, fill_T, local_steps=8, reps=3):
    """gpupr_autotune_batch on one packed batch (arguments as graph_cut_batch):
    returns the chosen entry of the batch's size bucket as a dict."""
    import torch

    G = len(toff) - 1
    toff = np.ascontiguousarray(toff, np.uint64)
    voff = np.ascontiguousarray(voff, np.uint64)
    v_dev = isinstance(vertices, torch.Tensor)
    l_dev = isinstance(labels, torch.Tensor)
    if not v_dev:
        vertices = np.ascontiguousarray(vertices, np.float64)
    if not l_dev:
        labels = np.ascontiguousarray(labels, np.uint8)
    e = TuneEntry()
    check(lib().gpupr_autotune_batch(G, _hp(toff), _hp(voff), _dp(vertices) if v_dev else _hp(vertices),
                                     int(v_dev), _dp(tets), _dp(nbrs), _dp(labels) if l_dev else _hp(labels),
                                     int(l_dev), float(fill_T), int(local_steps), int(reps), ctypes.byref(e),
                                     _stream(torch, tets.device)))
    return {k: getattr(e, k) for k, _ in TuneEntry._fields_}


def batch_tune_table():
    """The batch tuning table as a list of dicts."""
    cnt = ctypes.c_uint32(0)
    check(lib().gpupr_batch_tune_table(None, 0, ctypes.byref(cnt)))
    arr = (TuneEntry * max(cnt.value, 1))()
    check(lib().gpupr_batch_tune_table(arr, cnt.value, ctypes.byref(cnt)))
    return [{k: getattr(arr[i], k) for k, _ in TuneEntry._fields_} for i in range(cnt.value)]


def set_batch_tune_table(entries):
    arr = (TuneEntry * max(len(entries), 1))()
    for i, e in enumerate(entries):
        for k, _ in TuneEntry._fields_:
            setattr(arr[i], k, e[k])
    check(lib().gpupr_batch_tune_table_set(arr, len(entries)))


def tune_table():
    n = ctypes.c_uint32(0)
    check(lib().gpupr_tune_table(None, 0, ctypes.byref(n)))
    arr = (TuneEntry * max(n.value, 1))()
    check(lib().gpupr_tune_table(arr, n.value, ctypes.byref(n)))
    return [{k: getattr(arr[i], k) for k, _ in TuneEntry._fields_} for i in range(n.value)]


def set_tune_table(entries):
    arr = (TuneEntry * max(len(entries), 1))()
    for i, e in enumerate(entries):
        for k, _ in TuneEntry._fields_:
            setattr(arr[i], k, e.get(k, 0))
    check(lib().gpupr_tune_table_set(arr, len(entries)))


def save_tune_table(path):
    """Keep the autotuned table across processes (JSON)."""
    import json

    with open(path, "w") as f:
        json.dump(tune_table(), f, indent=1)


def load_tune_table(path):
    import json

    with open(path) as f:
        set_tune_table(json.load(f))


def release_cached_memory():
    check(lib().gpupr_release_cached_memory())
