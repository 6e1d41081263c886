"""C-ABI library and drop-in module on the CPU: they load, export every
declared symbol, and reject bad arguments with the reference's messages
before touching a GPU (native/gpupr/wtivo_gpupr_bindings.cpp:114-133)."""
from __future__ import annotations

import ctypes
import inspect

import numpy as np
import pytest
import torch


def test_library_exports_header(built):
    import gpupr_capi

    names = gpupr_capi.header_functions()
    assert "gpupr_graph_cut" in names and "gpupr_solve_reduced" in names
    L = ctypes.CDLL(str(gpupr_capi.LIB_PATH))
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert gpupr_capi.lib().gpupr_abi_version() == 6
    assert gpupr_capi.lib().gpupr_status_string(9) == b"GPUPr-FAST-v6.30 max macro rounds exceeded"


def test_module_exports_reference_names(built):
    import wtivo_gpupr

    for name in ("graph_cut_fast", "graph_cut_gpupr_fast_v630", "surface_extraction_topology_cuda"):
        assert hasattr(wtivo_gpupr, name)
    # keyword names are accepted (validation fails later, on the vertices)
    t = torch.zeros((2, 4), dtype=torch.int32)
    kw = dict(tets_cuda=t, neighbors_cuda=t, labels=np.ones(2, np.uint8), fill_T=10.0, threads=16,
              global_relabel_period=1024, max_rounds=2000000, local_steps=8)
    for fn in (wtivo_gpupr.graph_cut_fast, wtivo_gpupr.graph_cut_gpupr_fast_v630):
        with pytest.raises(RuntimeError, match="vertices must be float64 Nx3"):
            fn(vertices=np.zeros((2, 2)), **kw)
    with pytest.raises(RuntimeError, match="vertices must be float64 Nx3"):
        wtivo_gpupr.surface_extraction_topology_cuda(labels=np.ones(2, np.uint8),
                                                     vertices=np.zeros(3), tets_cuda=t,
                                                     neighbors_cuda=t, threads=16)
    doc = wtivo_gpupr.graph_cut_fast.__doc__.split("\n")[0]
    pos = [doc.index(x) for x in ("threads:", "= 16", "global_relabel_period:", "= 1024",
                                  "max_rounds:", "= 2000000", "local_steps:", "= 8")]
    assert pos == sorted(pos)
    assert "= 16" in wtivo_gpupr.surface_extraction_topology_cuda.__doc__


def _args(n=8):
    V = np.zeros((4, 3))
    t = torch.zeros((n, 4), dtype=torch.int32)
    lab = np.ones(n, np.uint8)
    return V, t, t.clone(), lab


def test_module_validation_order(built):
    import wtivo_gpupr as g

    V, t, nb, lab = _args()
    with pytest.raises(RuntimeError, match="vertices must be float64 Nx3"):
        g.graph_cut_fast(np.zeros((4, 2)), t, nb, lab, 10.0)
    with pytest.raises(RuntimeError, match="tets/neighbors must be CUDA tensors"):
        g.graph_cut_fast(V, t, nb, lab, 10.0)
    with pytest.raises(RuntimeError, match="tets/neighbors must be contiguous CUDA int32 Nx4 with same N"):
        g.surface_extraction_topology_cuda(lab, V, t, nb)
    with pytest.raises(TypeError):
        g.graph_cut_fast(V, "not a tensor", nb, lab, 10.0)


def test_capi_rejects_host_topology(built):
    """Host pointers for tets/neighbors are refused, not read."""
    import gpupr_capi

    st = gpupr_capi.CutStats()
    tets = np.zeros((8, 4), np.int32)
    lab = np.ones(8, np.uint8)
    out = np.empty(8, np.uint8)
    V = np.zeros((4, 3))
    rc = gpupr_capi.lib().gpupr_graph_cut(
        V.ctypes.data_as(ctypes.c_void_p), 4, 0, tets.ctypes.data_as(ctypes.c_void_p),
        tets.ctypes.data_as(ctypes.c_void_p), 8, lab.ctypes.data_as(ctypes.c_void_p), 0, 10.0,
        16, 1024, 0, 8, out.ctypes.data_as(ctypes.c_void_p), 0, None, ctypes.byref(st))
    assert rc != 0
    # an empty graph is a no-op that echoes threads/local_steps
    rc = gpupr_capi.lib().gpupr_graph_cut(None, 0, 0, None, None, 0, None, 0, 10.0, 0, 1024, 0, 5,
                                          None, 0, None, ctypes.byref(st))
    assert rc == 0 and st.threads == 1 and st.local_steps == 5


def test_python_side_is_plumbing_only():
    """The drop-in path has no CPU solver to fall back to."""
    import gpupr_capi

    src = inspect.getsource(gpupr_capi)
    assert "oracle" not in src.replace("no CPU fallback", "")


def test_topology_upload_shape_check(built):
    """wtivo.py:297-299: the shape is checked before anything is copied."""
    import wtivo_gpupr

    with pytest.raises(RuntimeError, match=r"tets: expected Nx4 topology array, got \(5, 3\)"):
        wtivo_gpupr.topology_to_cuda_chunked(np.zeros((5, 3), np.int32), "tets")
    with pytest.raises(RuntimeError, match=r"nb: expected Nx4 topology array, got \(8,\)"):
        wtivo_gpupr.topology_to_cuda_chunked(np.zeros(8, np.int64), "nb")


def test_is_watertight_checks_before_the_gpu(built):
    """wtivo_core.cpp:408-413: shape check and the empty-mesh answer."""
    import wtivo_gpupr

    with pytest.raises(RuntimeError, match="is_watertight expects Fx3 int32 faces"):
        wtivo_gpupr.is_watertight(np.zeros((5, 2), np.int32), 4)
    with pytest.raises(RuntimeError, match="is_watertight expects Fx3 int32 faces"):
        wtivo_gpupr.is_watertight(np.zeros(9, np.int32))
    assert wtivo_gpupr.is_watertight(np.zeros((0, 3), np.int32), 16) == (False, 0, 0.0, 0)


def test_tune_table_round_trip(built, tmp_path):
    """The autotuner's table is host state: set, read back, save/load,
    reject invalid entries, clear."""
    import gpupr_capi

    entries = [dict(size_class=18, blocks_per_sm=1, work_relabel_factor=2.0, solve_ms=10.0, default_ms=11.0,
                    chain_hops=4, chain_max_active=32768),
               dict(size_class=26, blocks_per_sm=4, work_relabel_factor=0.5, solve_ms=120.0, default_ms=130.0,
                    chain_hops=1, chain_max_active=1)]
    gpupr_capi.set_tune_table(entries)
    assert gpupr_capi.tune_table() == entries
    p = tmp_path / "tune.json"
    gpupr_capi.save_tune_table(p)
    gpupr_capi.set_tune_table([])
    assert gpupr_capi.tune_table() == []
    gpupr_capi.load_tune_table(p)
    assert gpupr_capi.tune_table() == entries
    for bad in (dict(entries[0], blocks_per_sm=0), dict(entries[0], size_class=40),
                dict(entries[0], work_relabel_factor=0.0), dict(entries[0], chain_hops=0)):
        with pytest.raises(gpupr_capi.GpuprError):
            gpupr_capi.set_tune_table([bad])
    assert gpupr_capi.tune_table() == entries        # a rejected set changes nothing
    gpupr_capi.set_tune_table([])


def test_python_structs_match_the_header(tmp_path):
    """The ctypes mirrors of the C structs have the header's size and field
    offsets (checked with a C program compiled against include/wtivo_gpupr.h)."""
    import subprocess

    import gpupr_capi

    checks = {"gpupr_cut_stats": gpupr_capi.CutStats, "gpupr_solve_options": gpupr_capi.SolveOptions,
              "gpupr_batch_item": gpupr_capi.BatchItem, "gpupr_request_result": gpupr_capi.RequestResult,
              "gpupr_tune_entry": gpupr_capi.TuneEntry, "gpupr_brick_grid": gpupr_capi.BrickGrid}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wtivo_gpupr.h"', "int main(void) {"]
    for cname, py in checks.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "sizes.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "sizes"
    subprocess.check_call(["gcc", "-I", str(gpupr_capi.HEADER.parent), str(src), "-o", str(exe)])
    got = dict(line.split() for line in subprocess.check_output([str(exe)], text=True).splitlines())
    for cname, py in checks.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_integration_stub_matches_the_stats_struct():
    """The ctypes stub a maintainer would paste from INTEGRATION.md declares
    as many eight-byte fields as gpupr_cut_stats has, and names the ABI
    version the library reports."""
    import re
    from pathlib import Path

    import gpupr_capi

    text = (Path(__file__).resolve().parents[1] / "INTEGRATION.md").read_text()
    m = re.search(r"class Stats\(ctypes.Structure\):.*?\((\d+) eight-byte fields, ABI (\d+)\).*?"
                  r"_fields_ = \[(.*?)\] \+ \\\s*\[\(\"pad%d\" % i, ctypes.c_uint64\) for i in range\((\d+)\)\]",
                  text, flags=re.S)
    assert m, "Stats stub not found in INTEGRATION.md"
    fields, abi, named, pads = int(m.group(1)), int(m.group(2)), m.group(3), int(m.group(4))
    n_named = named.count("ctypes.c_")
    assert ctypes.sizeof(gpupr_capi.CutStats) == 8 * fields == 8 * (n_named + pads)
    header = gpupr_capi.HEADER.read_text()
    assert int(re.search(r"#define GPUPR_ABI_VERSION (\d+)", header).group(1)) == abi


def test_every_header_function_has_argtypes(built):
    """The ctypes binding declares argument types for every function the
    header declares (an undeclared one would be called with guessed types)."""
    import gpupr_capi

    L = gpupr_capi.lib()
    missing = [n for n in gpupr_capi.header_functions()
               if getattr(L, n).argtypes is None and n not in ("gpupr_abi_version",)]
    assert not missing, missing
