"""Golden vectors made by the REFERENCE module (compiled from its sources and
run on a B200 by tests/golden/make_golden.py): the oracle must reproduce
them exactly on the CPU, and the CUDA path on the GPU."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import to_cuda
from oracle import oracle as orc

FILES = sorted((Path(__file__).resolve().parent / "golden").glob("ref_*.npz"))
KEYS = ("adjusted_flow", "raw_flow", "full_E", "free_E", "fixed_source", "fixed_sink",
        "terminal_edges")


def load(f):
    z = np.load(f)
    return {k: z[k] for k in z.files}


def test_fixtures_present():
    assert len(FILES) >= 5


@pytest.mark.parametrize("f", FILES, ids=[f.stem for f in FILES])
def test_oracle_matches_reference_outputs(f):
    z = load(f)
    lab, st = orc.graph_cut(z["vertices"], z["tets"], z["neighbors"], z["labels_in"],
                            float(z["fill_T"]))
    assert np.array_equal(lab, z["labels_out"])
    for k in KEYS:
        assert st[k] == int(z[f"ref_{k}"]), k
    # the reference's build-side sizes follow from the same counts
    assert int(z["ref_map_bytes"]) == len(z["tets"]) * 4 + st["free_n"] * 4
    assert int(z["ref_graph_bytes"]) == st["free_n"] * 36
    V, F = orc.surface(z["labels_out"], z["vertices"], z["tets"], z["neighbors"])
    assert np.array_equal(F, z["surface_F"]) and np.array_equal(V, z["surface_V"])


@pytest.mark.gpu
@pytest.mark.parametrize("f", FILES, ids=[f.stem for f in FILES])
def test_cuda_path_matches_reference_outputs(built, f):
    import wtivo_gpupr

    z = load(f)
    tets, nbrs = to_cuda(z["tets"], z["neighbors"])
    r = wtivo_gpupr.graph_cut_fast(z["vertices"], tets, nbrs, z["labels_in"], float(z["fill_T"]))
    assert len(r) == int(z["tuple_len"])
    assert np.array_equal(np.asarray(r[0]), z["labels_out"])
    for i, k in ((1, "adjusted_flow"), (2, "raw_flow"), (5, "full_E"), (6, "free_E"),
                 (7, "fixed_source"), (8, "fixed_sink"), (9, "terminal_edges"),
                 (10, "threads"), (13, "map_bytes"), (15, "local_steps")):
        assert int(r[i]) == int(z[f"ref_{k}"]), k
    V, F = wtivo_gpupr.surface_extraction_topology_cuda(z["labels_out"], z["vertices"], tets, nbrs)
    assert np.array_equal(F, z["surface_F"]) and np.array_equal(V, z["surface_V"])
