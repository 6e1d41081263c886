"""Shared test setup: import paths, the ``gpu`` marker and cached inputs."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "wtivo-watertightvoxel_b200"
for p in (str(PKG), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def built():
    """Compile (incrementally) the CUDA library, the module and the oracle."""
    import build as pkg_build

    pkg_build.build_all()
    from oracle import oracle as orc

    orc.build_library()
    return True


_cache = {}


def cached_graph(kind: str, seed: int = 0, size: int = 20_000):
    """Small seeded cell graphs shared by the tests."""
    import synth

    key = (kind, seed, size)
    if key not in _cache:
        if kind == "proxy":
            g = synth.config1(seed, n_points=size)
        elif kind == "lattice":
            mv, mf = synth.defective_torus_knot(seed, n_faces=40_000)
            g = synth.lattice_graph(mv, mf, size, seed + 1)
            g["fill_T"] = 10.0
        elif kind == "box":
            g = synth.config3_graph(2, size, seed)
        elif kind == "torus":
            g = synth.config3_graph(1, size, seed)
        else:
            raise KeyError(kind)
        _cache[key] = g
    return _cache[key]


def to_cuda(*arrays):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]
