"""Recipe: compile the reference's own graph-cut module from its sources.

TEST INFRASTRUCTURE ONLY.  Builds ``native/gpupr/wtivo_gpupr_bindings.cpp``
and ``native/gpupr/gpu_push_relabel_fast.cu`` exactly as they lie in the
reference checkout (read-only, never copied into this repository) into
``oracle/_ref/wtivo_gpupr_ref*.so`` for sm_100a, with the reference's own
flags (-O3 --std=c++17 for nvcc, scripts/build_gpupr.py:48; strict IEEE
doubles on the host: no FMA contraction, like MSVC /fp:precise at :68).
The module name is ``wtivo_gpupr_ref`` so it can sit beside the product's
``wtivo_gpupr``.  It is the reference partition source for the parity tests
and the ``--impl reference`` arm of bench.py on a machine with a GPU, which
uses the prebuilt .so (oracle/_ref is kept out of version control; the built
file is copied along with the working tree, not rebuilt there).

The reference checkout is read from $WTIVO_REFERENCE_SRC when it is set,
else from DEFAULT_SRC below.

    python oracle/build_ref.py [--src /path/to/reference]
"""
from __future__ import annotations

import argparse
import os
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_SRC = Path(os.environ.get("WTIVO_REFERENCE_SRC", "/root/reference"))


def built_module() -> Path | None:
    for p in sorted(OUT.glob("wtivo_gpupr_ref*.so")):
        return p
    return None


def build(src: Path = DEFAULT_SRC, quiet: bool = False, force: bool = False) -> Path:
    gp = src / "native" / "gpupr"
    sources = [gp / "wtivo_gpupr_bindings.cpp", gp / "gpu_push_relabel_fast.cu"]
    if not all(s.exists() for s in sources):
        raise FileNotFoundError(f"reference sources not found under {gp}")
    existing = built_module()
    if existing and not force and all(existing.stat().st_mtime >= s.stat().st_mtime for s in sources):
        return existing
    OUT.mkdir(exist_ok=True)
    bdir = OUT / "build"
    bdir.mkdir(exist_ok=True)
    os.environ.setdefault("MAX_JOBS", "4")
    # The system toolchain: a compiler wrapper that links the C++ runtime
    # statically into the module leaves two libstdc++ copies in the process,
    # which crashes the reference on its first std::cout of a double.
    for var, tool in (("CC", "gcc"), ("CXX", "g++")):
        path = shutil.which(tool, path="/usr/bin") or shutil.which(tool)
        if path:
            os.environ[var] = path
    from torch.utils.cpp_extension import load

    mod = load(
        name="wtivo_gpupr_ref",
        sources=[str(s) for s in sources],
        build_directory=str(bdir),
        extra_cflags=["-O2", "-std=c++17", "-ffp-contract=off"],
        extra_cuda_cflags=["-O3", "--std=c++17", "-gencode=arch=compute_100a,code=sm_100a"],
        with_cuda=True,
        verbose=not quiet,
    )
    so = Path(mod.__file__).resolve()
    dst = OUT / so.name
    if so != dst:
        shutil.copy2(so, dst)
    for name in ("graph_cut_fast", "graph_cut_gpupr_fast_v630", "surface_extraction_topology_cuda"):
        if not hasattr(mod, name):
            raise RuntimeError(f"reference module lacks {name}")
    return dst


def load_reference():
    """Import the built reference module (GPU box or here)."""
    import torch  # noqa: F401  (libtorch symbols must be loaded first)

    so = built_module()
    if so is None:
        raise ImportError("oracle/_ref/wtivo_gpupr_ref*.so is not built")
    if str(OUT) not in sys.path:
        sys.path.insert(0, str(OUT))
    import wtivo_gpupr_ref

    return wtivo_gpupr_ref


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=str(DEFAULT_SRC))
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(Path(a.src), force=a.force))
