"""Build recipe of the B200 graph-cut library (in-tree, sm_100a only).

Outputs, next to this file:
  libwtivo_gpupr.so                 CUDA kernels + C ABI (include/wtivo_gpupr.h)
  wtivo_gpupr<EXT_SUFFIX>           the drop-in pybind11 module
  synth/libsynth.so                 seeded input generators (test/bench inputs)

    python build.py [--force] [--ptxas-v]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libwtivo_gpupr.so"
EXT = PKG / ("wtivo_gpupr" + sysconfig.get_config_var("EXT_SUFFIX"))

CU_SOURCES = ["graph_build.cu", "push_relabel.cu", "batch.cu", "surface.cu", "capi.cu", "server.cu", "hostio.cu", "audit.cu", "labels.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        p = Path(c) / "bin" / "nvcc"
        if c and p.exists():
            return str(p)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found")
    return found


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _headers():
    return [INCLUDE / "wtivo_gpupr.h", CSRC / "gpupr_internal.cuh"]


def compile_cu(src: str, force: bool, ptxas_v: bool) -> Path:
    out = BUILD / (Path(src).stem + ".o")
    if not force and not _stale(out, [CSRC / src, *_headers()]):
        return out
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
           "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(CSRC / src), "-o", str(out)]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if ptxas_v:
        sys.stderr.write(r.stderr)
    return out


def build_lib(force=False, ptxas_v=False) -> Path:
    BUILD.mkdir(exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(CU_SOURCES)) as ex:
        objs = list(ex.map(lambda s: compile_cu(s, force, ptxas_v), CU_SOURCES))
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.check_call([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs)])
        os.replace(tmp, LIB)
    return LIB


def build_module(force=False) -> Path:
    src = CSRC / "pymodule.cpp"
    if not force and not _stale(EXT, [src, LIB, INCLUDE / "wtivo_gpupr.h"]):
        return EXT
    import pybind11

    inc = sysconfig.get_paths()["include"]
    tmp = EXT.with_name(EXT.name + ".tmp")
    subprocess.check_call([
        "g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
        "-I", inc, "-I", pybind11.get_include(), "-I", str(INCLUDE), str(src),
        "-L", str(PKG), "-lwtivo_gpupr", "-Wl,-rpath,$ORIGIN", "-o", str(tmp),
    ])
    os.replace(tmp, EXT)
    return EXT


def build_all(force=False, ptxas_v=False):
    build_lib(force, ptxas_v)
    build_module(force)
    sys.path.insert(0, str(PKG))
    import synth  # noqa: E402

    synth.build_library(force)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    build_all(a.force, a.ptxas_v)
    print("built", LIB.name, EXT.name)
