"""Generate golden vectors by running the REFERENCE module on small seeded inputs.

Needs a CUDA GPU and the reference module compiled from its own sources by
oracle/build_ref.py (oracle/_ref/wtivo_gpupr_ref*.so).  For each case it
stores the inputs and the reference's outputs of graph_cut_fast (labels and
the 18-tuple) and of surface_extraction_topology_cuda on those labels:

    python tests/golden/make_golden.py OUT_DIR

The committed ref_*.npz fixtures were made with this script on a B200.
"""
from __future__ import annotations

import contextlib
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "wtivo-watertightvoxel_b200"))
sys.path.insert(0, str(ROOT))

TUPLE_KEYS = ("adjusted_flow", "raw_flow", "graph_bytes", "workspace_bytes", "full_E", "free_E",
              "fixed_source", "fixed_sink", "terminal_edges", "threads", "rounds",
              "global_relabels", "map_bytes", "build_seconds", "local_steps", "solve_seconds",
              "native_total_seconds")


def cases():
    import synth

    yield "proxy_s11", synth.config1(11, n_points=6_000)
    yield "proxy_s12", synth.config1(12, n_points=12_000)
    mv, mf = synth.defective_torus_knot(13, n_faces=30_000)
    g = synth.lattice_graph(mv, mf, 40_000, 14)
    g["fill_T"] = 10.0
    yield "knot_lattice_s13", g
    g = synth.config3_graph(2, 25_000, 15)
    yield "box_lattice_s15", g
    g = synth.config3_graph(1, 25_000, 16)
    g["fill_T"] = 3.5
    yield "torus_lattice_s16_fill3p5", g


@contextlib.contextmanager
def quiet_stdout():
    """The reference prints progress lines from C++; keep them out of logs."""
    sys.stdout.flush()
    fd = os.dup(1)
    dn = os.open(os.devnull, os.O_WRONLY)
    os.dup2(dn, 1)
    try:
        yield
    finally:
        sys.stdout.flush()
        os.dup2(fd, 1)
        os.close(fd)
        os.close(dn)


def main(out_dir: str):
    import torch

    from oracle.build_ref import load_reference

    ref = load_reference()
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    for name, g in cases():
        tets = torch.from_numpy(g["tets"]).cuda()
        nbrs = torch.from_numpy(g["neighbors"]).cuda()
        with quiet_stdout():
            r = ref.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], float(g["fill_T"]),
                                   16, 1024, 2000000, 8)
            labels_out = np.asarray(r[0], np.uint8)
            V, F = ref.surface_extraction_topology_cuda(labels_out, g["vertices"], tets, nbrs, 16)
        stats = {k: np.asarray(v) for k, v in zip(TUPLE_KEYS, r[1:])} if len(r) == 18 else {}
        np.savez_compressed(out / f"ref_{name}.npz", vertices=g["vertices"], tets=g["tets"],
                            neighbors=g["neighbors"], labels_in=g["labels"],
                            fill_T=np.float64(g["fill_T"]), labels_out=labels_out,
                            tuple_len=np.int64(len(r)), surface_V=np.asarray(V),
                            surface_F=np.asarray(F), **{f"ref_{k}": v for k, v in stats.items()})
        print(name, len(g["tets"]), "flow", int(r[1]), "rounds", int(r[11]) if len(r) == 18 else 0,
              flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).resolve().parent))
