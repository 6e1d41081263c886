"""Parity at the benchmark's full size (80.3M tets, 77.0M free nodes): the
labels and flows equal the reference module's on the same B200, and the
returned flow equals the capacity of the returned cut in the original
reduced graph (max-flow = min-cut, a certificate of optimality that needs no
other solver)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from gpu_helpers import cut_capacity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    import synth

    return synth.config2(0, n_tets=80_000_000)


def test_fullsize_certificate(built, big):
    import gpupr_capi

    g = big
    tets = torch.from_numpy(g["tets"]).cuda()
    nbrs = torch.from_numpy(g["neighbors"]).cuda()
    r = gpupr_capi.build_reduced(g["vertices"], tets, nbrs, g["labels"], 10.0)
    nbr = torch.from_numpy(r["nbr"]).cuda()
    res = torch.from_numpy(r["res"].view(np.int32)).cuda()
    term = torch.from_numpy(r["term"]).cuda()
    cap0, term0 = res.clone(), term.clone()
    part, st, exc = gpupr_capi.solve_reduced(nbr, res, term, want_excess=True)
    assert cut_capacity(nbr, cap0, term0, torch.from_numpy(part).cuda()) == st["raw_flow"]
    assert int(term0.clamp_min(0).long().sum()) == st["raw_flow"] + int(exc.sum())
    # the full cut through the drop-in reports the same flow
    out, st2 = gpupr_capi.graph_cut(g["vertices"], tets, nbrs, g["labels"], 10.0)
    assert st2["raw_flow"] == st["raw_flow"]
    assert st2["adjusted_flow"] == st["raw_flow"] + r["info"]["terminal_base_flow"]
    free = r["full_to_free"] >= 0
    assert np.array_equal(out[free], part[r["full_to_free"][free]])


def test_fullsize_identical_to_reference(built, big, capfd):
    from oracle.build_ref import built_module, load_reference

    import wtivo_gpupr

    if built_module() is None:
        pytest.skip("reference module not built (oracle/build_ref.py needs the reference sources)")
    ref = load_reference()
    g = big
    tets = torch.from_numpy(g["tets"]).cuda()
    nbrs = torch.from_numpy(g["neighbors"]).cuda()
    r_ref = ref.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], 10.0)
    r_new = wtivo_gpupr.graph_cut_fast(g["vertices"], tets, nbrs, g["labels"], 10.0)
    capfd.readouterr()
    assert int(r_new[1]) == int(r_ref[1]) and int(r_new[2]) == int(r_ref[2])
    assert np.array_equal(np.asarray(r_new[0]), np.asarray(r_ref[0]))
    for i in (5, 6, 7, 8, 9, 15):
        assert int(r_new[i]) == int(r_ref[i]), i
