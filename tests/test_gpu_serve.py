"""Serving loop: a result is the same alone and in the mix."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import cached_graph
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _pool():
    return [cached_graph("proxy", 0, 20_000), cached_graph("lattice", 2, 80_000),
            cached_graph("box", 4, 60_000), cached_graph("torus", 5, 60_000)]


def test_results_same_alone_and_in_the_mix(built):
    import gpupr_capi

    pool = _pool()
    want = [orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0) for g in pool]
    with gpupr_capi.Server() as sv:
        # alone: one request at a time
        for g, (lab, st) in zip(pool, want):
            rid = sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"])
            out, res = sv.wait(rid, timeout_s=120)
            assert np.array_equal(out, lab) and res["adjusted_flow"] == st["adjusted_flow"]
        # in the mix: submitted together from several threads, repeated
        ids = {}

        def client(k):
            for rep in range(3):
                g = pool[(k + rep) % len(pool)]
                ids[(k, rep)] = ((k + rep) % len(pool),
                                 sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"]))

        ts = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        sizes = []
        for (k, rep), (gi, rid) in ids.items():
            out, res = sv.wait(rid, timeout_s=120)
            lab, st = want[gi]
            assert np.array_equal(out, lab), (k, rep)
            assert res["adjusted_flow"] == st["adjusted_flow"] and res["status"] == 0
            assert res["latency_ms"] >= res["queue_ms"] >= 0
            sizes.append(res["batch_size"])
        assert max(sizes) > 1          # requests really were batched together


def test_oversized_request_refused(built):
    import gpupr_capi

    g = _pool()[0]
    with gpupr_capi.Server(hbm_budget_bytes=1 << 20) as sv:
        with pytest.raises(gpupr_capi.GpuprError):
            sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"])


def test_destroy_finishes_submitted_requests(built):
    import gpupr_capi

    pool = _pool()
    want = [orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0)[0] for g in pool]
    sv = gpupr_capi.Server()
    outs = []
    for g in pool:
        rid = sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"])
        outs.append(sv._held[rid][4])
    sv.close()                          # returns only after every request is cut
    for out, lab in zip(outs, want):
        assert np.array_equal(out[:len(lab)], lab)


def test_bad_request_does_not_fail_its_batch(built):
    """A request with a neighbor id outside its graph fails alone, with the
    reference's message; the requests batched with it get their cuts."""
    import gpupr_capi

    pool = _pool()
    want = [orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0) for g in pool]
    bad = dict(pool[1])
    bad["neighbors"] = pool[1]["neighbors"].copy()
    i = int(np.nonzero((bad["neighbors"] >= 0).all(1))[0][0])
    bad["neighbors"][i, 0] = len(pool[1]["tets"]) + 9
    with gpupr_capi.Server() as sv:
        # a slow first request lets the rest pile up into one batch
        big = cached_graph("lattice", 2, 80_000)
        first = sv.submit(big["vertices"], big["tets"], big["neighbors"], big["labels"])
        ids = [sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"]) for g in pool[:1]]
        bad_id = sv.submit(bad["vertices"], bad["tets"], bad["neighbors"], bad["labels"])
        ids += [sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"]) for g in pool[2:]]
        sv.wait(first, timeout_s=120)
        with pytest.raises(gpupr_capi.GpuprError, match="neighbor out of range"):
            sv.wait(bad_id, timeout_s=120)
        for rid, gi in zip(ids, [0, 2, 3]):
            out, res = sv.wait(rid, timeout_s=120)
            lab, st = want[gi]
            assert res["status"] == 0 and np.array_equal(out, lab)
            assert res["adjusted_flow"] == st["adjusted_flow"]


@pytest.mark.parametrize("split", [0, 100_000])
def test_lanes_give_exact_cuts(built, split):
    """Requests split by size into two lanes whose solves overlap (or one lane
    with split 0): every result equals its cut alone; a large request always
    takes the large lane, a small one the small lane unless it spilled to an
    idle large lane."""
    import gpupr_capi

    big = cached_graph("lattice", 3, 300_000)
    pool = _pool() + [big]
    want = [orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0) for g in pool]
    with gpupr_capi.Server(split_tets=split) as sv:
        ids = []
        for rep in range(3):
            for gi in (4, 0, 1, 2, 3):
                g = pool[gi]
                ids.append((gi, sv.submit(g["vertices"], g["tets"], g["neighbors"], g["labels"])))
        for gi, rid in ids:
            out, res = sv.wait(rid, timeout_s=120)
            lab, st = want[gi]
            assert res["status"] == 0 and np.array_equal(out, lab), gi
            assert res["adjusted_flow"] == st["adjusted_flow"]
            n = len(pool[gi]["tets"])
            if split and n >= split:
                assert res["lane"] == 1, (gi, n)
            else:
                assert res["lane"] in ((0, 1) if split else (0,)), (gi, n)


def test_small_requests_spill_to_an_idle_large_lane(built):
    """A burst of small requests: the first takes the small lane; the second,
    submitted while the first is still in flight and the large lane is idle,
    spills to the large lane; the third finds both lanes busy and stays on the
    small lane.  Every result equals its cut alone."""
    import gpupr_capi

    pool = _pool()
    want = [orc.graph_cut(g["vertices"], g["tets"], g["neighbors"], g["labels"], 10.0) for g in pool]
    with gpupr_capi.Server(split_tets=10_000_000) as sv:
        ids = [(gi, sv.submit(pool[gi]["vertices"], pool[gi]["tets"], pool[gi]["neighbors"],
                              pool[gi]["labels"])) for gi in (0, 1, 2, 3)]
        lanes = []
        for gi, rid in ids:
            out, res = sv.wait(rid, timeout_s=120)
            lab, st = want[gi]
            assert res["status"] == 0 and np.array_equal(out, lab), gi
            assert res["adjusted_flow"] == st["adjusted_flow"]
            lanes.append(res["lane"])
    assert lanes[:3] == [0, 1, 0], lanes
