"""Helpers shared by the GPU tests (checks computed with torch on the GPU)."""
from __future__ import annotations

import numpy as np
import torch


def cut_capacity(nbr, cap0, term0, part):
    """Capacity of the cut (S = part==0, T = part==1) in the ORIGINAL reduced
    graph: n-links S->T, sink t-links of S nodes, source t-links of T nodes.
    Equal to the flow value iff both are optimal (max-flow min-cut)."""
    nbr = nbr.long()
    p = part.long()
    valid = nbr >= 0
    pu = torch.where(valid, p[nbr.clamp_min(0)], torch.zeros_like(nbr))
    s_to_t = valid & (p[:, None] == 0) & (pu == 1)
    nl = (cap0.long() * s_to_t).sum()
    t0 = term0.long()
    sink = torch.where((p == 0) & (t0 < 0), -t0, torch.zeros_like(t0)).sum()
    src = torch.where((p == 1) & (t0 > 0), t0, torch.zeros_like(t0)).sum()
    return int((nl + sink + src).item())


def reverse_slots(nbr):
    n = nbr.shape[0]
    valid = nbr >= 0
    rows = nbr.long().clamp_min(0)
    back = nbr[rows]                                   # [n,4,4]
    me = torch.arange(n, device=nbr.device)[:, None, None]
    hit = back == me
    return torch.where(valid, hit.int().argmax(dim=2), torch.full_like(nbr, -1))


def residual_consistent(nbr, cap0, res):
    """res[e] + res[rev e] == cap[e] + cap[rev e] on every arc pair."""
    rv = reverse_slots(nbr)
    valid = nbr >= 0
    u = nbr.long().clamp_min(0)
    k = rv.long().clamp_min(0)
    r_back = res.long()[u, k]
    c_back = cap0.long()[u, k]
    lhs = res.long() + r_back
    rhs = cap0.long() + c_back
    return bool(torch.all(torch.where(valid, lhs == rhs, torch.ones_like(valid))).item())


def np_(t):
    return t.detach().cpu().numpy()
