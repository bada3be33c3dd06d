"""Ensemble workloads and their distribution over ranks.

An ensemble is a list of independent flows (members); each rank advances
its share of the members as one :class:`~ins2d_b200.api.Ensemble` (one launch
per phase over its members), so the data path needs no collective.  Members
are assigned by estimated cost, longest first (LPT), and only the per-member
statistics are gathered at the end.
"""
from __future__ import annotations

import numpy as np

from . import cases


def random_members(n, seed=4, sizes=(64, 96, 128, 192, 256), stretch=1.05, Re_range=(100.0, 5000.0),
                   U_range=(0.5, 1.5), CG_acc=1e-10, CG_maxit=20000, RK="RK44", precision="fp64",
                   precond="default"):
    """Cavity and channel flows on tanh-stretched grids with nx, ny drawn from
    ``sizes``, Re and the lid / inflow velocity drawn uniformly (seeded):
    the batching configuration of the benchmark.  Even members are lid-driven
    cavities on [0,1]^2, odd members channels on [0,4] x [-0.5,0.5] with a
    parabolic inflow and an outflow at p = 0.  ``precond``: the members'
    PCG preconditioner ('default': fast diagonalization in the batched
    ensemble solves, the same as single contexts of these sizes; 'mg')."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        nx, ny = (int(v) for v in rng.choice(sizes, 2))
        Re = float(rng.uniform(*Re_range))
        U = float(rng.uniform(*U_range))
        if m % 2 == 0:
            x = cases.tanh_grid(nx, 0.0, 1.0, stretch)
            y = cases.tanh_grid(ny, 0.0, 1.0, stretch)
            kw = dict(x=x, y=y, BC=cases.BC_CAVITY, Re=Re, uBC=cases.lid_uBC(U, 1.0))
        else:
            x = cases.tanh_grid(nx, 0.0, 4.0, stretch)
            y = cases.tanh_grid(ny, -0.5, 0.5, stretch)
            kw = dict(x=x, y=y, BC=cases.BC_CHANNEL, Re=Re,
                      uBC=cases.channel_uBC(lambda yy, U=U: U * (1.0 - 4.0 * np.asarray(yy) ** 2)))
        kw.update(poisson=4, CG_acc=CG_acc, CG_maxit=CG_maxit, RK=RK, precision=precision, precond=precond)
        kw["_U"] = U
        out.append(kw)
    return out


def stable_dt(kw, U, safety=0.8):
    """Explicit RK4 step limit of a member: the diffusive eigenvalue bound
    (4/Re)(1/hx^2 + 1/hy^2) against RK4's real-axis reach 2.78 plus the
    convective bound U(1/hx + 1/hy) against its imaginary-axis reach 2.83,
    with the smallest cell widths."""
    hx = np.min(np.diff(kw["x"]))
    hy = np.min(np.diff(kw["y"]))
    lam_d = 4.0 / kw["Re"] * (1.0 / hx ** 2 + 1.0 / hy ** 2)
    lam_c = U * (1.0 / hx + 1.0 / hy)
    return safety / (lam_d / 2.78 + lam_c / 2.83)


def member_cost(kw):
    """Estimated relative cost of a member: its pressure cells (the solver's
    iteration count is nearly grid-independent with the multigrid
    preconditioner)."""
    return (len(kw["x"]) - 1) * (len(kw["y"]) - 1)


def lpt_partition(costs, nranks):
    """Longest-processing-time assignment of members to ranks: members in
    decreasing cost, each to the currently least loaded rank (ties to the
    lower rank).  Deterministic, so every rank computes the same split."""
    order = sorted(range(len(costs)), key=lambda m: (-costs[m], m))
    load = [0.0] * nranks
    parts = [[] for _ in range(nranks)]
    for m in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(m)
        load[r] += costs[m]
    return [sorted(p) for p in parts]


def gather_stats(local, members_of_rank, n_total, group=None):
    """All ranks' per-member statistics in member order (a list of dicts),
    gathered over torch.distributed (any backend); local[i] belongs to
    members_of_rank[i]."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    bucket = [None] * world
    dist.all_gather_object(bucket, list(zip(members_of_rank, local)), group=group)
    out = [None] * n_total
    for part in bucket:
        for m, st in part:
            out[m] = st
    return out
