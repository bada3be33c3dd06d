"""Snapshot output of ensemble runs for reduced-order-model generation.

The reference keeps, per run, the velocity and pressure of every time step as
matrices ``uh_total`` (Nt x Nu), ``vh_total`` (Nt x Nv), ``p_total`` (Nt x Np)
(process_iteration.m:79-83, ``save_eco = 0``) or one file ``Vp_n=<n>.mat`` per
step (process_iteration.m:84-86, ``save_eco = 1``), and its ROM solver loads
``uh_total, vh_total, p_total, dt, t_end, Re, k, umom, vmom, maxdiv``
(solver_unsteady_ROM.m:13).  :class:`SnapshotRecorder` produces the same
matrices for every member of an :class:`~ins2d_b200.api.Ensemble` (every
``every`` steps, with the check_conservation time series) and writes them as
MATLAB files with those variable names, one per member, or as ``Vp_n=<n>.mat``
files per member and step.
"""
from __future__ import annotations

import os

import numpy as np


class SnapshotRecorder:
    """Records members' (V, p) and check_conservation values every ``every``
    steps of an ensemble run (the initial state counts as step 0)."""

    def __init__(self, ens, nsteps, every=1, members=None):
        self.ens = ens
        self.every = int(every)
        self.members = list(range(len(ens))) if members is None else list(members)
        self.nsnap = nsteps // self.every + 1
        self.rows = 0
        self.t = np.zeros(self.nsnap)
        self.data = {}
        for m in self.members:
            o = ens.member(m)
            self.data[m] = dict(uh_total=np.zeros((self.nsnap, o.Nu)), vh_total=np.zeros((self.nsnap, o.Nv)),
                                p_total=np.zeros((self.nsnap, o.Np)), k=np.zeros(self.nsnap),
                                umom=np.zeros(self.nsnap), vmom=np.zeros(self.nsnap), maxdiv=np.zeros(self.nsnap))
        self._V = {m: np.empty(ens.member(m).NV) for m in self.members}
        self._p = {m: np.empty(ens.member(m).Np) for m in self.members}

    def record(self, t):
        r = self.rows
        if r >= self.nsnap:
            raise IndexError("snapshot buffer full")
        self.t[r] = t
        for m in self.members:
            o = self.ens.member(m)
            V, p = self.ens.get_state(m, self._V[m], self._p[m])
            d = self.data[m]
            d["uh_total"][r] = V[:o.Nu]
            d["vh_total"][r] = V[o.Nu:]
            d["p_total"][r] = p
            maxdiv, umom, vmom, k = o.check_conservation(V, t)
            d["maxdiv"][r], d["umom"][r], d["vmom"][r], d["k"][r] = maxdiv, umom, vmom, k
        self.rows += 1

    def save(self, directory, dt, prefix="member", eco=False):
        """One MATLAB file per member with the ROM solver's variable names, or
        (eco) a ``snapshots`` directory per member with ``Vp_n=<n>.mat`` files."""
        from scipy.io import savemat
        os.makedirs(directory, exist_ok=True)
        paths = []
        n_rows = self.rows
        for m in self.members:
            o = self.ens.member(m)
            d = self.data[m]
            if eco:
                sub = os.path.join(directory, f"{prefix}{m}", "snapshots")
                os.makedirs(sub, exist_ok=True)
                for r in range(n_rows):
                    n = r * self.every
                    V = np.r_[d["uh_total"][r], d["vh_total"][r]][:, None]
                    savemat(os.path.join(sub, f"Vp_n={n}.mat"), dict(V=V, p=d["p_total"][r][:, None]))
                paths.append(sub)
                continue
            path = os.path.join(directory, f"{prefix}{m}.mat")
            savemat(path, dict(uh_total=d["uh_total"][:n_rows], vh_total=d["vh_total"][:n_rows],
                               p_total=d["p_total"][:n_rows], dt=float(dt) * self.every,
                               t_end=float(self.t[n_rows - 1]), Re=float(o.Re), k=d["k"][:n_rows, None],
                               umom=d["umom"][:n_rows, None], vmom=d["vmom"][:n_rows, None],
                               maxdiv=d["maxdiv"][:n_rows, None]))
            paths.append(path)
        return paths


def run_with_snapshots(ens, t0, dt, nsteps, every=1, members=None):
    """Advances the ensemble nsteps, recording snapshots every ``every``
    steps; returns the recorder and the per-member solver statistics."""
    rec = SnapshotRecorder(ens, nsteps, every, members)
    rec.record(t0)
    stats = None
    n = 0
    while n < nsteps:
        k = min(every, nsteps - n)
        st = ens.time_ERK(t0 + n * dt, dt, k)
        stats = st if stats is None else [
            dict(n_solves=a["n_solves"] + b["n_solves"], iters_total=a["iters_total"] + b["iters_total"],
                 iters_max=max(a["iters_max"], b["iters_max"]), norm1_max=max(a["norm1_max"], b["norm1_max"]))
            for a, b in zip(stats, st)]
        n += k
        if n % every == 0:
            rec.record(t0 + n * dt)
    return rec, stats
