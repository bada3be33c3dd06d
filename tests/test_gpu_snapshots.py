"""Snapshot output of ensemble runs (ins2d_b200/snapshots.py): the recorded
uh_total / vh_total / p_total rows equal each member's own single-context
states at the recorded steps, and the files carry the variable names the
reference's ROM solver loads (solver_unsteady_ROM.m:13)."""
import os

import numpy as np
import pytest

from tests.test_gpu_ensemble import _members

pytestmark = pytest.mark.gpu


def test_snapshots_match_single_runs(tmp_path):
    import scipy.io
    import ins2d_b200
    from ins2d_b200 import snapshots
    members = _members(7, 3, [24, 32, 48])
    ens = ins2d_b200.Ensemble(members)
    starts = []
    for m, kw in enumerate(members):
        o = ins2d_b200.Options(**kw)
        V0 = np.zeros(o.NV)
        p0 = o.pressure_additional_solve(V0, np.zeros(o.Np), 0.0)
        ens.set_state(m, V0, p0)
        starts.append((o, V0, p0))
    dt = 2e-3
    rec, stats = snapshots.run_with_snapshots(ens, 0.0, dt, 4, every=2)
    assert rec.rows == 3 and all(s["n_solves"] == 16 for s in stats)
    for m, (o, V0, p0) in enumerate(starts):
        V, p = V0.copy(), p0.copy()
        for r in range(3):
            if r > 0:
                V, p = o.time_ERK(V, p, (r - 1) * 2 * dt, dt, nsteps=2)
            d = rec.data[m]
            scale = max(np.max(np.abs(V)), 1e-30)
            assert np.max(np.abs(np.r_[d["uh_total"][r], d["vh_total"][r]] - V)) <= 1e-10 * scale
            assert np.max(np.abs(d["p_total"][r] - p)) <= 1e-8 * max(np.max(np.abs(p)), 1e-30)
            assert abs(d["k"][r] - o.check_conservation(V, r * 2 * dt)[3]) <= 1e-10 * max(d["k"][r], 1e-30)
    paths = rec.save(str(tmp_path), dt)
    f = scipy.io.loadmat(paths[1])
    for name in ("uh_total", "vh_total", "p_total", "dt", "t_end", "Re", "k", "umom", "vmom", "maxdiv"):
        assert name in f
    assert f["uh_total"].shape == (3, ens.member(1).Nu)
    eco = rec.save(str(tmp_path / "eco"), dt, eco=True)
    assert os.path.exists(os.path.join(eco[0], "Vp_n=4.mat"))
    g = scipy.io.loadmat(os.path.join(eco[0], "Vp_n=4.mat"))
    assert g["V"].shape == (ens.member(0).NV, 1)
