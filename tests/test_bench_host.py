"""Host-side pieces of the benchmark: the host-only turbulence field equals
the context-normalised one (the oracle's check_conservation for the
normalisation), and the reference arm reports the GPU arm's workload
configuration (grid, dt, cells) with the steps it was asked for."""
import json
import os
import subprocess
import sys

import numpy as np

from oracle import ins2d_ref as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_turbulence_ic_host_matches_oracle_energy():
    from types import SimpleNamespace
    from ins2d_b200 import cases
    N = 48
    x = cases.uniform_grid(N, 0.0, 1.0)
    o = R.make_options(x, x.copy(), cases.BC_PERIODIC, Re=2000.0, poisson=6)

    class Ctx(SimpleNamespace):
        def check_conservation(self, V, t):
            return R.check_conservation(V, t, o)

    ctx = Ctx(Nx=N, Ny=N, x=x, y=x.copy())
    V_ref = cases.decaying_turbulence_ic(ctx, k0=6.0, seed=7)
    V = cases.decaying_turbulence_ic_host(N, 1.0, k0=6.0, seed=7)
    assert np.max(np.abs(V - V_ref)) <= 1e-14 * np.max(np.abs(V_ref))
    assert abs(R.check_conservation(V, 0.0, o)[3] - 1.0) < 1e-14
    assert R.check_conservation(V, 0.0, o)[0] < 1e-12  # discretely divergence-free


def test_reference_arm_config():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "tg512",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["config"]["grid"] == [512, 512] and line["config"]["cells"] == 512 * 512
    assert line["config"]["dt"] == 1e-3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["cpu_model"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["value"] == cb["value"] > 0
