"""Extracts the reference's logged per-step results into small fixtures.

Reads, from the reference checkout named by the INS2D_REFERENCE environment
variable (required; the script stops with an error when it is unset):
  results/LDC_unsteady_1.000e+02_20x20_0/convergence.txt
  results/shear_layer01/convergence.txt
and writes tests/golden/{ldc_re100_20x20,shear_layer_40x40}.json with the
columns n, dt, t, res, maxdiv, umom, vmom, k (process_iteration.m:112-120).

The run parameters are not recorded next to those logs; they were identified
by reproducing the logs with the oracle (see tests/test_oracle_pins.py):
  LDC 20x20: unit square, uniform, Re=100, lid u=1, RK33P2, dt=0.01, 100 steps
  shear layer 40x40: [0,2pi]^2 periodic, Re=1e100, RK44, dt=0.01, 400 steps,
  FFT Poisson, u = 1 + tanh-profile of testsuite/shear_layer/shear_layer_IC.m.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

LOGS = {
    "ldc_re100_20x20.json": "results/LDC_unsteady_1.000e+02_20x20_0/convergence.txt",
    "shear_layer_40x40.json": "results/shear_layer01/convergence.txt",
}


def parse(path):
    rows = []
    with open(path) as fh:
        for line in fh:
            s = line.split()
            if len(s) == 8 and s[0].isdigit():
                rows.append([float(v) for v in s])
    return rows


def main():
    REF = os.environ.get("INS2D_REFERENCE")
    if not REF or not os.path.isdir(REF):
        sys.exit("make_golden.py: set INS2D_REFERENCE to the reference checkout (the directory holding results/)")
    for out, rel in LOGS.items():
        rows = parse(os.path.join(REF, rel))
        with open(os.path.join(HERE, out), "w") as fh:
            json.dump({"source": rel, "columns": ["n", "dt", "t", "res", "maxdiv", "umom", "vmom", "k"],
                       "rows": rows}, fh)
        print(out, len(rows), file=sys.stderr)


if __name__ == "__main__":
    main()
