"""Builds the oracle's C restatements (oracle/cg_dic.c: cg.F's DIC-PCG;
oracle/erk_periodic.c: the periodic explicit RK step, OpenMP) into
oracle/_build/libins2d_oracle.so.  Test infrastructure only."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(force=False):
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    srcs = [os.path.join(HERE, "cg_dic.c"), os.path.join(HERE, "erk_periodic.c")]
    out = os.path.join(out_dir, "libins2d_oracle.so")
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out
    subprocess.check_call(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", out] + srcs + ["-lm"])
    return out


if __name__ == "__main__":
    print(build(force=True))
