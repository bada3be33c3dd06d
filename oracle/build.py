"""Builds the oracle's C restatement (oracle/cg_dic.c) into
oracle/_build/libins2d_oracle.so.  Test infrastructure only."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(force=False):
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    src = os.path.join(HERE, "cg_dic.c")
    out = os.path.join(out_dir, "libins2d_oracle.so")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", out, src, "-lm"])
    return out


if __name__ == "__main__":
    print(build(force=True))
