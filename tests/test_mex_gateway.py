"""The MATLAB/Octave MEX gateway (mex/ins2d_mex.cpp) compiles against the
documented MEX C API (declarations in tests/native/mex.h; MATLAB and Octave
are not installed here) and every C-ABI function it calls is declared in
include/ins2d.h and exported by libins2d.so."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_mex_gateway_compiles(tmp_path):
    obj = tmp_path / "ins2d_mex.o"
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", "-Wno-unused-function", "-fPIC", "-c",
           "-I", os.path.join(ROOT, "tests", "native"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "mex", "ins2d_mex.cpp"), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the gateway's entry point and its undefined references: MEX API + ins2d_*
    nm = subprocess.run(["nm", "-C", str(obj)], capture_output=True, text=True, check=True).stdout
    assert re.search(r"\bT mexFunction\b", nm)
    undefined = set(re.findall(r"^\s+U (\S+)$", nm, re.M))
    calls = {u for u in undefined if u.startswith("ins2d_")}
    assert {"ins2d_ctx_create", "ins2d_F", "ins2d_pressure_poisson", "ins2d_erk_step",
            "ins2d_conservation"} <= calls
    from ins2d_b200 import _lib
    assert calls <= set(_lib.EXPORTED)
