"""Builds libins2d.so in-tree (ins2d_b200/libins2d.so) with nvcc for sm_100a.

The library is plain C-ABI (include/ins2d.h); it links the CUDA runtime
statically and nothing from PyTorch.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libins2d.so")
SOURCES = ["setup.cpp", "kernels.cu", "stencil.cu", "fft.cu", "pcg.cu", "mg_host.cpp", "mg.cu", "fdm_host.cpp", "fdm.cu", "ens_pcg.cu", "cnn.cu", "ctx.cu", "noalloc.cu", "slab.cu"]
HEADERS = ["setup.hpp", "device.cuh", "kernels.cuh", "reduce.cuh", "mg.cuh", "mg_host.hpp", "cnn.cuh", "fdm_host.hpp",
           "fdm_block.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "ins2d.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, out=None, defines=(), objdir=None):
    """Compiles the library (to `out`, default ins2d_b200/libins2d.so); extra
    -D definitions select launch-shape tunables."""
    target = out or LIB
    if not force and out is None and not _stale():
        return LIB
    objdir = objdir or os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC] + ARCH + common + ["-D" + d for d in defines] + ["-lineinfo", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = target + ".tmp"
    subprocess.check_call([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs)
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    print(build(force=True, verbose="-v" in sys.argv))
