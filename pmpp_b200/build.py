"""Build libpmb200.so in-tree with nvcc for sm_100a.

Usage: ``python -m pmpp_b200.build`` (or ``__graft_entry__.build()``).
The library is a plain C-ABI shared object (include/pmb200.h); it links cuFFT
from the CUDA toolkit and statically links the CUDA runtime.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpmb200.so")
SOURCES = ["cic.cu", "spectral.cu", "integrate.cu", "sort.cu", "ic.cu", "capi.cu", "cosmo.cpp", "noalloc.cu", "cic_general.cu", "mlp.cu", "ensemble.cu", "f64.cu", "pmfft.cu", "observe.cu", "meshcnn.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def cuda_home():
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found")


def needs_rebuild():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(os.path.dirname(HERE), "include", "pmb200.h")
    return os.path.exists(hdr) and os.path.getmtime(hdr) > t


def build(force=False, verbose=False, jobs=None):
    if not force and not needs_rebuild():
        return LIB
    home = cuda_home()
    nvcc = os.path.join(home, "bin", "nvcc")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
                     "-I", os.path.join(os.path.dirname(HERE), "include")]
    if verbose:
        common += ["-Xptxas", "-v"]
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        cmd = [nvcc, "-c", os.path.join(CSRC, src), "-o", obj] + common
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(" ".join(cmd) + "\n" + (out or ""))
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc compilation failed")
    tmp = LIB + ".tmp"
    link = [nvcc, "-shared", "-o", tmp] + objs + ARCH + [
        "-L", os.path.join(home, "lib64"), "-lcufft", "-Xlinker", "-rpath," + os.path.join(home, "lib64")
    ]
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(link) + "\n" + r.stdout)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
