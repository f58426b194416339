"""Build the sm_100a CUDA library ``liblepic_gpu.so`` in-tree with nvcc.

Every translation unit is compiled for ``arch=compute_100a,code=sm_100a``
with ``--fmad=false`` (the FP64 kernels must round exactly like the
strict-IEEE oracle) and linked with the static CUDA runtime.  The library
lands next to this file so it travels with the source tree.

    python -m essaitemporaire_lepic_module_b200.build [--force] [-v]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblepic_gpu.so")
SOURCES = ["context.cu", "timing.cu", "fields.cu", "mg.cu", "particles.cu", "step.cu", "mcc.cu", "mixed.cu", "mgmixed.cu",
           "adjoint.cu", "residency.cu", "heating.cu", "injection.cu", "capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=default", "--expt-relaxed-constexpr"]
# The FP64 kernels keep the reference's operation order bit for bit, so no
# multiply-add contraction; the mixed-precision kernels have no bit-parity
# contract and use fused multiply-adds.
FMAD = {"mixed.cu": "--fmad=true", "mgmixed.cu": "--fmad=true"}


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liblepic_gpu.so")
    return exe


def _deps():
    inc = os.path.join(os.path.dirname(HERE), "include", "lepic_gpu.h")
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")] + [inc]
    return max(os.path.getmtime(h) for h in hdrs)


def build(force=False, verbose=False):
    """Compile (if stale) and return the path of liblepic_gpu.so."""
    os.makedirs(BUILD, exist_ok=True)
    exe = nvcc()
    hdr_t = _deps()
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        cmd = [exe, *ARCH, *FLAGS, FMAD.get(src, "--fmad=false"), "-c", s, "-o", o]
        # an object is stale when its source, a header or its flags changed
        stamp = o + ".cmd"
        same = os.path.exists(stamp) and open(stamp).read() == " ".join(cmd)
        if force or not same or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {cmd[-3]}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr)
        return r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    for cmd in jobs:
        with open(cmd[-1] + ".cmd", "w") as f:
            f.write(" ".join(cmd))
    if jobs or force or not os.path.exists(LIB):
        run([exe, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    return LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
