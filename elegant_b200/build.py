"""Build the engine's shared library in-tree with nvcc for sm_100a.

The output, ``elegant_b200/libelegant_b200.so``, exports the C ABI declared in
``include/elegant_b200.h``.  It is built next to the sources (not in a JIT
cache) so the built file travels with the repository snapshot.

Usage: ``python -m elegant_b200.build`` (or ``build()`` from Python).
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libelegant_b200.so")
BUILD_DIR = os.path.join(ROOT, "_build")

SOURCES = ["b2e_ring.cu", "b2e_csr.cu", "b2e_lattice.cu", "b2e_capi.cu", "b2e_tmap.cu", "b2e_wakenet.cu",
           "b2e_naff.cu"]
HEADERS = ["b2e_engine.h", "b2e_elements.cuh", "b2e_math.h", "b2e_kernels.h", "b2e_lattice.h",
           "b2e_csr.h", "b2e_sg.h", "b2e_umma.cuh", "b2e_tmap.h"]

# --fmad=false: no implicit multiply-add contraction, so every product and sum
# rounds exactly where the reference's C expression rounds; the explicit fma()
# calls inside b2e_math.h are unaffected.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "--fmad=false",
              "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build elegant_b200")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every CUDA source for sm_100a and link the shared library."""
    nvcc = nvcc_path()
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "elegant_b200.h")]
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd))
            jobs.append(cmd)
    # translation units compile independently
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=not verbose, text=True), jobs)):
            if r.returncode != 0:
                sys.stderr.write((r.stdout or "") + (r.stderr or ""))
                raise subprocess.CalledProcessError(r.returncode, r.args)
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
