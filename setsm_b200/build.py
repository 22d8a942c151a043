"""Builds the CUDA library in-tree: setsm_b200/lib/libsetsm_vll.so (sm_100a).

Plain nvcc invocations (no torch extension machinery): each .cu becomes an
object, then one shared library exporting the C ABI of include/setsm_vll.h and
the C++ VerticalLineLocus drop-in.  Files whose results must be bit-exact with
the reference's FP64 arithmetic are compiled with -fmad=false.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libsetsm_vll.so")
# the same library with the window kernel's phase counters compiled in
# (VLL_PHASE_CYCLES; bench.py --phase-cycles reads them)
LIB_PHASES = os.path.join(LIBDIR, "libsetsm_vll_phases.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC,
          "-I", os.path.join(ROOT, "include")]
SOURCES = {
    "vll_plain.cu": ["-fmad=false"],
    "vll_preprocess.cu": ["-fmad=false"],
    "vll_sgm.cu": ["-fmad=false"],
    "vll_ortho.cu": ["-fmad=false"],
    "vll_orthotin.cu": ["-fmad=false"],
    "vll_heightrange.cu": ["-fmad=false"],
    "vll_selectmps.cu": ["-fmad=false"],
    "vll_initvoxel.cu": ["-fmad=false"],
    "vll_tinblunder.cu": ["-fmad=false"],
    "vll_tin.cu": ["-fmad=false"],
    "vll_split.cu": [],
    "vll_capi.cu": [],
    "vll_shim.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    objs = []
    nv = nvcc()
    for src, extra in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nv, *ARCH, *COMMON, *extra, "-c", path, "-o", obj]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"nvcc failed on {src}")
            if ptxas_info or verbose:
                sys.stderr.write(r.stderr)
    if force or _stale(LIB, objs):
        cmd = [nv, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


def build_phase_cycles(verbose: bool = False, force: bool = False) -> str:
    """lib/libsetsm_vll_phases.so: the library with vll_split.cu compiled
    with -DVLL_PHASE_CYCLES (the other objects are the default build's)."""
    build(verbose=verbose, force=force)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    src = os.path.join(CSRC, "vll_split.cu")
    obj = os.path.join(BUILD, "vll_split_phases.o")
    nv = nvcc()
    if force or _stale(obj, [src] + headers):
        cmd = [nv, *ARCH, *COMMON, "-DVLL_PHASE_CYCLES", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed on vll_split.cu (phase counters)")
    objs = [obj if s_ == "vll_split.cu" else os.path.join(BUILD, s_.replace(".cu", ".o"))
            for s_ in SOURCES]
    if force or _stale(LIB_PHASES, objs):
        r = subprocess.run([nv, *ARCH, "-shared", "-o", LIB_PHASES, *objs, "-lcudart"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed (phase counters)")
    return LIB_PHASES


if __name__ == "__main__":
    if "--phase-cycles" in sys.argv:
        build_phase_cycles(verbose=True, force="-f" in sys.argv)
    else:
        build(verbose=True, ptxas_info="-v" in sys.argv, force="-f" in sys.argv)
