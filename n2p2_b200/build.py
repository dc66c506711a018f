"""Builds the in-tree CUDA library n2p2_b200/libn2p2b200.so for sm_100a.

    python -m n2p2_b200.build          # or: python n2p2_b200/build.py

Every .cu / .cpp file of n2p2_b200/csrc is compiled separately (in parallel)
with nvcc for `-gencode arch=compute_100a,code=sm_100a`, then linked into one
shared library that exports the C-ABI of include/n2p2_b200.h.  Host code is
compiled with -ffp-contract=off so that host-side geometry (inverse box,
periodic image counts, scaling factors) rounds exactly as the reference's
ISO C++ build does.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libn2p2b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags() -> list[str]:
    return ARCH + [
        "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
        "-ccbin", "g++",
        "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
    ]


def _sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def _needs_build(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                    if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "n2p2_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not _needs_build(src, obj):
        return obj
    cmd = [_nvcc()] + _flags() + extra + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd += ["-x", "c++"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    if (not os.path.exists(LIB)
            or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_apps()
    if verbose:
        print(LIB)
    return LIB


APPS = {"nnp-predict": "nnp_predict.cpp", "lammps-emulate": "lammps_emulate.cpp"}


def build_apps() -> list[str]:
    """The command-line programs (n2p2_b200/bin/): host C++ over the C-ABI,
    linked against the in-tree library (rpath $ORIGIN/..)."""
    out_dir = os.path.join(PKG, "bin")
    os.makedirs(out_dir, exist_ok=True)
    out = []
    for name, src in APPS.items():
        srcp = os.path.join(PKG, "apps", src)
        exe = os.path.join(out_dir, name)
        deps = [srcp, LIB, os.path.join(ROOT, "include", "n2p2_b200.h"),
                os.path.join(ROOT, "include", "n2p2_b200.hpp")]
        if (not os.path.exists(exe)
                or any(os.path.getmtime(d) > os.path.getmtime(exe)
                       for d in deps)):
            cmd = ["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT,
                                                                  "include"),
                   srcp, "-L" + PKG, "-ln2p2b200",
                   "-Wl,-rpath,$ORIGIN/..", "-o", exe]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"g++ failed for {src}:\n{r.stderr}")
        out.append(exe)
    return out


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
