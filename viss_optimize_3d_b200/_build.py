"""Build libviss.so (the sm_100a CUDA library behind include/viss.h) and the
drop-in host executables, in-tree, with nvcc.

    python -m viss_optimize_3d_b200._build [--force] [-v]

Every CUDA source is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); there is no other target.
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
HOST = os.path.join(PKG, "host")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build_obj")
LIB = os.path.join(PKG, "libviss.so")
BIN = os.path.join(PKG, "bin")

CU_SOURCES = ["healpix.cu", "geometry.cu", "visibility.cu", "dcf.cu", "capi.cu", "noalloc.cu",
              "days.cu", "formation.cu", "gridded.cu"]
HEADERS = ["viss_common.cuh", "visibility.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
                     "-I", CSRC, "--expt-relaxed-constexpr"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build_library(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "viss.h")]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-c", s, "-o", o]
            jobs.append(cmd)
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for out in ex.map(lambda c: _run(c, verbose), jobs):
                logs.append(out)
    if force or jobs or _newer(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lcufft", "-lrt", "-ldl",
                                                                 "-lpthread"], verbose)
    if ptxas_verbose:
        print("\n".join(logs))
    return LIB


HOST_PROGRAMS = {
    # executable name: (source, compile-time definitions)
    "pix2ang": ("pix2ang_main.cpp", []),
    "vissgen3d_blockage": ("vissgen_main.cpp", ["-DVISS_VARIANT_BLOCKAGE=1", "-DVISS_VARIANT_10M=0"]),
    "vissgen3d_blockage_10m": ("vissgen_main.cpp", ["-DVISS_VARIANT_BLOCKAGE=1", "-DVISS_VARIANT_10M=1"]),
    "vissgen3d_noblockage": ("vissgen_main.cpp", ["-DVISS_VARIANT_BLOCKAGE=0", "-DVISS_VARIANT_10M=0"]),
    "vissgen3d_noblockage_10m": ("vissgen_main.cpp", ["-DVISS_VARIANT_BLOCKAGE=0", "-DVISS_VARIANT_10M=1"]),
    # streaming day loop over binary day files (not a drop-in: new interface);
    # the per-GPU day sums are reduced with NCCL
    "vissgen_stream": ("vissgen_stream_main.cpp", [], ["-lnccl"]),
}


def build_host(force: bool = False, verbose: bool = False):
    """The drop-in executables: C++ host code over libviss.so."""
    if not os.path.isdir(HOST):
        return []
    os.makedirs(BIN, exist_ok=True)
    out = []
    common = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith((".h", ".hpp"))]
    for name, (src, defs, *libs) in HOST_PROGRAMS.items():
        s = os.path.join(HOST, src)
        if not os.path.exists(s):
            continue
        exe = os.path.join(BIN, name)
        if force or _newer(exe, [s, LIB, __file__] + common):
            cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-Wall", "-I", INCLUDE,
                   "-I", "/usr/local/cuda/include", *defs, s, "-o", exe, "-L", PKG, "-lviss",
                   f"-Wl,-rpath,$ORIGIN/..", "-L/usr/local/cuda/lib64", "-lcudart", "-lpthread",
                   *(libs[0] if libs else [])]
            _run(cmd, verbose)
        out.append(exe)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    lib = build_library(force=force, verbose=verbose)
    build_host(force=force, verbose=verbose)
    return lib


if __name__ == "__main__":
    force = "--force" in sys.argv
    verbose = "-v" in sys.argv
    if "--ptxas" in sys.argv:
        build_library(force=True, verbose=verbose, ptxas_verbose=True)
    else:
        print(build(force=force, verbose=verbose))
