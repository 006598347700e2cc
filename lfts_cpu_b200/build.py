"""Build the native parts of lfts_cpu_b200 in-tree.

* ``lfts_cpu_b200/liblfts_b200.so`` -- the CUDA kernels for sm_100a and the C ABI
  declared in ``include/lfts_b200.h`` (nvcc, cross-compiles without a GPU).
* ``lfts_cpu_b200/lfts-b200`` -- the drop-in driver program (host C++ above the
  C ABI), built when its sources are present.

Usage: ``python -m lfts_cpu_b200.build [--force] [-v]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
DRIVER = os.path.join(PKG, "driver")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "liblfts_b200.so")
EXE = os.path.join(PKG, "lfts-b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-I" + os.path.join(ROOT, "include")] + ARCH
CU_SOURCES = ["fft_fp64.cu", "fft_fp32.cu", "lfts_capi.cu", "lfts_noalloc.cu", "lfts_ensemble.cu"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build lfts_cpu_b200")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd[:4]) + " ...")
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile everything that is out of date; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in sorted(os.listdir(CSRC)) if h.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(ROOT, "include", "lfts_b200.h"))
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([nvcc] + NVFLAGS + ["-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    host = os.path.join(CSRC, "lfts_host.cc")
    host_o = os.path.join(BUILD, "lfts_host.o")
    if force or _newer(host_o, [host, os.path.join(ROOT, "include", "lfts_b200.h")]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-c", host, "-o", host_o], verbose)
        jobs.append(host_o)
    objs.append(host_o)
    if force or jobs or _newer(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], verbose)
    drv = os.path.join(DRIVER, "lfts_driver.cc")
    if os.path.exists(drv):
        dsrcs = [os.path.join(DRIVER, f) for f in sorted(os.listdir(DRIVER)) if f.endswith(".cc")]
        dhdrs = [os.path.join(DRIVER, f) for f in os.listdir(DRIVER) if f.endswith(".h")]
        if force or _newer(EXE, dsrcs + dhdrs + [LIB]):
            _run(["g++", "-O3", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-o", EXE] + dsrcs
                 + ["-L" + PKG, "-llfts_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
