"""Build recipe for libxtb200.so (CUDA kernels + C ABI, sm_100a only) and the
``xtric`` command-line driver, in-tree.

    python xxtric_b200/build.py            # incremental
    python xxtric_b200/build.py --force    # rebuild everything

(Run it as a script: importing the package needs the library it builds.)

nvcc cross-compiles for sm_100a without a GPU. Objects go to _build/ at the
repository root (git-ignored); the library lands next to this file.
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
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libxtb200.so")
CLI = os.path.join(PKG, "xtric")

CUDA_SOURCES = ["csrc/capi.cu", "csrc/build.cu", "csrc/count.cu", "csrc/gen.cu", "csrc/rgg.cu",
                "csrc/vite.cu", "csrc/count_static.cu", "csrc/batch.cu", "csrc/serve.cu"]
HOST_SOURCES = ["host/host_io.cpp"]
CLI_SOURCES = ["host/xtric_main.cpp"]
HEADERS = ["csrc/xt_internal.cuh", "csrc/xt_rng.cuh", "../include/xtric.h", "host/xtric_host.hpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libxtb200.so")


def host_cxx() -> str:
    # the plain system compiler; some images point $CXX at a wrapper without libgomp
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    if r.stderr.strip() and os.environ.get("XT_BUILD_VERBOSE"):
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(PKG, h) for h in HEADERS]
    jobs = []
    objs = []
    for src in CUDA_SOURCES + HOST_SOURCES:
        s = os.path.join(PKG, src)
        o = os.path.join(BUILD, src.replace("/", "_") + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc()] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                                     "--expt-relaxed-constexpr", "-ccbin", host_cxx(), "-c", s, "-o", o]
            if verbose_ptxas and src.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(_run, jobs))
    if force or jobs or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        _run([nvcc()] + ARCH + ["-shared", "-ccbin", host_cxx(), "-o", tmp] + objs)
        os.replace(tmp, LIB)
    cli_src = [os.path.join(PKG, s) for s in CLI_SOURCES]
    if force or _stale(CLI, cli_src + hdrs + [LIB]):
        _run([host_cxx(), "-O2", "-std=c++17", "-o", CLI] + cli_src +
             ["-L" + PKG, "-lxtb200", "-Wl,-rpath,$ORIGIN"])
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas resource usage")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.ptxas))


if __name__ == "__main__":
    main()
