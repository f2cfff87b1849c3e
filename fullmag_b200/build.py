"""Build recipe for libfullmag_fdm.so.0 (sm_100a), in-tree.

The library is compiled with nvcc straight from fullmag_b200/csrc into
fullmag_b200/lib/, so the built object travels with the source tree.  The
exported symbols are exactly those of include/fullmag_fdm.h and
include/fullmag_fdm_ext.h.
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
SONAME = "libfullmag_fdm.so.0"
LIB = os.path.join(LIBDIR, SONAME)

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return [os.path.join(CSRC, f) for f in cu + cpp]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    env = dict(os.environ)
    # nvcc must use the system host compiler
    host_cxx = shutil.which("g++", path="/usr/bin") or "g++"
    cmds = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmds.append([nvcc(), *NVCC_FLAGS, "-ccbin", host_cxx, "-I", os.path.join(ROOT, "include"),
                     "-I", CSRC, "-c", src, "-o", obj])
        objs.append(obj)
    # translation units compile concurrently; any failure stops the build
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, env=env)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", host_cxx,
           "-Xlinker", f"-soname,{SONAME}", "-o", tmp, *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, env=env)
    os.replace(tmp, LIB)
    link = os.path.join(LIBDIR, "libfullmag_fdm.so")
    if os.path.islink(link) or os.path.exists(link):
        os.remove(link)
    os.symlink(SONAME, link)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
