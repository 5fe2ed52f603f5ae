"""Build libsphgpu.so (sm_100a) in-tree with nvcc.

    python -m sph_swe_b200.build [--force] [--verbose]

The library is written next to this file so that it travels with the
repository; nothing is installed into site-packages.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libsphgpu.so")
CLI_SRC = os.path.join(HERE, "cli", "sh_example.cpp")
CLI = os.path.join(HERE, "sh_example")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "sph_swe", "*.hpp")))


def up_to_date() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return False
    t = min(os.path.getmtime(LIB), os.path.getmtime(CLI))
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [CLI_SRC, __file__])


def build_cli() -> str:
    """The sh_example driver, linked against the in-tree library (rpath $ORIGIN)."""
    cuda = os.path.dirname(os.path.dirname(nvcc()))
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
    tmp = CLI + ".tmp"
    cmd = [cxx, "-std=c++17", "-O2", "-I", INCLUDE, "-I", os.path.join(cuda, "include"), CLI_SRC, "-o", tmp,
           "-L", HERE, "-lsphgpu", "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN",
           "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    subprocess.run(cmd, check=True)
    os.replace(tmp, CLI)
    return CLI


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"] + list(extra or [])
    if verbose:
        common += ["-Xptxas", "-v"]
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = common + ["-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if out.strip() and (verbose or p.returncode):
            sys.stdout.write(out)
        if p.returncode:
            failed = True
            sys.stdout.write("FAILED: " + " ".join(cmd) + "\n")
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    build_cli()
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
