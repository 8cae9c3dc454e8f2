"""Builds libmarl_cuda.so in-tree for sm_100a with nvcc.

    python marl-ochre_b200/build.py [--force] [-v]

Each translation unit under csrc/ is compiled to an object under _build/
(rebuilt when it or a header is newer than the object), then linked into
marl-ochre_b200/libmarl_cuda.so.  The kernels that must reproduce the
reference's arithmetic bit-for-bit are compiled with -fmad=false (no fused
multiply-add contraction) and without fast-math.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmarl_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# Per-file extra flags (default: exact IEEE float semantics).
EXACT = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
FLAGS = {"mlp.cu": ["-prec-div=true", "-prec-sqrt=true", "-ftz=false"]}  # MLP: FMA contraction allowed


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(
        os.path.join(ROOT, "include", "*.h"))


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in headers())
    objs, cmds = [], []
    for src in sources():
        name = os.path.basename(src)
        obj = os.path.join(BUILD, name + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_header)
        if not stale:
            continue
        cmd = [nvcc(), "-ccbin", host_cxx(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr", *FLAGS.get(name, EXACT),
               "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c", src, "-o", obj]
        if ptxas_v and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        cmds.append(cmd)
    # Translation units compile independently: run them side by side.
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1) or 1) as ex:
        for r in ex.map(lambda c: subprocess.run(c, capture_output=ptxas_v), cmds):
            if ptxas_v:
                sys.stdout.write(r.stdout.decode() + r.stderr.decode())
            if r.returncode != 0:
                if not ptxas_v:
                    raise subprocess.CalledProcessError(r.returncode, r.args)
                raise subprocess.CalledProcessError(r.returncode, r.args, r.stdout, r.stderr)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), "-ccbin", host_cxx(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/shared-memory usage per kernel")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_v))
    sys.exit(0)
