"""Builds the prover's CUDA library in-tree: circlepacking_b200/_lib/libcp_b200.so.

All device code is compiled for sm_100a only (B200).  Usage:
    python -m circlepacking_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT_DIR = os.path.join(PKG, "_lib")
OBJ_DIR = os.path.join(PKG, "_build")
LIB = os.path.join(OUT_DIR, "libcp_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no implicit contraction anywhere; every fused multiply-add in the
# library is an explicit __fma_rn.
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2", "-I" + INCLUDE,
              "-I" + CSRC]


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, name))
    return out


def headers():
    hs = [os.path.join(CSRC, n) for n in os.listdir(CSRC) if n.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, n) for n in os.listdir(INCLUDE) if n.endswith(".h")]
    return hs


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    cmd = [NVCC, *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
    if verbose and src.endswith(".cu"):
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = sources()
    newest_header = max((os.path.getmtime(h) for h in headers()), default=0.0)
    todo = []
    for s in srcs:
        obj = os.path.join(OBJ_DIR, os.path.basename(s) + ".o")
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(s), newest_header):
            todo.append(s)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    objs = [os.path.join(OBJ_DIR, os.path.basename(s) + ".o") for s in srcs]
    if todo or force or not os.path.exists(LIB):
        # link to a temporary name and rename: a reader of the tree (a process
        # loading the library, a copy of the tree) sees the old or the new file,
        # never a partly written one
        tmp = LIB + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
