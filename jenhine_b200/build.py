"""Build libjfdk.so (the engine's C ABI + sm_100a kernels) in-tree.

    python -m jenhine_b200.build [--force] [--verbose]

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with line info; host sources are
compiled by nvcc's host compiler.  The library links the CUDA runtime
statically so it does not depend on which libcudart another module loaded.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
LIB = os.path.join(PKG, "libjfdk.so")
OBJ = os.path.join(PKG, "_obj")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]
CU_FLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]


HOST = os.path.join(PKG, "host")   # C++ Agent/Pipe layer over the C ABI


def sources():
    cs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp"))]
    hs = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp")]
    return sorted(cs) + sorted(hs)


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    jeng = os.path.join(INCLUDE, "jengine")
    return hs + inc + [os.path.join(jeng, f) for f in os.listdir(jeng) if f.endswith(".h")]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed ({r.returncode})")
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdr_time = max(os.path.getmtime(h) for h in headers())
    objs, relink = [], force or not os.path.exists(LIB)
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_time):
            continue
        flags = CU_FLAGS if src.endswith(".cu") else COMMON
        _run([NVCC] + flags + ["-c", src, "-o", obj], verbose)
        relink = True
    if relink or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run([NVCC, "-shared"] + ARCH + ["-o", LIB] + objs, verbose)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))


if __name__ == "__main__":
    main()
