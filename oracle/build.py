"""Build recipe for the parity oracles (TEST INFRASTRUCTURE).

Two shared libraries:

* ``oracle/libjfdk_oracle.so`` -- the plain-C restatement in ``fdk_oracle.c``
  (always buildable: it has no dependency on the reference tree).
* ``oracle/_ref/libjref.so`` -- the reference's own Core classes compiled from
  the JEngine sources where they lie (read-only, never copied), with the
  project's scalar shims for Intel IPP / MKL (``ref_shims/``).  Only possible
  where the reference tree is present; the built ``.so`` is git-ignored but
  travels with the working tree.

The reference writes Windows include paths (``#include "..\\Common\\TypeDefs.h"``).
g++ takes such a header name literally, so this script writes one forwarding
header per distinct backslash include name into ``oracle/_ref/inc`` (a file
whose *name* is that literal string) and puts that directory on the quoted
include path.  Nothing from the reference is copied; the forwarders only hold
an ``#include`` of the real file.

A third library, ``baseline/_ref/libbpcuda_ref.so``, holds the reference's
GPU backprojector (``BPCUDAAgent/BPCUDACore.cu`` and ``BPCUDACore.cpp`` with
the ``CUDA/`` wrappers it uses), compiled unchanged for sm_100a, plus
``ref_gpu/bpcuda_driver.cpp``, which drives it the way BPCUDAAgent does.  It
is the GPU baseline bench.py times beside the engine; git-ignored, it travels
with the working tree like the others.

The reference tree is taken from ``--reference DIR``, else from
``$JFDK_REFERENCE_DIR``, else from the path it is mounted at in the build
container.

Usage:  python oracle/build.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DEFAULT = os.environ.get("JFDK_REFERENCE_DIR", "/root/reference")
REPO = os.path.dirname(HERE)
OUT_GPU = os.path.join(REPO, "baseline", "_ref")
GPU_SO = os.path.join(OUT_GPU, "libbpcuda_ref.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(NVCC))
OUT_REF = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(HERE, "libjfdk_oracle.so")
REF_SO = os.path.join(OUT_REF, "libjref.so")

# The hot-path Core classes (and their helpers) that run in the reference's
# CPU pipeline.  Everything IPP/MKL-backed is replaced by ref_shims/.
REF_SOURCES = [
    "PreProcessingAgent/PreProcessingCore.cpp",
    "PreProcessingAgent/GainCorr.cpp",
    "PreProcessingAgent/NLog.cpp",
    "PreProcessingAgent/BeamHardeningCorr.cpp",
    "FilterAgent/FilterCore.cpp",
    "FilterAgent/PreFilterWeightGenerator.cpp",
    "BPAgent/BPCore.cpp",
    "CompositeAgent/CompositeCore.cpp",
    "CTNumAgent/CTNumCore.cpp",
    "TransformMatrix/MatrixConvertor.cpp",
    "TransformMatrix/ProjectionMatrixModifier.cpp",
    "Common/Timer.cpp",
]
FORCE_INCLUDES = ["cmath", "cstring", "cstddef", "sstream", "algorithm", "stdexcept", "string"]
INC_RE = re.compile(r'^\s*#\s*include\s*"([^"]+)"', re.M)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"compile failed: {cmd[0]} (exit {r.returncode})")


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "fdk_oracle.c")
    if (not force and os.path.exists(ORACLE_SO)
            and os.path.getmtime(ORACLE_SO) >= os.path.getmtime(src)
            and os.path.getmtime(ORACLE_SO) >= os.path.getmtime(os.path.join(HERE, "fdk_oracle.h"))):
        return ORACLE_SO
    _run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", "-D_GNU_SOURCE",
          src, "-o", ORACLE_SO, "-lm", "-lpthread"])
    return ORACLE_SO


def _write_forwarders(ref: str, inc_dir: str) -> None:
    """Scan the compiled sources and the headers they reach; for every quoted
    include containing a backslash, write a forwarder named by that string."""
    os.makedirs(inc_dir, exist_ok=True)
    seen, todo, fwd = set(), [os.path.join(ref, s) for s in REF_SOURCES], {}
    while todo:
        path = os.path.normpath(todo.pop())
        if path in seen or not os.path.exists(path):
            continue
        seen.add(path)
        with open(path, encoding="utf-8", errors="replace") as f:
            text = f.read()
        for name in INC_RE.findall(text):
            rel = name.replace("\\\\", "/").replace("\\", "/")
            target = os.path.normpath(os.path.join(os.path.dirname(path), rel))
            if "\\" in name:
                prev = fwd.get(name)
                if prev is not None and prev != target:
                    raise RuntimeError(f"include {name!r} resolves to two files")
                fwd[name] = target
            todo.append(target)
    for name, target in fwd.items():
        with open(os.path.join(inc_dir, name), "w") as f:
            f.write(f'#include "{target}"\n')


def build_ref(ref: str = REF_DEFAULT, force: bool = False) -> str | None:
    """Compile the reference Cores + shims + driver.  Returns the .so path, or
    None when the reference tree is absent (then any earlier build is kept)."""
    if not os.path.isdir(ref):
        return REF_SO if os.path.exists(REF_SO) else None
    shim_dir = os.path.join(HERE, "ref_shims")
    deps = [os.path.join(ref, s) for s in REF_SOURCES] + [
        os.path.join(shim_dir, f) for f in os.listdir(shim_dir)] + [
        os.path.join(HERE, "fdk_oracle.c"), os.path.join(HERE, "fdk_oracle.h")]
    if (not force and os.path.exists(REF_SO)
            and all(os.path.getmtime(REF_SO) >= os.path.getmtime(d) for d in deps)):
        return REF_SO
    inc_dir = os.path.join(OUT_REF, "inc")
    obj_dir = os.path.join(OUT_REF, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    _write_forwarders(ref, inc_dir)
    common = ["-O2", "-fPIC", "-ffp-contract=off", "-w"]
    cxx = ["g++", "-std=c++17"] + common + ["-iquote", inc_dir, "-I", ref]
    for h in FORCE_INCLUDES:
        cxx += ["-include", h]
    objs = []
    for s in REF_SOURCES:
        o = os.path.join(obj_dir, s.replace("/", "_") + ".o")
        _run(cxx + ["-c", os.path.join(ref, s), "-o", o])
        objs.append(o)
    for s in sorted(os.listdir(shim_dir)):
        if s.endswith(".cpp"):
            o = os.path.join(obj_dir, "shim_" + s + ".o")
            _run(cxx + ["-c", os.path.join(shim_dir, s), "-o", o])
            objs.append(o)
    o = os.path.join(obj_dir, "fdk_oracle.o")
    _run(["gcc", "-std=c11", "-D_GNU_SOURCE"] + common + ["-c", os.path.join(HERE, "fdk_oracle.c"), "-o", o])
    objs.append(o)
    _run(["g++", "-shared", "-o", REF_SO] + objs + ["-lpthread", "-lm"])
    return REF_SO


# The reference's GPU backprojector and the CUDA wrappers it uses.
# CUDA/Tex2DFloat.cpp specialises Tex2D<float>'s members without `template<>`
# (accepted by MSVC, rejected by g++); ref_gpu/tex2d_shim.cpp restates it.
GPU_CU = ["BPCUDAAgent/BPCUDACore.cu"]
GPU_CPP = ["BPCUDAAgent/BPCUDACore.cpp", "CUDA/DeviceMemory.cpp", "CUDA/ErrorChecking.cpp"]


def build_ref_gpu(ref: str = REF_DEFAULT, force: bool = False) -> str | None:
    """Compile the reference's BPCUDACore (unchanged, sm_100a) + the scalar
    shims + the driver into baseline/_ref/libbpcuda_ref.so.  Returns the .so
    path, or None when the reference tree is absent (an earlier build is
    kept)."""
    if not os.path.isdir(ref):
        return GPU_SO if os.path.exists(GPU_SO) else None
    shim = os.path.join(HERE, "ref_shims", "ipp_mkl_shims.cpp")
    drv = os.path.join(HERE, "ref_gpu", "bpcuda_driver.cpp")
    tex = os.path.join(HERE, "ref_gpu", "tex2d_shim.cpp")
    deps = [os.path.join(ref, s) for s in GPU_CU + GPU_CPP] + [shim, drv, tex, os.path.join(HERE, "fdk_oracle.c")]
    if (not force and os.path.exists(GPU_SO)
            and all(os.path.getmtime(GPU_SO) >= os.path.getmtime(d) for d in deps)):
        return GPU_SO
    if not os.path.exists(os.path.join(OUT_REF, "inc")):
        build_ref(ref)   # writes the forwarding headers the shims include
    obj_dir = os.path.join(OUT_GPU, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    inc = ["-I", ref, "-I", os.path.join(CUDA_HOME, "include")]
    force_inc = []
    for h in FORCE_INCLUDES:
        force_inc += ["-include", h]
    cxx = ["g++", "-std=c++17", "-O2", "-fPIC", "-w"] + inc + force_inc
    objs = []
    for s in GPU_CU:
        o = os.path.join(obj_dir, s.replace("/", "_") + ".o")
        _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-w", "-Xcompiler", "-fPIC"]
             + inc + force_inc + ["-c", os.path.join(ref, s), "-o", o])
        objs.append(o)
    for s in GPU_CPP:
        o = os.path.join(obj_dir, s.replace("/", "_") + ".o")
        # DeviceMemory.cpp instantiates DeviceMemory<float> only through a
        # sample function; without inlining the members are emitted out of line
        extra = ["-fno-inline"] if s.endswith("DeviceMemory.cpp") else []
        _run(cxx + extra + ["-c", os.path.join(ref, s), "-o", o])
        objs.append(o)
    for src, name in ((shim, "shim.o"), (drv, "driver.o"), (tex, "tex2d.o")):
        o = os.path.join(obj_dir, name)
        _run(cxx + ["-iquote", os.path.join(OUT_REF, "inc"), "-I", HERE, "-c", src, "-o", o])
        objs.append(o)
    o = os.path.join(obj_dir, "fdk_oracle.o")
    _run(["gcc", "-std=c11", "-D_GNU_SOURCE", "-O2", "-fPIC", "-ffp-contract=off", "-w", "-c",
          os.path.join(HERE, "fdk_oracle.c"), "-o", o])
    objs.append(o)
    _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", GPU_SO] + objs +
         ["-lpthread", "-lm"])
    return GPU_SO


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REF_DEFAULT)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build_oracle(a.force))
    print(build_ref(a.reference, a.force))
    print(build_ref_gpu(a.reference, a.force))


if __name__ == "__main__":
    main()
