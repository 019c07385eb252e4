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

Usage:  python oracle/build.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DEFAULT = "/root/reference"
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


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REF_DEFAULT)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build_oracle(a.force))
    print(build_ref(a.reference, a.force))


if __name__ == "__main__":
    main()
