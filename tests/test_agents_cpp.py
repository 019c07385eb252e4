"""The C++ Agent/Pipe layer (include/jengine, jenhine_b200/host).

CPU: the runtime (pipes, tokens, agent bases) compiled on its own and run as a
native test program.  GPU: the reference's agent chain on libjfdk.so, two
identical scans back to back, against the reference cores' HU volume."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_l2

CPP = os.path.join(ROOT, "tests", "cpp")


def _build(out, sources, extra=()):
    cmd = ["g++", "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "include")] + sources + ["-o", out]
    cmd += list(extra)
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_pipeline_runtime_cpu(tmp_path):
    exe = str(tmp_path / "test_pipeline")
    host = os.path.join(ROOT, "jenhine_b200", "host")
    _build(exe, [os.path.join(CPP, "test_pipeline.cpp"), os.path.join(host, "Pipe.cpp"),
                 os.path.join(host, "Agent.cpp")])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout


def test_file_format_agents_cpu(tmp_path):
    """InputAgent / OutputAgent / ReadPTMFile (include/jengine/IO.h) on files
    the test program writes and reads back."""
    exe = str(tmp_path / "test_io")
    host = os.path.join(ROOT, "jenhine_b200", "host")
    _build(exe, [os.path.join(CPP, "test_io.cpp"), os.path.join(host, "Pipe.cpp"), os.path.join(host, "Agent.cpp"),
                 os.path.join(host, "IO.cpp")])
    r = subprocess.run([exe, str(tmp_path / "files")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout


def test_recon_parts_retry_cpu(tmp_path):
    """z-part plans and the retry on "CUDA failed to malloc " (include/jengine/ReconParts.h)."""
    exe = str(tmp_path / "test_recon_parts")
    host = os.path.join(ROOT, "jenhine_b200", "host")
    _build(exe, [os.path.join(CPP, "test_recon_parts.cpp"), os.path.join(host, "Pipe.cpp"),
                 os.path.join(host, "Agent.cpp"), os.path.join(host, "ReconParts.cpp")])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout


def test_cmake_build_cpu(tmp_path):
    """The CMake build (CMakeLists.txt) compiles libjfdk.so for sm_100a and the
    C++ test programs; the CPU ones run."""
    import shutil
    cmake = shutil.which("cmake")
    if cmake is None or shutil.which("ninja") is None:
        pytest.skip("cmake / ninja not installed")
    b = str(tmp_path / "build")
    r = subprocess.run([cmake, "-S", ROOT, "-B", b, "-G", "Ninja", "-DCMAKE_CUDA_COMPILER=/usr/local/cuda/bin/nvcc"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    r = subprocess.run([cmake, "--build", b, "-j", "16"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert os.path.exists(os.path.join(b, "libjfdk.so"))
    for t in ("test_pipeline", "test_recon_parts"):
        r = subprocess.run([os.path.join(b, t)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0 and "OK (0 failures)" in r.stdout, r.stdout + r.stderr
    r = subprocess.run([os.path.join(b, "test_io"), str(tmp_path / "io")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "OK (0 failures)" in r.stdout, r.stdout + r.stderr


def _write_case(path, g):
    raw = g["raw"]
    V, H, U = raw.shape
    X, Y, Z = (int(v) for v in g["vol"])
    comp = int(g["det_right"]) if "det_right" in g else -1
    hdr = np.array([V, U, H, X, Y, Z, comp], np.int32)
    adj_p, adj_l = g["adj_pts"].astype(np.float32), g["adj_db"].astype(np.float32)
    prm = np.array([g["dso"], g["hsr"], g["bright_field"], *g["bhc"], *g["pitch"], *g["norm"], *g["cut"],
                    adj_p.size], np.float32)
    with open(path, "wb") as f:
        for a in (hdr, prm, adj_p, adj_l, g["ptms"].astype(np.float32), raw.astype(np.uint16)):
            f.write(np.ascontiguousarray(a).tobytes())


def _write_files(folder, g):
    """The application's input files: Proj_%d.prj (uint16 frame, no header)
    per view and PTM.dat (12 numbers per view, written with enough digits to
    read back the same float32)."""
    os.makedirs(folder, exist_ok=True)
    for v, frame in enumerate(g["raw"].astype(np.uint16)):
        frame.tofile(os.path.join(folder, f"Proj_{v}.prj"))
    with open(os.path.join(folder, "PTM.dat"), "w") as f:
        for p in g["ptms"].astype(np.float32).reshape(-1, 12):
            f.write(" ".join("%.9g" % x for x in p) + "\n")


@pytest.mark.gpu
@pytest.mark.parametrize("files", [False, True], ids=["pipes", "files"])
@pytest.mark.parametrize("name", ["mini_c1", "mini_c2", "mini_comp", "mini_odd", "mini_tilt"])
def test_agent_chain_gpu(tmp_path, name, files):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from jenhine_b200 import build
    lib = build.build()
    exe = str(tmp_path / "test_agents_gpu")
    _build(exe, [os.path.join(CPP, "test_agents_gpu.cpp")],
           ["-L", os.path.dirname(lib), "-ljfdk", f"-Wl,-rpath,{os.path.dirname(lib)}"])
    g = load_golden(name)
    case, out = str(tmp_path / "case.bin"), str(tmp_path / "out.bin")
    _write_case(case, g)
    args = [exe, case, out]
    if files:
        folder = str(tmp_path / "scan")
        _write_files(folder, g)
        args.append(folder)
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    X, Y, Z = (int(v) for v in g["vol"])
    hu = np.fromfile(out, np.float32).reshape(Z, Y, X)
    assert rel_l2(hu + 1000.0, g["hu"] + 1000.0) <= 1e-5
    assert np.max(np.abs(hu - g["hu"])) < 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("parts", ["3", "retry"])
@pytest.mark.parametrize("name", ["mini_c1", "mini_comp"])
def test_agent_chain_zparts_gpu(tmp_path, name, parts):
    """The volume in z-parts (BPCUDAAgent numReconParts / numSlicesPerRecon):
    3 parts given, or found by the application's retry loop under a
    device-memory budget that only 3 or more parts fit."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from jenhine_b200 import build
    lib = build.build()
    exe = str(tmp_path / "test_agents_gpu")
    _build(exe, [os.path.join(CPP, "test_agents_gpu.cpp")],
           ["-L", os.path.dirname(lib), "-ljfdk", f"-Wl,-rpath,{os.path.dirname(lib)}"])
    g = load_golden(name)
    case, out = str(tmp_path / "case.bin"), str(tmp_path / "out.bin")
    _write_case(case, g)
    r = subprocess.run([exe, case, out, "-", parts], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    X, Y, Z = (int(v) for v in g["vol"])
    assert f"plan: 3 parts of {(Z + 2) // 3} slices" in r.stdout, r.stdout
    hu = np.fromfile(out, np.float32).reshape(Z, Y, X)
    assert rel_l2(hu + 1000.0, g["hu"] + 1000.0) <= 1e-5
    assert np.max(np.abs(hu - g["hu"])) < 0.5
