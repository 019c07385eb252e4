"""The C-ABI library loads and exports every entry point include/jfdk.h
declares (no compute without a GPU)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "jfdk.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jfdk_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_stage_api():
    names = declared_functions()
    for n in ("jfdk_create", "jfdk_destroy", "jfdk_preprocess_frames", "jfdk_filter_frames",
              "jfdk_bp_accumulate", "jfdk_finalize", "jfdk_ctnum", "jfdk_reconstruct"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from jenhine_b200 import _lib, build
    build.build()
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the whole header
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_device_check_without_gpu_is_an_error_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from jenhine_b200 import _lib
    buf = ctypes.create_string_buffer(256)
    assert _lib.load().jfdk_device_check(buf, 256) == _lib.JFDK_ERR_NO_DEVICE


def test_create_rejects_bad_sizes_before_touching_the_device():
    from jenhine_b200 import fdk, _lib
    scan = fdk.ScanConfig(num_views=4, dso=500.0, dsd=800.0, num_dets_u=2, num_dets_v=8,
                          detector_pixel_size=0.5)
    recon = fdk.ReconConfig(8, 8, 8, 1.0, 1.0)
    with pytest.raises(_lib.JfdkError) as e:
        fdk.FDKEngine(scan, recon, [[0.0] * 12] * 4)
    assert e.value.status == _lib.JFDK_ERR_INVALID


def test_engine_fails_loudly_without_the_library(monkeypatch, tmp_path):
    from jenhine_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(ImportError):
        _lib.load()


def test_gather_rate_rejects_bad_arguments_before_touching_the_device():
    from jenhine_b200 import _lib
    lib = _lib.load()
    r = ctypes.c_double(-1.0)
    for args in ((12, 1, 6, 32), (16, 1, 0, 32), (16, 1, 33, 32), (8, 0, 4, 30), (8, 0, 4, 68)):
        assert lib.jfdk_measure_gather_rate(*args, ctypes.byref(r)) == _lib.JFDK_ERR_INVALID
    assert lib.jfdk_measure_gather_rate(16, 1, 6, 32, None) == _lib.JFDK_ERR_INVALID
