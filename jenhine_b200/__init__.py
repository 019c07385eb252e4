"""B200-native FDK cone-beam reconstruction engine.

The compute path lives in libjfdk.so (C ABI: include/jfdk.h; CUDA sources in
csrc/).  This package holds its Python binding (``fdk.FDKEngine``), the
synthetic workloads and the build recipe.
"""
from .fdk import FDKEngine, ReconConfig, ScanConfig  # noqa: F401

__all__ = ["FDKEngine", "ReconConfig", "ScanConfig"]
