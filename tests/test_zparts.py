"""Backprojection of a volume in z-parts through the C ABI (jfdk_bp_set_slab)
and the device-memory bound (JFDK_OPT_DEVICE_MEMORY_LIMIT): each part's
slices equal the whole volume's bit for bit in the FP32 form (the per-voxel
arithmetic does not depend on the slab); an allocation past the bound fails
like cudaMalloc, with the message prefix JEngine's retry loop matches."""
import numpy as np
import pytest

from conftest import load_golden
from test_gpu_parity import engine_for, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def accumulate(e, filt, chunk=7):
    for v0 in range(0, filt.shape[0], chunk):
        e.bp_accumulate(filt[v0:v0 + chunk].contiguous(), v0)


@pytest.mark.parametrize("name", ["mini_c1", "mini_c2", "mini_odd", "mini_tilt"])
def test_parts_equal_whole_volume(torch_cuda, name):
    torch = torch_cuda
    g = load_golden(name)
    e = engine_for(g)
    filt = to_dev(torch, g["filt"])
    Z = int(g["vol"][2])
    e.bp_reset()
    accumulate(e, filt)
    whole = e.finalize(apply_ctnum=True).clone()
    parts = 3
    S = (Z - 1) // parts + 1
    for p in range(parts):
        z0, nz = p * S, min(S, Z - p * S)
        e.bp_set_slab(z0, nz)
        e.bp_reset()
        accumulate(e, filt)
        got = e.finalize(apply_ctnum=True, z0=z0, nz=nz)
        torch.cuda.synchronize()
        assert torch.equal(torch.nan_to_num(got, 1e30), torch.nan_to_num(whole[z0:z0 + nz], 1e30)), (p, z0, nz)


def test_parts_mixed_form_close(torch_cuda):
    """The mixed form steps u, v from each thread's first slice, so a slab
    that starts elsewhere moves sample points by rounding (and can flip an
    in-range decision at the detector edge): within 1e-4 of the whole
    volume, half the form's bar against FP64 on these fixtures."""
    torch = torch_cuda
    g = load_golden("mini_c2")
    e = engine_for(g, precision="mixed")
    filt = to_dev(torch, g["filt"])
    e.bp_reset()
    accumulate(e, filt)
    whole = e.finalize(apply_ctnum=False).clone()
    e.bp_set_slab(5, 19)
    e.bp_reset()
    accumulate(e, filt)
    got = e.finalize(apply_ctnum=False, z0=5, nz=19)
    ref = whole[5:24]
    ok = torch.isfinite(ref)
    err = ((got[ok] - ref[ok]).norm() / ref[ok].norm()).item()
    assert err <= 1e-4, err


def test_slab_bounds_and_state(torch_cuda):
    from jenhine_b200 import _lib
    g = load_golden("mini_c1")
    e = engine_for(g)
    Z = int(g["vol"][2])
    for z0, nz in ((-1, 4), (0, 0), (Z - 3, 4)):
        with pytest.raises(_lib.JfdkError) as ei:
            e.bp_set_slab(z0, nz)
        assert ei.value.status == _lib.JFDK_ERR_INVALID
    e.bp_set_slab(8, 8)
    e.bp_reset()
    e.bp_accumulate(to_dev(torch_cuda, g["filt"][:4]).contiguous(), 0)
    with pytest.raises(_lib.JfdkError) as ei:      # slices outside the slab
        e.finalize(z0=4, nz=8)
    assert ei.value.status == _lib.JFDK_ERR_INVALID
    with pytest.raises(_lib.JfdkError) as ei:      # derivatives need every slice
        e.bp_adjoint(torch_cuda.zeros((Z, int(g["vol"][1]), int(g["vol"][0])), device="cuda"))
    assert ei.value.status == _lib.JFDK_ERR_STATE


def test_memory_limit_fails_like_malloc(torch_cuda):
    from jenhine_b200 import _lib
    g = load_golden("mini_c1")
    e = engine_for(g)
    X, Y, Z = (int(v) for v in g["vol"])
    plane = X * Y * 4 * 2            # sum + weight
    held = e.device_bytes
    assert held > 0
    e.set_option(_lib.OPT_DEVICE_MEMORY_LIMIT, held + plane * (Z // 2))
    with pytest.raises(_lib.JfdkError) as ei:
        e.bp_set_slab(0, Z)
    assert ei.value.status == _lib.JFDK_ERR_OOM
    assert "CUDA failed to malloc " in str(ei.value)
    assert e.device_bytes == held     # nothing left behind
    e.bp_set_slab(0, Z // 2)          # half the volume fits
    assert e.device_bytes == held + plane * (Z // 2)
    with pytest.raises(_lib.JfdkError) as ei:   # no room left for the packed store
        e._check(e.lib.jfdk_bp_reserve(e.ctx, 4))
    assert ei.value.status == _lib.JFDK_ERR_OOM
    e.set_option(_lib.OPT_DEVICE_MEMORY_LIMIT, 0)
    e.bp_set_slab(0, Z)
    assert e.device_bytes == held + plane * Z
