"""One volume in z-slabs (jfdk_filter_raw, then jfdk_bp_set_slab /
jfdk_bp_reset / jfdk_bp_accumulate / jfdk_finalize per slab;
jenhine_b200.zslab) on one GPU: the ranks are emulated in turn on one
engine -- each filters its views into the shared frames, then each
backprojects every view, in order, into its slab -- and the slabs together
equal jfdk_reconstruct bit for bit, in both forms and with compositing.  The
store-level entry points (jfdk_filter_to_store, jfdk_store_range,
jfdk_backproject_store) are checked the same way.  The exchange between
processes is covered on CPU (test_multirank.py)."""
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


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
@pytest.mark.parametrize("name", ["mini_c1", "mini_c2", "mini_comp", "mini_odd", "mini_tilt"])
def test_emulated_ranks_equal_reconstruct(torch_cuda, name, precision, world):
    torch = torch_cuda
    from jenhine_b200.zslab import slab_ranges, view_ranges
    g = load_golden(name)
    e = engine_for(g, precision=precision)
    raw = to_dev(torch, g["raw"])
    whole = e.reconstruct(raw).clone()
    Z = whole.shape[0]
    views = view_ranges(raw.shape[0], world)
    frames = torch.empty((raw.shape[0], e.rows, e.filter_out_w), dtype=torch.float32, device="cuda")
    for v0, nv in views:              # each rank filters its views
        e.filter_raw(raw, v0, nv, out=frames[v0:v0 + nv])
    parts = []
    for z0, nz in slab_ranges(Z, world, e.tile_depth):
        if not nz:
            continue
        e.bp_set_slab(z0, nz)         # each rank backprojects every view into its slab
        e.bp_reset()
        for v0, nv in views:
            e.bp_accumulate(frames[v0:v0 + nv], v0)
        parts.append(e.finalize(apply_ctnum=True, z0=z0, nz=nz))
    got = torch.cat(parts)
    torch.cuda.synchronize()
    assert torch.equal(torch.nan_to_num(got, 1e30), torch.nan_to_num(whole, 1e30))
    # the store-level entry points, the same way
    e.bp_set_slab(0, Z)
    for v0, nv in views:
        e.filter_to_store(raw, v0, nv)
    got = torch.cat([e.backproject_store(z0, nz) for z0, nz in slab_ranges(Z, world, e.tile_depth) if nz])
    torch.cuda.synchronize()
    assert torch.equal(torch.nan_to_num(got, 1e30), torch.nan_to_num(whole, 1e30))


def test_store_range_describes_the_store(torch_cuda):
    from jenhine_b200 import _lib
    g = load_golden("mini_c2")
    for precision in ("fp32", "mixed"):
        e = engine_for(g, precision=precision)
        (p0, n0), sc0 = e.store_range(0, 4)
        (p1, n1), sc1 = e.store_range(4, 6)
        frame = e.rows * e.filter_out_w * (8 if precision == "mixed" else 16)   # FP16 records / FP32 quads
        assert n0 == 4 * frame and n1 == 6 * frame and p1 == p0 + 4 * frame
        if precision == "mixed":
            assert sc0[1] == 16 and sc1[0] == sc0[0] + 16
        else:
            assert sc0 is None and sc1 is None
        with pytest.raises(_lib.JfdkError):
            e.store_range(g["raw"].shape[0] - 2, 4)


def test_world_of_one_is_reconstruct(torch_cuda):
    torch = torch_cuda
    from jenhine_b200.zslab import reconstruct_zslab
    g = load_golden("mini_c2")
    e = engine_for(g, precision="mixed")
    raw = to_dev(torch, g["raw"])
    whole = e.reconstruct(raw).clone()
    z0, vol = reconstruct_zslab(e, raw, 0, 1)
    torch.cuda.synchronize()
    assert z0 == 0 and torch.equal(torch.nan_to_num(vol, 1e30), torch.nan_to_num(whole, 1e30))
