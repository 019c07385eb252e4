"""Batches of scans of uneven size (jfdk_batch_*, jfdk_autotune): one persistent
backprojection launch over all scans' tiles, recorded as a CUDA graph and
replayed.  Each scan's volume must equal its own jfdk_reconstruct bit for
bit with the same options: the batch runs the same per-voxel arithmetic.  In
the FP32 form the options the autotuner picks (tile depth, views per chunk)
do not change the arithmetic either; in the mixed form the coordinates step
from each thread's first slice, so the tile depth moves u, v by rounding and
the single reconstructions are taken with the batch's tuned options."""
import pytest

pytestmark = pytest.mark.gpu

# (views, detector, volume) of four small scans of uneven size
SHAPES = [(36, 48, (24, 24, 24)), (60, 64, (32, 32, 20)), (24, 40, (16, 16, 16)), (48, 56, (40, 24, 12))]


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def make_scans(precision, shapes=SHAPES):
    from jenhine_b200.fdk import FDKEngine, ReconConfig
    from jenhine_b200.phantom import ScanGeometry
    from jenhine_b200.workloads import Workload
    out = []
    for i, (views, det, (X, Y, Z)) in enumerate(shapes):
        pix = 60.0 / det
        vox = 30.0 / X
        w = Workload(f"s{i}", ScanGeometry(views, 480.0 + 20 * i, 760.0 + 30 * i, det, det, pix, pix, seed=900 + i),
                     ReconConfig(X, Y, Z, vox, vox, ct_norm0=1.0, ct_norm1=1.0), 6, 0, 1e5)
        e = FDKEngine(w.scan, w.recon, w.geom.ptms(), precision=precision)
        out.append((w, e, w.raw_torch()))
    return out


def same(torch, a, b):
    return torch.equal(torch.nan_to_num(a, 1e30), torch.nan_to_num(b, 1e30))


@pytest.mark.parametrize("schedule", [None, "persistent", "pipelined"])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_batch_equals_single_reconstructions(torch_cuda, precision, schedule):
    torch = torch_cuda
    from jenhine_b200.fdk import FDKBatch
    scans = make_scans(precision)
    untuned = [e.reconstruct(raw).clone() for _, e, raw in scans]
    batch = FDKBatch([e for _, e, _ in scans], autotune=True, graph=True, schedule=schedule)
    refs = [e.reconstruct(raw).clone() for _, e, raw in scans]   # with the tuned options
    if precision == "fp32":
        assert all(same(torch, u, r) for u, r in zip(untuned, refs))
    raws = [raw for _, _, raw in scans]
    outs = [torch.full_like(r, -7.0) for r in refs]
    batch.run(raws, outs)            # direct run, recorded as a graph
    torch.cuda.synchronize()
    assert all(same(torch, o, r) for o, r in zip(outs, refs))
    assert batch.schedule == (schedule or batch.schedule) and batch.schedule in ("persistent", "pipelined")
    for o in outs:
        o.fill_(-7.0)
    n0 = batch.launches
    batch.run(raws, outs)            # graph replay
    torch.cuda.synchronize()
    assert batch.launches > n0
    assert all(same(torch, o, r) for o, r in zip(outs, refs))
    outs2 = [torch.empty_like(r) for r in refs]
    batch.run(raws, outs2)           # new buffers: recorded again
    torch.cuda.synchronize()
    assert all(same(torch, o, r) for o, r in zip(outs2, refs))
    batch.close()


def test_batch_rejects_mixed_forms(torch_cuda):
    from jenhine_b200 import _lib
    from jenhine_b200.fdk import FDKBatch
    a = make_scans("fp32", SHAPES[:1])
    b = make_scans("mixed", SHAPES[:1])
    with pytest.raises(_lib.JfdkError):
        FDKBatch([a[0][1], b[0][1]], autotune=False)


def test_sixteen_uneven_scans_in_one_persistent_launch(torch_cuda):
    """16 scans of uneven size (views, detectors and volumes drawn from the
    four shapes, tile depths 4 and 8 mixed): one persistent backprojection
    launch, every volume equal to the scan's own reconstruction."""
    torch = torch_cuda
    from jenhine_b200 import _lib
    from jenhine_b200.fdk import FDKBatch
    shapes = [SHAPES[i % 4] for i in range(16)]
    for precision in ("fp32", "mixed"):
        scans = make_scans(precision, shapes)
        for i, (_, e, _) in enumerate(scans):
            e.set_option(_lib.OPT_BP_ZPT, 4 if i % 3 == 0 else 8)
        refs = [e.reconstruct(raw).clone() for _, e, raw in scans]
        batch = FDKBatch([e for _, e, _ in scans], autotune=False, graph=False, schedule="persistent")
        outs = [torch.full_like(r, -7.0) for r in refs]
        n0 = batch.launches
        batch.run([raw for _, _, raw in scans], outs)
        torch.cuda.synchronize()
        assert batch.launches - n0 == 1
        assert all(same(torch, o, r) for o, r in zip(outs, refs))
        batch.close()


def test_mixed_scans_of_sixteen_slice_tiles_in_one_launch(torch_cuda):
    """The mixed form's 16-slice tiles (its default on large volumes) run in
    launches of their own kind: scans of 16-slice tiles share one persistent
    launch, and the scans of 8-slice tiles among them share another."""
    torch = torch_cuda
    from jenhine_b200 import _lib
    from jenhine_b200.fdk import FDKBatch
    for depths, launches in (((16, 16, 16, 16), 1), ((16, 8, 16, 4), 2)):
        scans = make_scans("mixed")
        for d, (_, e, _) in zip(depths, scans):
            e.set_option(_lib.OPT_BP_ZPT, d)
            assert e.tile_depth == d
        refs = [e.reconstruct(raw).clone() for _, e, raw in scans]
        batch = FDKBatch([e for _, e, _ in scans], autotune=False, graph=False, schedule="persistent")
        outs = [torch.full_like(r, -7.0) for r in refs]
        n0 = batch.launches
        batch.run([raw for _, _, raw in scans], outs)
        torch.cuda.synchronize()
        assert batch.launches - n0 == launches
        assert all(same(torch, o, r) for o, r in zip(outs, refs))
        batch.close()


def test_batch_on_contexts_that_have_not_reconstructed(torch_cuda):
    """Contexts straight from creation, two of one shape (the autotuner
    answers the second from its cache): the batch allocates their
    backprojection stores before it plans its persistent launches, whose
    parameters name them, and every volume equals the scan's own
    reconstruction taken afterwards."""
    torch = torch_cuda
    from jenhine_b200.fdk import FDKBatch
    for precision in ("fp32", "mixed"):
        scans = make_scans(precision, [SHAPES[0], SHAPES[1], SHAPES[0]])
        batch = FDKBatch([e for _, e, _ in scans], autotune=True, graph=False, schedule="persistent")
        outs = [torch.full((w.recon.num_pixels_z, w.recon.num_pixels_y, w.recon.num_pixels_x), -7.0, device="cuda")
                for w, _, _ in scans]
        batch.run([raw for _, _, raw in scans], outs)
        torch.cuda.synchronize()
        refs = [e.reconstruct(raw).clone() for _, e, raw in scans]
        assert all(same(torch, o, r) for o, r in zip(outs, refs))
        batch.close()
