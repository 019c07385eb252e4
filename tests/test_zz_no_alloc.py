"""jfdk_filter_frames_noalloc: the ramp-filter stage for callers that cannot
allocate device memory while they run (framework-owned memory pools or
budgets, real-time acquisition threads).  Its working rows sit in a fixed
4 MiB array inside libjfdk.so and its ramp product runs on FP32 CUDA cores in
either form.  Checked through the C ABI against jfdk_filter_frames on two
calls in a row (the array keeps the first call's contents when the second
starts): at the filter's parity tolerance against the FP32 form's default
product (rel-L2 <= 1e-5, as in test_gpu_parity), at the BF16x3 product's
tolerance (5e-5) against the mixed form's default, bit for bit against
jfdk_filter_frames with the same FP32 CUDA-core product; and for its size
limit.

This file is collected last on purpose."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def _engine(g, precision="fp32"):
    from jenhine_b200.fdk import FDKEngine, ReconConfig, ScanConfig
    raw = g["raw"]
    X, Y, Z = (int(v) for v in g["vol"])
    scan = ScanConfig(num_views=raw.shape[0], dso=float(g["dso"]), dsd=0.0, num_dets_u=raw.shape[2],
                      num_dets_v=raw.shape[1], detector_pixel_size=0.0, bright_field=float(g["bright_field"]),
                      beam_hardening=tuple(g["bhc"]), half_sample_rate=float(g["hsr"]))
    recon = ReconConfig(X, Y, Z, float(g["pitch"][0]), float(g["pitch"][1]),
                        filter_cutoff_start=float(g["cut"][0]), filter_cutoff_end=float(g["cut"][1]),
                        adjust_points=tuple(g["adj_pts"]), adjust_level_db=tuple(g["adj_db"]))
    return FDKEngine(scan, recon, g["ptms"], precision=precision)


def test_noalloc_filter_matches_filter_on_two_calls_in_a_row():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    g = load_golden("mini_c2")
    e = _engine(g)
    prep = torch.from_numpy(np.ascontiguousarray(g["prep"])).cuda()
    # two different view ranges back to back: the second call must not see
    # anything left in the shared array by the first
    for v0, v1 in ((0, 9), (9, 30)):
        frames = prep[v0:v1].contiguous()
        want = e.filter(frames, v0=v0).cpu().numpy()
        out = torch.full((v1 - v0, e.rows, e.filter_out_w), float("nan"), device="cuda")
        got = e.filter_noalloc(frames, v0=v0, out=out).cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_l2(got, want) <= 1e-5
        assert rel_l2(got, g["filt"][v0:v1]) <= 1e-5


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_noalloc_filter_runs_the_fp32_cuda_core_product_in_either_form(precision):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from jenhine_b200 import _lib
    g = load_golden("mini_c2")
    e = _engine(g, precision)
    simt = _engine(g, precision)
    simt.set_option(_lib.OPT_RAMP_PRODUCT, _lib.RAMP_FP32_SIMT)
    prep = torch.from_numpy(np.ascontiguousarray(g["prep"])).cuda()
    for v0, v1 in ((0, 9), (9, 30)):
        frames = prep[v0:v1].contiguous()
        got = e.filter_noalloc(frames, v0=v0).cpu().numpy()
        np.testing.assert_array_equal(got, simt.filter(frames, v0=v0).cpu().numpy())
        default = e.filter(frames, v0=v0).cpu().numpy()   # TF32x3 (fp32) or BF16x3 (mixed)
        assert rel_l2(got, default) <= (5e-5 if precision == "mixed" else 1e-5)


def test_noalloc_filter_rejects_requests_beyond_the_array():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from jenhine_b200 import _lib
    from jenhine_b200.fdk import FDKEngine, ReconConfig, ScanConfig
    # 768 x 768 frames: one view fits the 1,048,576-float array, two do not
    scan = ScanConfig(num_views=2, dso=500.0, dsd=800.0, num_dets_u=768, num_dets_v=768,
                      detector_pixel_size=0.2)
    from jenhine_b200.phantom import ScanGeometry
    ptms = ScanGeometry(2, 500.0, 800.0, 768, 768, 0.2, 0.2).ptms()
    e = FDKEngine(scan, ReconConfig(8, 8, 8, 1.0, 1.0), ptms)
    frames = torch.zeros((2, 768, 768), device="cuda")
    out = torch.empty_like(frames)
    e.filter_noalloc(frames[:1], v0=0, out=out[:1])
    with pytest.raises(_lib.JfdkError) as err:
        e.filter_noalloc(frames, v0=0, out=out)
    assert err.value.status == _lib.JFDK_ERR_INVALID
    assert "static scratch" in str(err.value)
