"""GPU parity: libjfdk.so (through its C ABI) against the reference Cores'
outputs (golden fixtures) and the CPU oracle.

Tolerances (stated per test):
  * CT numbers and the EXACT-mode backprojection: bit for bit;
  * preprocessing: logf on the GPU vs glibc (both < 1 ulp), rel-L2 <= 1e-6;
  * ramp filter (dense product vs FFT) and fast-mode BP: rel-L2 <= 1e-5, the
    plain-FP32 parity bar.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def engine_for(g, **kw):
    from jenhine_b200.fdk import FDKEngine, ReconConfig, ScanConfig
    raw = g["raw"]
    X, Y, Z = (int(v) for v in g["vol"])
    pxy, pz = (float(v) for v in g["pitch"])
    scan = ScanConfig(num_views=raw.shape[0], dso=float(g["dso"]), dsd=0.0, num_dets_u=raw.shape[2],
                      num_dets_v=raw.shape[1], detector_pixel_size=0.0,
                      bright_field=float(g["bright_field"]), beam_hardening=tuple(g["bhc"]),
                      half_sample_rate=float(g["hsr"]))
    if "det_right" in g:   # conjugate-view compositing: the filter reads 2W-wide rows
        scan.filter_input_width = 2 * raw.shape[2]
        scan.detector_on_right = bool(g["det_right"])
    recon = ReconConfig(X, Y, Z, pxy, pz, ct_norm0=float(g["norm"][0]), ct_norm1=float(g["norm"][1]),
                        filter_cutoff_start=float(g["cut"][0]), filter_cutoff_end=float(g["cut"][1]),
                        adjust_points=tuple(g["adj_pts"]), adjust_level_db=tuple(g["adj_db"]))
    return FDKEngine(scan, recon, g["ptms"], **kw)


@pytest.fixture(scope="module", params=["mini_c1", "mini_c2", "mini_odd", "mini_tilt"])
def case(request):
    return load_golden(request.param)


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_preprocess_matches_reference(torch_cuda, case):
    e = engine_for(case)
    out = e.preprocess(to_dev(torch_cuda, case["raw"])).cpu().numpy()
    assert rel_l2(out, case["prep"]) <= 1e-6
    assert np.max(np.abs(out - case["prep"])) <= 4 * np.spacing(np.abs(case["prep"]).max())


def test_filter_matches_reference(torch_cuda, case):
    e = engine_for(case)
    out = e.filter(to_dev(torch_cuda, case["prep"]), v0=0).cpu().numpy()
    assert rel_l2(out, case["filt"]) <= 1e-5


def test_filter_matches_ramp_operator_and_oracle(torch_cuda, case, oracle):
    # the same rows through the oracle's FFT path, views 9..17 (second group)
    e = engine_for(case)
    v = slice(9, 18)
    out = e.filter(to_dev(torch_cuda, case["prep"][v]), v0=9).cpu().numpy()
    W = case["prep"].shape[2]
    H = oracle.filter_spectrum(oracle.fft_length(W), float(case["hsr"]), *case["cut"], case["adj_pts"],
                               case["adj_db"])
    ref = oracle.filter_projections(case["prep"], case["ptms"], H, float(case["dso"]))[v]
    assert rel_l2(out, ref) <= 1e-5


@pytest.mark.parametrize("kind,bar", [(1, 1e-5), (2, 5e-5), (3, 1e-5), (4, 1e-5), (5, 1e-7)],
                         ids=["tf32x3", "bf16x3", "fp16x3", "fp32-simt", "i8x14"])
def test_filter_ramp_products(torch_cuda, case, oracle, kind, bar):
    """Every ramp product against the oracle's FFT filter, in both forms."""
    from jenhine_b200 import _lib
    W = case["prep"].shape[2]
    H = oracle.filter_spectrum(oracle.fft_length(W), float(case["hsr"]), *case["cut"], case["adj_pts"],
                               case["adj_db"])
    ref = oracle.filter_projections(case["prep"], case["ptms"], H, float(case["dso"]))
    for form in ("fp32", "mixed"):
        e = engine_for(case, precision=form)
        e.set_option(_lib.OPT_RAMP_PRODUCT, kind)
        out = e.filter(to_dev(torch_cuda, case["prep"]), v0=0).cpu().numpy()
        assert rel_l2(out, ref) <= bar, (form, rel_l2(out, ref))


def test_int8_product_is_as_close_to_fp64_as_the_fft(torch_cuda, case, oracle):
    """The int8 product (the FP32 form's default) against the FP64 filter:
    no farther than the reference's float FFT filter (both start from the
    same float pre-weighted rows, whose rounding sets the floor), and
    within 1e-7 of that FFT filter."""
    from jenhine_b200 import _lib
    W = case["prep"].shape[2]
    H = oracle.filter_spectrum(oracle.fft_length(W), float(case["hsr"]), *case["cut"], case["adj_pts"],
                               case["adj_db"])
    fft = oracle.filter_projections(case["prep"], case["ptms"], H, float(case["dso"]))
    f64 = oracle.filter_projections_f64(case["prep"], case["ptms"], H, float(case["dso"]))
    e = engine_for(case)
    out = e.filter(to_dev(torch_cuda, case["prep"]), v0=0).cpu().numpy()
    e.set_option(_lib.OPT_RAMP_PRODUCT, _lib.RAMP_I8X14)
    assert np.array_equal(e.filter(to_dev(torch_cuda, case["prep"]), v0=0).cpu().numpy(), out)
    assert rel_l2(out, fft) <= 1e-7
    assert rel_l2(out, f64) <= 1.1 * rel_l2(fft, f64) + 1e-8, (rel_l2(out, f64), rel_l2(fft, f64))


@pytest.mark.parametrize("exact", [True, False])
def test_backprojection_matches_bpcore(torch_cuda, case, exact):
    e = engine_for(case, bp_exact=exact)
    e.bp_reset()
    e.bp_accumulate(to_dev(torch_cuda, case["filt"]), 0)
    out = e.finalize(apply_ctnum=False).cpu().numpy()
    if exact:
        np.testing.assert_array_equal(out, case["bp"])
    else:
        assert rel_l2(out, case["bp"]) <= 1e-5


def test_backprojection_in_chunks_equals_one_pass(torch_cuda, case):
    e = engine_for(case, bp_exact=True)
    f = to_dev(torch_cuda, case["filt"])
    e.bp_reset()
    for v0 in range(0, f.shape[0], 7):
        e.bp_accumulate(f[v0:v0 + 7].contiguous(), v0)
    np.testing.assert_array_equal(e.finalize(apply_ctnum=False).cpu().numpy(), case["bp"])


@pytest.mark.parametrize("form", ["exact", "fast", "mixed"])
def test_weight_volume_is_bit_identical(torch_cuda, case, form):
    """A backprojection over every view divides by a once-per-geometry volume
    of normalisation weights (JFDK_OPT_BP_WEIGHTS, default on): the same
    volume bit for bit as with the weights accumulated per sample, in both
    roundings of the FP32 form and in the mixed form, and again after the
    geometry changes (the weights follow it)."""
    torch = torch_cuda
    from jenhine_b200 import _lib
    raw = to_dev(torch, case["raw"])
    kw = {"precision": "mixed"} if form == "mixed" else {"bp_exact": form == "exact"}
    on = engine_for(case, **kw)
    off = engine_for(case, **kw)
    off.set_option(_lib.OPT_BP_WEIGHTS, 0)
    same = lambda a, b: torch.equal(torch.nan_to_num(a, 1e30), torch.nan_to_num(b, 1e30))
    assert same(on.reconstruct(raw).clone(), off.reconstruct(raw).clone())
    ptms = np.array(case["ptms"], np.float32).reshape(-1, 12).copy()
    ptms[:, 3] += 0.25 * ptms[:, 11]          # shift the detector by a quarter pixel in u
    on.set_bp_geometry(ptms)
    off.set_bp_geometry(ptms)
    assert same(on.reconstruct(raw).clone(), off.reconstruct(raw).clone())


def test_weight_volume_follows_the_rounding_and_the_memory_bound(torch_cuda, case):
    """One context switched between the roundings recomputes its weights
    (fast and EXACT weights differ), and under a device-memory bound that
    leaves no room for the weight volume a reconstruction falls back to the
    per-sample weights -- the same volume either way."""
    torch = torch_cuda
    from jenhine_b200 import _lib
    raw = to_dev(torch, case["raw"])
    same = lambda a, b: torch.equal(torch.nan_to_num(a, 1e30), torch.nan_to_num(b, 1e30))
    ref = {}
    for exact in (False, True):
        off = engine_for(case, bp_exact=exact)
        off.set_option(_lib.OPT_BP_WEIGHTS, 0)
        ref[exact] = off.reconstruct(raw).clone()
    e = engine_for(case)
    assert same(e.reconstruct(raw).clone(), ref[False])
    e.set_option(_lib.OPT_BP_EXACT, 1)
    assert same(e.reconstruct(raw).clone(), ref[True])
    e.set_option(_lib.OPT_BP_EXACT, 0)
    assert same(e.reconstruct(raw).clone(), ref[False])
    tight = engine_for(case)
    tight.reconstruct(raw)                     # allocates the stores (and the weights)
    X, Y, Z = (int(v) for v in case["vol"])
    fresh = engine_for(case)
    fresh.set_option(_lib.OPT_BP_WEIGHTS, 0)
    fresh.reconstruct(raw)
    without = fresh.device_bytes               # everything a reconstruction holds but the weights
    assert tight.device_bytes >= without + X * Y * Z * 4
    bound = engine_for(case)
    bound.set_option(_lib.OPT_DEVICE_MEMORY_LIMIT, without + X * Y * Z * 4 - 1)
    assert same(bound.reconstruct(raw).clone(), ref[False])
    assert bound.device_bytes <= without + X * Y * Z * 4 - 1


def test_ctnum_bit_exact(torch_cuda, case):
    e = engine_for(case)
    vol = to_dev(torch_cuda, case["bp"])
    np.testing.assert_array_equal(e.ctnum(vol).cpu().numpy(), case["hu"])


@pytest.mark.parametrize("exact", [True, False])
def test_reconstruct_end_to_end(torch_cuda, case, exact):
    e = engine_for(case, bp_exact=exact)
    hu = e.reconstruct(to_dev(torch_cuda, case["raw"])).cpu().numpy()
    # HU = mu * s - 1000: compare attenuation (HU + 1000) at the plain bar
    assert rel_l2(hu + 1000.0, case["hu"] + 1000.0) <= 1e-5
    assert np.max(np.abs(hu - case["hu"])) < 0.5
    hu_host = e.reconstruct_host(case["raw"])
    np.testing.assert_array_equal(hu_host, hu)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_reconstruct_host_overlapped_equals_device(torch_cuda, case, precision):
    """jfdk_reconstruct_host uploads chunk by chunk and backprojects and
    downloads slab by slab on two compute streams: the same volume as
    jfdk_reconstruct, bit for bit, in both forms and for several chunk and
    tile choices."""
    from jenhine_b200 import _lib
    e = engine_for(case, precision=precision)
    raw = to_dev(torch_cuda, case["raw"])
    for chunk, zpt in ((32, 8), (7, 4), (16, 8)):
        e.set_option(_lib.OPT_VIEW_CHUNK, chunk)
        e.set_option(_lib.OPT_BP_ZPT, zpt)
        hu = e.reconstruct(raw).cpu().numpy()
        np.testing.assert_array_equal(e.reconstruct_host(case["raw"]), hu)


def test_reconstruct_int16_output(torch_cuda, case, oracle):
    e = engine_for(case)
    import torch
    raw = to_dev(torch_cuda, case["raw"])
    hu = e.reconstruct(raw)
    hu16 = torch.empty(hu.shape, dtype=torch.int16, device="cuda")
    e.reconstruct(raw, out16=hu16)
    np.testing.assert_array_equal(hu16.cpu().numpy(), oracle.to_int16(hu.cpu().numpy()))


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_voxel_tiles_give_the_same_volume(torch_cuda, case, precision):
    """Every backprojection tile the autotuner chooses between (4, 8 or 32
    threads wide in x; 4, 8 or 16 slices per thread, 16-slice tiles 4 wide)
    computes each voxel the same way: the volume equals the default tile's
    bit for bit, in chunks too."""
    from jenhine_b200 import _lib
    raw = to_dev(torch_cuda, case["raw"])
    filt = to_dev(torch_cuda, case["filt"])
    e = engine_for(case, precision=precision, bp_exact=(precision == "fp32"))

    def run(zpt, tx):
        e.set_option(_lib.OPT_BP_ZPT, zpt)
        e.set_option(_lib.OPT_BP_TILE, tx)
        hu = e.reconstruct(raw).clone()
        e.bp_reset()
        for v0 in range(0, filt.shape[0], 9):
            e.bp_accumulate(filt[v0:v0 + 9].contiguous(), v0)
        return hu, e.finalize(apply_ctnum=False).clone()

    def same(a, b):
        return torch_cuda.equal(torch_cuda.nan_to_num(a, 1e30), torch_cuda.nan_to_num(b, 1e30))

    for zpt in (4, 8, 16):
        # the mixed form steps z from each thread's first slice: compare
        # within one tile depth; the FP32 volume does not depend on it either
        want = run(zpt, 4) if precision == "mixed" or zpt == 4 else want
        for tx in (8, 32):
            got = run(zpt, tx)
            assert same(got[0], want[0]) and same(got[1], want[1]), (zpt, tx)
    if precision == "fp32":
        np.testing.assert_array_equal(want[1].cpu().numpy(), case["bp"])


def test_voxel_tile_option_is_checked(torch_cuda, case):
    from jenhine_b200 import _lib
    e = engine_for(case)
    with pytest.raises(_lib.JfdkError):
        e.set_option(_lib.OPT_BP_TILE, 16)
    with pytest.raises(_lib.JfdkError):
        e.set_option(_lib.OPT_BP_ZPT, 32)


def test_tile_depth_in_effect(torch_cuda):
    """jfdk_get_option resolves the defaults: 16 slices per thread in the
    mixed form when W does not depend on z and the volume holds at least 8
    waves of 16-slice tiles (c2), else 8 (the small fixtures, a tilted orbit,
    the FP32 form); a set value as set."""
    from jenhine_b200 import _lib
    from jenhine_b200.fdk import FDKEngine
    from jenhine_b200.workloads import c2
    w = c2()
    for precision, want in (("fp32", 8), ("mixed", 16)):
        e = FDKEngine(w.scan, w.recon, w.geom.ptms(), precision=precision)
        assert e.tile_depth == want, precision
        e.close()
    for name, precision in (("mini_c2", "fp32"), ("mini_c2", "mixed"), ("mini_tilt", "mixed")):
        e = engine_for(load_golden(name), precision=precision)
        assert e.tile_depth == 8, (name, precision)
        assert e.get_option(_lib.OPT_BP_TILE) == 4
        e.set_option(_lib.OPT_BP_ZPT, 16)
        assert e.tile_depth == 16 and e.get_option(_lib.OPT_BP_TILE) == 4
        e.set_option(_lib.OPT_BP_ZPT, 0)
        assert e.tile_depth == 8
    e = engine_for(load_golden("mini_c2"))
    assert e.get_option(_lib.OPT_RAMP_PRODUCT) == _lib.RAMP_I8X14
    assert e.get_option(_lib.OPT_BP_WEIGHTS) == 1
    with pytest.raises(_lib.JfdkError):
        e.get_option(999)


def test_zfilter_matches_reference_order(torch_cuda, case):
    e = engine_for(case)
    x = case["filt"][:5].copy()
    out = e.zfilter(to_dev(torch_cuda, x)).cpu().numpy()
    f32 = np.float32
    ref = np.empty_like(x)
    H = x.shape[1]
    for i in range(H):  # ZFilterAgent.cpp:59-70
        o = x[:, i] * f32(0.5)
        o = o + x[:, max(i - 1, 0)] * f32(0.25)
        o = o + x[:, min(i + 1, H - 1)] * f32(0.25)
        ref[:, i] = o
    np.testing.assert_array_equal(out, ref)


def test_reference_bpcuda_case(torch_cuda, oracle):
    """UTBPAgent/UTBPCUDACore.cpp:16-201: one view, fixed PTM, 644 x 686
    detector, 500 x 500 x 50 volume (0.25 / 1.0 mm), first half of the
    projection 0.5, second half 1.0.  The reference accepts |d| > 0.05 on at
    most 0.2% of voxels between its GPU kernel and BPCore; here EXACT mode is
    bit-exact and the fast mode meets both that bar and rel-L2 <= 1e-5."""
    from jenhine_b200.fdk import FDKEngine, ReconConfig, ScanConfig
    ptm = np.array([-1.33897, -7.81194, 0.01236, 575.79443, -0.97515, -0.03862, 7.51861, 346.26642,
                    -0.00226, -0.00004, 0.00000, 1.00000], np.float32)
    U, V, X, Y, Z = 644, 686, 500, 500, 50
    proj = np.ones((1, V, U), np.float32)
    proj.reshape(-1)[: U * V // 2] = 0.5
    ref = oracle.bp(proj, ptm[None], X, Y, Z, 0.25, 1.0)
    for exact in (True, False):
        scan = ScanConfig(num_views=1, dso=443.0, dsd=683.0, num_dets_u=U, num_dets_v=V,
                          detector_pixel_size=0.198)
        e = FDKEngine(scan, ReconConfig(X, Y, Z, 0.25, 1.0), ptm[None], bp_exact=exact)
        e.bp_reset()
        e.bp_accumulate(to_dev(torch_cuda, proj), 0)
        out = e.finalize(apply_ctnum=False).cpu().numpy()
        if exact:
            np.testing.assert_array_equal(out, ref)
        else:
            # with one view a voxel that projects exactly onto the detector
            # edge may fall on either side of it (never seen -> 0/0); such
            # voxels count as differing, within the reference's 0.2% budget
            both = ~np.isnan(ref) & ~np.isnan(out)
            bad = np.count_nonzero(np.isnan(ref) != np.isnan(out))
            bad += np.count_nonzero(np.abs(out[both] - ref[both]) > 0.05)
            assert bad <= out.size // 500, f"fast mode: {bad} voxels differ"
            assert rel_l2(out[both], ref[both]) <= 1e-5


# ---- full benchmark size (c2): size-independent properties -------------------

@pytest.fixture(scope="module")
def c2_setup(torch_cuda):
    from jenhine_b200.fdk import FDKEngine
    from jenhine_b200.workloads import c2
    w = c2()
    e = FDKEngine(w.scan, w.recon, w.geom.ptms())
    return w, e


def test_c2_constant_projection_normalises_to_one(torch_cuda, c2_setup):
    """BP of an all-ones projection set is sum/weight == 1 exactly wherever a
    voxel is seen (the interpolated taper and the interpolated tapered ones
    are the same arithmetic), at the full 640 x 640 x 480 / 600-view size."""
    w, e = c2_setup
    ones = torch_cuda.ones((50, e.rows, e.filter_out_w), dtype=torch_cuda.float32, device="cuda")
    e.bp_reset()
    for v0 in range(0, w.geom.n_views, 50):
        e.bp_accumulate(ones, v0)
    out = e.finalize(apply_ctnum=False)
    seen = ~torch_cuda.isnan(out)
    assert seen.float().mean().item() > 0.99
    assert torch_cuda.all(out[seen] == 1.0).item()


def test_c2_slab_matches_oracle(torch_cuda, c2_setup, oracle):
    """End to end at full size; the oracle backprojects the engine's own
    filtered views for 2 slices (all 600 views) and filters 3 views."""
    w, e = c2_setup
    raw = w.raw_torch()
    hu = e.reconstruct(raw)
    pre = e.preprocess(raw[:3])
    filt_gpu = e.filter(pre, v0=0).cpu().numpy()
    H = oracle.filter_spectrum(e.fft_length, w.geom.half_sample_rate)
    pw = oracle.preweight_for_view(w.geom.ptms()[4], w.geom.sid, e.filter_in_w, e.rows)
    filt_ref = np.stack([oracle.filter_rows(pre[i].cpu().numpy(), H, e.fft_length, preweight=pw) for i in range(3)])
    assert rel_l2(filt_gpu, filt_ref) <= 1e-5
    # all views, filtered on the GPU, backprojected by the oracle on a slab
    allf = []
    for v0 in range(0, w.geom.n_views, 100):
        allf.append(e.filter(e.preprocess(raw[v0:v0 + 100]), v0=v0).cpu().numpy())
    allf = np.concatenate(allf)
    r = w.recon
    for z0 in (0, 237):
        ref = oracle.bp(allf, w.geom.ptms(), r.num_pixels_x, r.num_pixels_y, r.num_pixels_z, r.pitch_xy,
                        r.pitch_z, z0=z0, nz=2)
        ref = oracle.ctnum(ref, r.ct_norm0, r.ct_norm1)
        got = hu[z0:z0 + 2].cpu().numpy()
        assert rel_l2(got + 1000.0, ref + 1000.0) <= 1e-5
        assert np.nanmax(np.abs(got - ref)) < 1.0
