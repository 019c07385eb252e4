"""GPU parity at the benchmark configurations, against the reference's own
Cores compiled from source (oracle/_ref: PreProcessingCore, FilterAgent's
FilterCore + PreFilterWeightGenerator, BPCore, CTNumCore).

* c1 at its full size: 360 views of 256 x 256 into 128^3, every voxel.
* c2 (600 views of 768 x 768, 640 x 640 voxels at 0.125 mm) on its central
  16-slice slab, every view, filter included.  The slab is a 16-slice volume
  whose axis (i - 7.5) * pitch equals the full volume's at slices 232..247
  bit for bit (BPCore.cpp:47-66), so the reference backprojects exactly the
  full volume's arithmetic there.

Bars:
  * preprocessing rel-L2 <= 1e-6 (GPU logf vs glibc);
  * filter rel-L2 <= 1e-6: the FP32 form's int8 product (exact integer
    accumulation, rounded once) against the reference's float FFT filter,
    both computing the same convolution of the same float pre-weighted rows;
  * EXACT-mode backprojection of the reference's filtered views: bit for
    bit, and the set of voxels seen identical;
  * default (fast) backprojection rel-L2 <= 1e-5;
  * CT numbers bit for bit given the same float volume;
  * the whole pipeline (the engine's own filter and backprojection) rel-L2 <=
    1e-5 on the attenuation HU + 1000, in both backprojection modes.  For c2
    the engine is also held against the exact FDK (the FP64 oracle,
    tests/fp64_fdk.py): its rel-L2 to FP64 at most 1.1 x that of the
    reference's own cores.
The reference runs on all host cores, as its agents thread it
(FilterAgent rows per thread, BPAgent slices per thread)."""
import os

import numpy as np
import pytest

from test_gpu_parity import to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def rel_l2_seen(a, b):
    """rel-L2 over the voxels both volumes see (never-seen voxels are 0/0)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.linalg.norm(a[m] - b[m]) / np.linalg.norm(b[m]))


def reference_run(refcores, w, raw_np):
    """The reference Cores on the whole scan: preprocessed, filtered,
    backprojected and CT-numbered volumes."""
    g, r = w.geom, w.recon
    n = os.cpu_count() or 1
    ptms = g.ptms()
    prep = refcores.preprocess(raw_np, w.bright_field, w.beam_hardening, nthreads=n)
    filt = refcores.filter(prep, ptms, g.half_sample_rate, g.sid, nthreads=n)
    bp = refcores.bp(filt, ptms, r.num_pixels_x, r.num_pixels_y, r.num_pixels_z, r.pitch_xy, r.pitch_z,
                     nthreads=n)
    hu = refcores.ctnum(bp, r.ct_norm0, r.ct_norm1)
    return {"prep": prep, "filt": filt, "bp": bp, "hu": hu}


def rel_l2_chunked(torch, ref_in, ref_out, fn, chunk=50):
    """rel-L2 of fn(device input chunk, first view) against ref_out over all
    views, accumulated chunk by chunk (the c2 arrays are 1.4 GB each)."""
    num = den = 0.0
    for v0 in range(0, ref_in.shape[0], chunk):
        got = fn(to_dev(torch, ref_in[v0:v0 + chunk]), v0).cpu().numpy().astype(np.float64)
        exp = ref_out[v0:v0 + chunk].astype(np.float64)
        num += float(np.sum((got - exp) ** 2))
        den += float(np.sum(exp ** 2))
    return (num / den) ** 0.5


def check_config(torch, refcores, w, raw, fp64_oracle=None):
    from jenhine_b200.fdk import FDKEngine
    raw_np = raw.cpu().numpy()
    ref = reference_run(refcores, w, raw_np)
    ptms = w.geom.ptms()
    exact = FDKEngine(w.scan, w.recon, ptms, bp_exact=True)
    fast = FDKEngine(w.scan, w.recon, ptms)
    res = {}
    # stage by stage, each stage fed the reference's own input
    res["prep"] = rel_l2_chunked(torch, raw_np, ref["prep"], lambda x, v0: exact.preprocess(x))
    res["filt"] = rel_l2_chunked(torch, ref["prep"], ref["filt"], lambda x, v0: exact.filter(x, v0=v0))
    assert res["prep"] <= 1e-6, res
    assert res["filt"] <= 1e-6, res
    for name, e in (("exact", exact), ("fast", fast)):
        e.bp_reset()
        for v0 in range(0, w.geom.n_views, 50):
            e.bp_accumulate(to_dev(torch, ref["filt"][v0:v0 + 50]), v0)
        out = e.finalize(apply_ctnum=False).cpu().numpy()
        assert np.array_equal(np.isfinite(out), np.isfinite(ref["bp"])), name
        if name == "exact":
            np.testing.assert_array_equal(out, ref["bp"])
        else:
            res["bp_fast"] = rel_l2_seen(out, ref["bp"])
            assert res["bp_fast"] <= 1e-5, res
    np.testing.assert_array_equal(exact.ctnum(to_dev(torch, ref["bp"])).cpu().numpy(), ref["hu"])
    # the whole pipeline
    hus = {}
    for name, e in (("exact", exact), ("fast", fast)):
        hus[name] = e.reconstruct(raw).cpu().numpy()
        res["recon_" + name] = rel_l2_seen(hus[name] + 1000.0, ref["hu"] + 1000.0)
    exact.close()
    fast.close()
    for name in hus:
        assert res["recon_" + name] <= 1e-5, res
    if fp64_oracle is None:
        return res
    from fp64_fdk import all_points, case_from_workload, fdk_f64, interior
    r = w.recon
    g = case_from_workload(w, raw_np)
    pts = all_points(r.num_pixels_x, r.num_pixels_y, r.num_pixels_z)
    f64 = fdk_f64(fp64_oracle, g, pts).reshape(ref["hu"].shape)
    inside = interior(g, pts).reshape(ref["hu"].shape)
    def to_f64(hu):
        m = inside & np.isfinite(hu) & np.isfinite(f64)
        return float(np.linalg.norm(hu[m] - f64[m]) / np.linalg.norm(f64[m] + 1000.0))
    res["reference_vs_fp64"] = to_f64(ref["hu"].astype(np.float64))
    for name in hus:
        res[name + "_vs_fp64"] = to_f64(hus[name].astype(np.float64))
        assert res[name + "_vs_fp64"] <= 1.1 * res["reference_vs_fp64"], res
    return res


def test_c1_full_size_matches_reference_cores(torch_cuda, refcores):
    """c1 at its full size (360 views of 256 x 256 -> 128^3), every voxel."""
    from jenhine_b200.workloads import c1
    w = c1()
    res = check_config(torch_cuda, refcores, w, w.raw_torch())
    print("c1 full size vs reference cores:", res)


def test_c2_central_slab_matches_reference_cores(torch_cuda, refcores, oracle):
    """c2: every view (600 of 768 x 768) of c2's own scan, the central 16 of
    480 slices of the 640 x 640 x 480 volume."""
    from jenhine_b200.workloads import c2
    w = c2()
    raw = w.raw_torch()          # c2's scan of c2's phantom
    Z = w.recon.num_pixels_z
    w.recon.num_pixels_z = 16    # slices Z/2 - 8 .. Z/2 + 7: the axis (i - 7.5) * pitch
    assert Z // 2 - 8 + 7.5 == (Z - 1) / 2
    res = check_config(torch_cuda, refcores, w, raw, fp64_oracle=oracle)
    print("c2 central slab vs reference cores:", res)
