"""Conjugate-view compositing on the GPU (jfdk_composite_frames and the
compositing jfdk_reconstruct path) against the reference's CompositeCore,
2W-wide mirrored FilterCore, BPCore and CTNumCore (fixture mini_comp: an
offset detector whose principal point is 10 columns from its left edge).

Bars: the composite rows rel-L2 <= 1e-6 (the same float operations; the
inverse transform matrices come from a separate restatement of the same
solve); filter <= 1e-5; HU + 1000 <= 1e-5 and < 0.5 HU."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from test_gpu_parity import engine_for, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


@pytest.fixture(scope="module")
def comp_case():
    return load_golden("mini_comp")


def test_composite_frames_match_reference(torch_cuda, comp_case):
    g = comp_case
    e = engine_for(g)
    N = g["prep"].shape[0]
    conj = np.stack([g["prep"][(k + N // 2) % N] for k in range(N)])
    out = e.composite(to_dev(torch_cuda, g["prep"]), to_dev(torch_cuda, conj), v0=0).cpu().numpy()
    assert out.shape == g["comp"].shape
    assert rel_l2(out, g["comp"]) <= 1e-6
    assert np.max(np.abs(out - g["comp"])) <= 1e-5 * np.abs(g["comp"]).max()


def test_filter_of_composite_rows(torch_cuda, comp_case):
    g = comp_case
    e = engine_for(g)
    out = e.filter(to_dev(torch_cuda, g["comp"]), v0=0).cpu().numpy()
    assert rel_l2(out, g["filt"]) <= 1e-5


@pytest.mark.parametrize("exact", [True, False])
def test_reconstruct_with_compositing(torch_cuda, comp_case, exact):
    g = comp_case
    e = engine_for(g, bp_exact=exact)
    hu = e.reconstruct(to_dev(torch_cuda, g["raw"])).cpu().numpy()
    assert rel_l2(hu + 1000.0, g["hu"] + 1000.0) <= 1e-5
    assert np.max(np.abs(hu - g["hu"])) < 0.5


def test_reconstruct_host_with_compositing(torch_cuda, comp_case):
    """The host path uploads each chunk's views and their conjugates before
    the chunk's compositing pass: the same volume as the device path."""
    from jenhine_b200 import _lib
    g = comp_case
    e = engine_for(g)
    e.set_option(_lib.OPT_VIEW_CHUNK, 5)
    hu = e.reconstruct(to_dev(torch_cuda, g["raw"])).cpu().numpy()
    np.testing.assert_array_equal(e.reconstruct_host(g["raw"]), hu)


def test_reconstruct_with_compositing_mixed(torch_cuda, comp_case):
    g = comp_case
    hu = engine_for(g, precision="mixed").reconstruct(to_dev(torch_cuda, g["raw"])).cpu().numpy()
    assert rel_l2(hu + 1000.0, g["hu"] + 1000.0) <= 2e-4


def test_composite_needs_a_compositing_context(torch_cuda):
    from jenhine_b200 import _lib
    g = load_golden("mini_c1")
    e = engine_for(g)
    x = to_dev(torch_cuda, g["prep"][:2])
    with pytest.raises(_lib.JfdkError):
        e.composite(x, x)
