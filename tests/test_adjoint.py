"""Derivatives of the FP32 form (jfdk_bp_adjoint, jfdk_filter_adjoint,
jfdk_geometry_gradient, jenhine_b200.autograd).

  * dot-product tests <A x, y> = <x, A^T y> for the backprojector, the ramp
    filter and their composition, on signed random FP32 vectors (standard
    normal; inner products summed in FP64), at the fixture sizes and at the
    differentiation workload's size (360 views of 512 x 512 -> 256^3):
    |<A x, y> - <x, A^T y>| / (|A x| |y|) <= 1e-6 (signed vectors cancel in
    the inner products, so the difference is measured against the norms; the
    plain relative difference is reported beside it).  The filter adjoint is
    the transpose of the FP32 product (JFDK_RAMP_FP32_SIMT), which these tests
    select; the tensor-core split products differ from it by their ~2^-22
    rounding;
  * the gradients of L = sum over interior voxels of (vol - target)^2 with
    respect to 32 random per-view motion parameters and 32 random projection
    samples, against FP64 central finite differences of the same loss computed
    by the FP64 oracle (filter and backprojection in double, FP64 matrices),
    on the 40-view fixture and at the differentiation workload's full size.
"""
import numpy as np
import pytest

from conftest import load_golden
from fp64_fdk import report
from test_gpu_parity import engine_for, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def dot(a, b):
    return float((a.double() * b.double()).sum().item())


def bp_forward(e, q, chunk=64):
    import torch
    e.bp_reset()
    for v0 in range(0, q.shape[0], chunk):
        e.bp_accumulate(q[v0:v0 + chunk], v0)
    vol = e.finalize(apply_ctnum=False)
    return vol, torch.isfinite(vol)


def dot_errors(lhs, rhs, norm):
    """(|lhs - rhs| / norm, |lhs - rhs| / |lhs|): the difference against the
    Cauchy-Schwarz bound |A x| |y| of both inner products, and against lhs."""
    d = abs(lhs - rhs)
    return d / max(norm, 1e-300), d / max(abs(lhs), 1e-300)


def check_bp_dot(torch, e, nv, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    q = torch.randn((nv, e.rows, e.filter_out_w), generator=gen, device="cuda")
    vol, seen = bp_forward(e, q)
    vol = torch.nan_to_num(vol)
    y = torch.randn(vol.shape, generator=gen, device="cuda") * seen
    qb = torch.cat([e.bp_adjoint(y, v0, min(64, nv - v0)) for v0 in range(0, nv, 64)])
    lhs, rhs = dot(vol, y), dot(q, qb)
    return dot_errors(lhs, rhs, vol.double().norm().item() * y.double().norm().item())


def check_filter_dot(torch, e, nv, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn((nv, e.rows, e.filter_in_w), generator=gen, device="cuda")
    y = torch.randn((nv, e.rows, e.filter_out_w), generator=gen, device="cuda")
    fx = e.filter(x, v0=0)
    xb = e.filter_adjoint(y, v0=0)
    lhs, rhs = dot(fx, y), dot(x, xb)
    return dot_errors(lhs, rhs, fx.double().norm().item() * y.double().norm().item())


@pytest.mark.parametrize("name", ["mini_c1", "mini_c2", "mini_odd", "mini_tilt"])
def test_bp_adjoint_dot_product(torch_cuda, name):
    g = load_golden(name)
    e = engine_for(g)
    r, rel = check_bp_dot(torch_cuda, e, g["raw"].shape[0], 1)
    report(name, "bp_adjoint_dot", {"over_norms": r, "rel": rel})
    assert r <= 1e-6


def fp32_product(e):
    from jenhine_b200 import _lib
    e.set_option(_lib.OPT_RAMP_PRODUCT, _lib.RAMP_FP32_SIMT)
    return e


@pytest.mark.parametrize("name", ["mini_c1", "mini_c2", "mini_odd", "mini_tilt"])
def test_filter_adjoint_dot_product(torch_cuda, name):
    g = load_golden(name)
    e = fp32_product(engine_for(g))
    r, rel = check_filter_dot(torch_cuda, e, g["raw"].shape[0], 2)
    report(name, "filter_adjoint_dot", {"over_norms": r, "rel": rel})
    assert r <= 1e-6


@pytest.mark.parametrize("name", ["mini_c1", "mini_c2", "mini_odd", "mini_tilt"])
def test_filter_adjoint_against_tensor_core_forward(torch_cuda, name):
    """The default (TF32x3) forward against the same adjoint: within its
    split's rounding."""
    g = load_golden(name)
    assert check_filter_dot(torch_cuda, engine_for(g), g["raw"].shape[0], 2)[0] <= 1e-5


def test_derivatives_after_reconstruct(torch_cuda):
    """A whole reconstruction first (it allocates the filter stage's working
    buffers) must leave the derivative operators intact: the same adjoint
    filter and adjoint backprojection as on a fresh context."""
    torch = torch_cuda
    g = load_golden("mini_c2")
    nv = g["raw"].shape[0]
    gen = torch.Generator(device="cuda").manual_seed(7)
    fresh, used = fp32_product(engine_for(g)), fp32_product(engine_for(g))
    used.reconstruct(to_dev(torch, g["raw"]))
    y = torch.rand((nv, fresh.rows, fresh.filter_out_w), generator=gen, device="cuda")
    assert torch.equal(fresh.filter_adjoint(y, v0=0), used.filter_adjoint(y, v0=0))
    q = torch.rand((nv, fresh.rows, fresh.filter_out_w), generator=gen, device="cuda")
    vols = [bp_forward(e, q)[0] for e in (fresh, used)]
    assert torch.equal(torch.nan_to_num(vols[0]), torch.nan_to_num(vols[1]))
    vb = torch.rand(vols[0].shape, generator=gen, device="cuda")
    # the adjoint scatters with float atomics: equal up to the order of additions
    a, b = fresh.bp_adjoint(vb, 0, nv), used.bp_adjoint(vb, 0, nv)
    assert ((a - b).norm() / a.norm()).item() <= 1e-6


def test_fdk_adjoint_dot_product(torch_cuda):
    """<B F x, y> = <x, F^T B^T y> through the autograd binding's backward."""
    import torch
    from jenhine_b200.autograd import FDKFunction
    g = load_golden("mini_c2")
    e = fp32_product(engine_for(g))
    nv = g["raw"].shape[0]
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((nv, e.rows, e.filter_in_w), generator=gen, device="cuda", requires_grad=True)
    theta = torch.zeros((nv, 6), dtype=torch.float64, requires_grad=True)
    vol = FDKFunction.apply(x, theta, e, g["ptms"])
    y = torch.randn(vol.shape, generator=gen, device="cuda") * torch.isfinite(vol)
    (torch.nan_to_num(vol) * y).sum().backward()
    v = torch.nan_to_num(vol.detach())
    lhs, rhs = dot(v, y), dot(x.detach(), x.grad)
    r, rel = dot_errors(lhs, rhs, v.double().norm().item() * y.double().norm().item())
    report("mini_c2", "fdk_adjoint_dot", {"over_norms": r, "rel": rel})
    assert r <= 1e-6


def test_adjoint_dot_products_differentiation_size(torch_cuda):
    """At the differentiation workload's size: 360 views of 512 x 512,
    256^3 voxels, with the workload's per-view motion in the geometry."""
    from jenhine_b200.fdk import FDKEngine
    from jenhine_b200.motion import moved_ptms, seeded_motion
    from jenhine_b200.workloads import c3
    w = c3()
    P0 = w.geom.ptms()
    e = fp32_product(FDKEngine(w.scan, w.recon, P0))
    e.set_bp_geometry(moved_ptms(P0, seeded_motion(w.geom.n_views, 7)).astype(np.float32))
    (rb, rb_rel), (rf, rf_rel) = check_bp_dot(torch_cuda, e, w.geom.n_views, 4), check_filter_dot(torch_cuda, e, 40, 5)
    report("c3", "adjoint_dot", {"bp_over_norms": rb, "bp_rel": rb_rel, "filter_over_norms": rf, "filter_rel": rf_rel})
    assert rb <= 1e-6 and rf <= 1e-6


# ---- gradients against FP64 finite differences -------------------------------

def make_fd_case(torch, oracle, name):
    """A case under seeded motion; target = the motion-free reconstruction;
    the loss runs over voxels that every view samples >= 3 pixels inside the
    detector for the nominal geometry (motion of +/- 0.5 mm / 0.3 deg moves
    samples by < 1.5 pixel here, so no sample crosses the detector edge).
    mini_c2: the 40-view fixture; c4: the differentiation workload at full
    size (360 views of 512 x 512 -> 256^3 at 0.4 mm), its projections
    preprocessed by the oracle."""
    from fp64_fdk import all_points, case_from_workload, interior
    from jenhine_b200.autograd import FDKFunction
    from jenhine_b200.fdk import FDKEngine
    from jenhine_b200.motion import seeded_motion
    if name == "mini_c2":
        g = load_golden("mini_c2")
        e = engine_for(g)
    else:
        from jenhine_b200.workloads import c3
        w = c3()
        g = case_from_workload(w, w.raw_torch().cpu().numpy())
        g["prep"] = np.stack([oracle.preprocess(f, float(g["bright_field"]), tuple(g["bhc"])) for f in g["raw"]])
        e = FDKEngine(w.scan, w.recon, g["ptms"])
    X, Y, Z = (int(v) for v in g["vol"])
    P0 = g["ptms"].astype(np.float64)
    nv = g["raw"].shape[0]
    theta = seeded_motion(nv, 11)
    pts = all_points(X, Y, Z)
    mask = interior(g, pts, margin=3.0)
    p = to_dev(torch, g["prep"])
    target = FDKFunction.apply(p, torch.zeros((nv, 6), dtype=torch.float64), e, P0).detach().clone()
    mask_t = torch.from_numpy(mask.reshape(Z, Y, X)).cuda()
    return dict(g=g, P0=P0, theta=theta, pts=pts, mask=mask, mask_t=mask_t, e=e, p=p, target=target,
                X=X, Y=Y, Z=Z, nv=nv, name=name)


@pytest.fixture(scope="module", params=["mini_c2", "c4"])
def fd_case(torch_cuda, oracle, request):
    return make_fd_case(torch_cuda, oracle, request.param)


def gpu_gradients(torch, c):
    from jenhine_b200.autograd import FDKFunction
    p = c["p"].clone().requires_grad_(True)
    th = torch.tensor(c["theta"], dtype=torch.float64, requires_grad=True)
    vol = FDKFunction.apply(p, th, c["e"], c["P0"])
    loss = (torch.where(c["mask_t"], vol - c["target"], 0.0) ** 2).sum()
    loss.backward()
    return th.grad.numpy(), p.grad.cpu().numpy()


class FP64Loss:
    """L = sum over the mask of (vol - target)^2 in FP64.  The sums over all
    views are kept; a view's own sums are computed when its entry is varied,
    so that one view can be re-evaluated alone."""

    def __init__(self, oracle, c):
        from jenhine_b200.motion import moved_ptms
        g = c["g"]
        self.o, self.c = oracle, c
        W = g["prep"].shape[2]
        self.L = oracle.fft_length(W)
        self.H = oracle.filter_spectrum(self.L, float(g["hsr"]), *map(float, g["cut"]), g["adj_pts"], g["adj_db"])
        self.q = oracle.filter_projections_f64(g["prep"], g["ptms"], self.H, float(g["dso"]))
        self.uw = oracle.bp_uweights(g["ptms"], W)
        self.P = moved_ptms(c["P0"], c["theta"])
        self.pts = c["pts"][c["mask"]]
        self.target = c["target"].cpu().numpy().ravel()[c["mask"]].astype(np.float64)
        self.S, self.C = oracle.bp_points_f64d(self.q, self.P, self.uw, self.pts, c["X"], c["Y"], c["Z"],
                                               *map(float, c["g"]["pitch"]))

    def view_sums(self, v, P, qv):
        c = self.c
        return self.o.bp_points_f64d(qv[None], np.asarray(P, np.float64)[None], self.uw[v:v + 1], self.pts,
                                     c["X"], c["Y"], c["Z"], *map(float, c["g"]["pitch"]))

    def loss_with_view(self, v, P=None, qv=None):
        s0, c0 = self.view_sums(v, self.P[v], self.q[v])
        s, cc = self.view_sums(v, self.P[v] if P is None else P, self.q[v] if qv is None else qv)
        vol = (self.S - s0 + s) / (self.C - c0 + cc)
        return float(np.sum((vol - self.target) ** 2))


def fp64_loss(oracle, c):
    """The case's FP64Loss, made once (its filter and sums over all views take
    ~40 s at the c4 size)."""
    if "f64" not in c:
        c["f64"] = FP64Loss(oracle, c)
    return c["f64"]


def fd_report(c, what, got, fd):
    """Errors of the 32 entries: max error over the largest entry, and the
    median relative error over the entries whose difference quotient is not
    exactly zero."""
    err = np.abs(got - fd)
    scale = np.abs(fd).max()
    nz = fd != 0.0
    out = {"max_err_over_max": float(err.max() / scale), "median_rel": float(np.median(err[nz] / np.abs(fd[nz]))),
           "zero_entries": int(np.count_nonzero(~nz))}
    report(c["name"], what, out)
    print(c["name"], what, out)
    return err, scale


def test_geometry_gradient_vs_fp64_finite_differences(torch_cuda, oracle, fd_case):
    from jenhine_b200.motion import moved_ptms
    c = fd_case
    g_gpu, _ = gpu_gradients(torch_cuda, c)
    f = fp64_loss(oracle, c)
    rng = np.random.default_rng(12)
    entries = [(int(rng.integers(c["nv"])), int(rng.integers(6))) for _ in range(32)]
    h = 1e-3
    fd = []
    for v, j in entries:
        tp, tm = c["theta"][v].copy(), c["theta"][v].copy()
        tp[j] += h
        tm[j] -= h
        Pp = moved_ptms(c["P0"][v:v + 1], tp[None])[0]
        Pm = moved_ptms(c["P0"][v:v + 1], tm[None])[0]
        fd.append((f.loss_with_view(v, P=Pp) - f.loss_with_view(v, P=Pm)) / (2 * h))
    fd = np.array(fd)
    got = np.array([g_gpu[v, j] for v, j in entries])
    err, scale = fd_report(c, "geometry_gradient_fd", got, fd)
    assert scale > 0
    assert np.all(err <= 3e-3 * np.abs(fd) + 1e-3 * scale), list(zip(got, fd))


def test_projection_gradient_vs_fp64_finite_differences(torch_cuda, oracle, fd_case):
    c = fd_case
    _, p_grad = gpu_gradients(torch_cuda, c)
    f = fp64_loss(oracle, c)
    g = c["g"]
    rng = np.random.default_rng(13)
    h = 1e-2
    got, fd = [], []
    V, W = g["prep"].shape[1:]
    pw_cache = {}
    # entries on detector rows the masked voxels sample (elsewhere the
    # gradient is exactly zero)
    _, vr = oracle.points_survey(g["ptms"], f.pts, c["X"], c["Y"], c["Z"], *map(float, g["pitch"]), W, V)
    r_lo, r_hi = int(np.floor(vr[0])), int(np.floor(vr[1])) + 1
    for _ in range(32):
        v, r, i = int(rng.integers(c["nv"])), int(rng.integers(r_lo, r_hi + 1)), int(rng.integers(W))
        s = oracle.preweight_source_view(v, c["nv"])
        if s not in pw_cache:
            pw_cache[s] = oracle.preweight_for_view(g["ptms"][s], float(g["dso"]), W, V)
        vals, steps = [], []
        for sign in (1.0, -1.0):
            row = g["prep"][v, r].astype(np.float32).copy()
            base = float(row[i])
            row[i] = np.float32(base + sign * h)
            steps.append(abs(float(row[i]) - base))      # the step as stored in float
            qv = f.q[v].copy()
            qv[r] = oracle.filter_rows_f64(row[None], f.H, f.L, W, False, pw_cache[s][r:r + 1])[0]
            vals.append(f.loss_with_view(v, qv=qv))
        fd.append((vals[0] - vals[1]) / (steps[0] + steps[1]))
        got.append(p_grad[v, r, i])
    got, fd = np.array(got), np.array(fd)
    err, scale = fd_report(c, "projection_gradient_fd", got, fd)
    assert scale > 0
    assert np.all(err <= 1e-3 * np.abs(fd) + 2e-4 * scale), list(zip(got, fd))
