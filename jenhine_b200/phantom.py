"""Seeded synthetic cone-beam data: geometry, ellipsoid phantoms, raw frames.

There is no public dataset for this path; every workload is generated from a
seed.  Geometry is composed in FP64 and rounded to the FP32 3x4 projection
matrices (PTMs) the engine and the reference consume.

PTM convention (the one the reference's BPCore assumes, BPAgent/BPCore.cpp:
207-220): P maps world (x, y, z, 1) in mm to (u*w, v*w, w), and the detector
sample read for that point is index (u + 0.5, v + 0.5).  Pixel (i, j) of a
frame therefore sits at PTM coordinates (i - 0.5, j - 0.5).  P is scaled so
that P[11] == 1, like the reference's calibrated matrices.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class ScanGeometry:
    """Circular cone-beam orbit around the z axis, or around z tilted about x
    by gantry_tilt_deg."""
    n_views: int
    sid: float            # source to isocentre (DSO), mm
    sdd: float            # source to detector (DSD), mm
    det_u: int            # detector columns
    det_v: int            # detector rows
    pixel_u: float        # mm
    pixel_v: float        # mm
    arc_deg: float = 360.0
    start_deg: float = 0.0
    flex_shift_px: float = 0.0   # seeded per-view detector shift, +/- px
    flex_tilt_deg: float = 0.0   # seeded per-view in-plane detector tilt, +/- deg
    seed: int = 0
    offset_u_px: float = 0.0     # detector offset: the principal point moves by this many columns
    gantry_tilt_deg: float = 0.0  # orbit plane tilted about the x axis: W then depends on z (P[10] != 0)

    @property
    def half_sample_rate(self) -> float:
        """Config/ConfigHelper.cpp:52-53: 0.5 / (pixel * DSO / DSD), in float."""
        det_at_iso = np.float32(self.pixel_u) / np.float32(self.sdd) * np.float32(self.sid)
        return float(np.float32(0.5) * (np.float32(1.0) / det_at_iso))

    def frames(self):
        """Per-view (source, n_hat, e_u, e_v, cu, cv) in FP64."""
        rng = np.random.default_rng(self.seed + 7919)
        shift = rng.uniform(-1.0, 1.0, size=(self.n_views, 2)) * self.flex_shift_px
        tilt = np.deg2rad(rng.uniform(-1.0, 1.0, size=self.n_views) * self.flex_tilt_deg)
        out = []
        for k in range(self.n_views):
            b = math.radians(self.start_deg + self.arc_deg * k / self.n_views)
            c, s = math.cos(b), math.sin(b)
            src = np.array([self.sid * c, self.sid * s, 0.0])
            n_hat = np.array([-c, -s, 0.0])
            eu0 = np.array([-s, c, 0.0])
            ev0 = np.array([0.0, 0.0, 1.0])
            ct, st = math.cos(tilt[k]), math.sin(tilt[k])
            eu = ct * eu0 + st * ev0
            ev = -st * eu0 + ct * ev0
            cu = self.det_u / 2.0 - 1.0 + shift[k, 0] + self.offset_u_px
            cv = self.det_v / 2.0 - 1.0 + shift[k, 1]
            if self.gantry_tilt_deg:
                g = math.radians(self.gantry_tilt_deg)
                Rx = np.array([[1.0, 0.0, 0.0], [0.0, math.cos(g), -math.sin(g)], [0.0, math.sin(g), math.cos(g)]])
                src, n_hat, eu, ev = Rx @ src, Rx @ n_hat, Rx @ eu, Rx @ ev
            out.append((src, n_hat, eu, ev, cu, cv))
        return out

    def ptms_f64(self) -> np.ndarray:
        P = np.zeros((self.n_views, 12), np.float64)
        for k, (src, n_hat, eu, ev, cu, cv) in enumerate(self.frames()):
            r2 = np.concatenate([n_hat, [-src @ n_hat]])
            r0 = (self.sdd / self.pixel_u) * np.concatenate([eu, [-src @ eu]]) + cu * r2
            r1 = (self.sdd / self.pixel_v) * np.concatenate([ev, [-src @ ev]]) + cv * r2
            m = np.concatenate([r0, r1, r2])
            P[k] = m / m[11]
        return P

    def ptms(self) -> np.ndarray:
        return self.ptms_f64().astype(np.float32)

    def rays(self, k: int):
        """The source of view k and its unit ray directions [V][U][3] (FP64)."""
        src, n_hat, eu, ev, cu, cv = self.frames()[k]
        a = (np.arange(self.det_u) - 0.5 - cu) * self.pixel_u
        b = (np.arange(self.det_v) - 0.5 - cv) * self.pixel_v
        d = (self.sdd * n_hat[None, None, :] + a[None, :, None] * eu[None, None, :]
             + b[:, None, None] * ev[None, None, :])
        d /= np.linalg.norm(d, axis=-1, keepdims=True)
        return src, d


@dataclasses.dataclass
class Ellipsoid:
    center: np.ndarray     # mm
    axes: np.ndarray       # semi-axes, mm
    rot: np.ndarray        # 3x3, columns = ellipsoid axes in world
    mu: float              # additive attenuation, 1/mm


def random_phantom(seed: int, extent_mm, n: int = 10, mu_range=(0.0, 0.05),
                   n_metal: int = 0, metal_mu: float = 0.5):
    """A body ellipsoid filling ~80% of the volume plus n-1 seeded inner ones
    (mu drawn from mu_range) and n_metal small high-mu inserts."""
    rng = np.random.default_rng(seed)
    ex = np.asarray(extent_mm, np.float64) / 2.0
    out = [Ellipsoid(np.zeros(3), ex * np.array([0.8, 0.7, 0.85]), np.eye(3), 0.02)]

    def rot(rng):
        a, b, c = rng.uniform(0, 2 * math.pi, 3)
        Rz = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
        Rx = np.array([[1, 0, 0], [0, math.cos(b), -math.sin(b)], [0, math.sin(b), math.cos(b)]])
        Rz2 = np.array([[math.cos(c), -math.sin(c), 0], [math.sin(c), math.cos(c), 0], [0, 0, 1]])
        return Rz @ Rx @ Rz2

    for _ in range(n - 1):
        ctr = rng.uniform(-0.45, 0.45, 3) * ex
        axes = rng.uniform(0.05, 0.3, 3) * ex
        out.append(Ellipsoid(ctr, axes, rot(rng), float(rng.uniform(*mu_range))))
    for _ in range(n_metal):
        ctr = rng.uniform(-0.35, 0.35, 3) * ex
        axes = rng.uniform(0.01, 0.03, 3) * ex
        out.append(Ellipsoid(ctr, axes, rot(rng), metal_mu))
    return out


def line_integrals(geom: ScanGeometry, phantom, views=None) -> np.ndarray:
    """Analytic sum of mu * chord length per detector pixel, [nv][V][U] f64."""
    views = range(geom.n_views) if views is None else views
    res = []
    for k in views:
        src, d = geom.rays(k)
        acc = np.zeros(d.shape[:2])
        for e in phantom:
            Rt = e.rot.T / e.axes[:, None]
            q0 = Rt @ (src - e.center)
            q1 = d @ Rt.T
            A = np.einsum("...i,...i", q1, q1)
            B = q1 @ q0
            Cc = q0 @ q0 - 1.0
            disc = B * B - A * Cc
            acc += np.where(disc > 0, 2.0 * np.sqrt(np.maximum(disc, 0.0)) / A, 0.0) * e.mu
        res.append(acc)
    return np.stack(res)


def raw_frames_torch(geom: ScanGeometry, phantom, seed: int, i0: float, bright_field: float,
                     gain_spread: float = 0.0, offset_max: float = 0.0, device="cuda",
                     views_per_batch: int = 8):
    """Same data path as line_integrals + raw_frames, evaluated with torch on
    the GPU (FP64 geometry) for the full-size workloads; returns a uint16
    tensor [n_views][V][U] on `device`."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed + 104729)
    shape = (geom.det_v, geom.det_u)
    gain = 1.0 + (torch.rand(shape, generator=g, device=device, dtype=torch.float64) * 2 - 1) * gain_spread
    off = torch.rand(shape, generator=g, device=device, dtype=torch.float64) * offset_max
    frames = geom.frames()
    out = torch.empty((geom.n_views,) + shape, dtype=torch.uint16, device=device)
    ell = [(torch.tensor(e.rot.T / e.axes[:, None], device=device), torch.tensor(e.center, device=device), e.mu)
           for e in phantom]
    a_idx = torch.arange(geom.det_u, device=device, dtype=torch.float64)
    b_idx = torch.arange(geom.det_v, device=device, dtype=torch.float64)
    for k0 in range(0, geom.n_views, views_per_batch):
        ks = range(k0, min(geom.n_views, k0 + views_per_batch))
        src = torch.tensor(np.stack([frames[k][0] for k in ks]), device=device)
        nh = torch.tensor(np.stack([frames[k][1] for k in ks]), device=device)
        eu = torch.tensor(np.stack([frames[k][2] for k in ks]), device=device)
        ev = torch.tensor(np.stack([frames[k][3] for k in ks]), device=device)
        cu = torch.tensor([frames[k][4] for k in ks], device=device, dtype=torch.float64)
        cv = torch.tensor([frames[k][5] for k in ks], device=device, dtype=torch.float64)
        a = (a_idx[None, :] - 0.5 - cu[:, None]) * geom.pixel_u            # [b][U]
        b = (b_idx[None, :] - 0.5 - cv[:, None]) * geom.pixel_v            # [b][V]
        d = (geom.sdd * nh[:, None, None, :] + a[:, None, :, None] * eu[:, None, None, :]
             + b[:, :, None, None] * ev[:, None, None, :])                # [b][V][U][3]
        d = d / torch.linalg.norm(d, dim=-1, keepdim=True)
        acc = torch.zeros(d.shape[:3], device=device, dtype=torch.float64)
        for Rt, ctr, mu in ell:
            q0 = (src - ctr) @ Rt.T                                        # [b][3]
            q1 = d @ Rt.T                                                  # [b][V][U][3]
            A = (q1 * q1).sum(-1)
            B = (q1 * q0[:, None, None, :]).sum(-1)
            Cc = (q0 * q0).sum(-1)[:, None, None] - 1.0
            disc = B * B - A * Cc
            acc += torch.where(disc > 0, 2.0 * torch.sqrt(disc.clamp_min(0)) / A, 0.0) * mu
        photons = torch.poisson(i0 * torch.exp(-acc), generator=g)
        adu = photons * (bright_field / i0) * gain + off
        out[k0:k0 + len(ks)] = torch.clamp(torch.round(adu), 0, 65535).to(torch.int32).to(torch.uint16)
    return out


def raw_frames(lint: np.ndarray, seed: int, i0: float = 1e5, bright_field: float = 50000.0,
               gain_spread: float = 0.0, offset_max: float = 0.0) -> np.ndarray:
    """uint16 detector frames: Poisson(i0 * exp(-lint)) photons scaled to ADU so
    that an unattenuated pixel reads bright_field, times a seeded per-pixel
    gain (1 +/- gain_spread) plus a seeded offset in [0, offset_max]."""
    rng = np.random.default_rng(seed + 104729)
    photons = rng.poisson(i0 * np.exp(-lint))
    shape = lint.shape[-2:]
    gain = 1.0 + rng.uniform(-gain_spread, gain_spread, shape)
    off = rng.uniform(0.0, offset_max, shape)
    adu = photons * (bright_field / i0) * gain + off
    return np.clip(np.rint(adu), 0, 65535).astype(np.uint16)
