"""The benchmark workloads, each a seeded synthetic scan.

c1  plain FDK, CPU-runnable: 360 views over 360 deg, SID 500 mm, SDD 800 mm,
    256 x 256 detector at 0.5 mm, 10-ellipsoid phantom (mu 0-0.05 /mm),
    I0 = 1e5 Poisson noise, per-pixel gain 1 +/- 0.05 and offset 0-50 in the
    raw data, 128^3 volume at 0.5 mm.
c2  dental-CBCT size, plain FP32: 600 views over 360 deg, 768 x 768 detector
    at 0.2 mm, 640 x 640 x 480 volume at 0.125 mm, per-view flexmap
    (+/- 0.5 px detector shift, +/- 0.2 deg tilt), 20 ellipsoids plus 3
    metal inserts (mu 0.5 /mm), I0 = 5e4.  The orbit is not given for this
    case; it uses c1's SID 500 mm / SDD 800 mm.
c3  differentiation: 360 views of 512 x 512 at 0.5 mm -> 256^3 at 0.4 mm
    (the detector pitch is not given for this case; 0.5 mm covers the volume).
c2_tilt  c2 with the orbit tilted 1 deg (P[10] != 0, as in calibrated
    projection matrices): the backprojectors' W(z) form.
batch  16 seeded scans of uneven size for the batched launch (batch()).
mini_*  reduced versions of c1 / c2 for parity tests.

The reference corrects gain with one scalar bright field
(PreProcessingAgent/GainCorr.cpp:10-13); the per-pixel gain and offset are
properties of the synthetic detector, left in the raw frames.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .fdk import ReconConfig, ScanConfig
from .phantom import ScanGeometry, random_phantom


@dataclasses.dataclass
class Workload:
    name: str
    geom: ScanGeometry
    recon: ReconConfig
    n_ellipsoids: int
    n_metal: int
    i0: float
    bright_field: float = 50000.0
    gain_spread: float = 0.05
    offset_max: float = 50.0
    beam_hardening: tuple = (1.0, 0.0, 0.0)
    composite: bool = False        # offset detector read with conjugate-view compositing
    detector_on_right: bool = True

    @property
    def scan(self) -> ScanConfig:
        g = self.geom
        sc = ScanConfig(num_views=g.n_views, dso=g.sid, dsd=g.sdd, num_dets_u=g.det_u,
                        num_dets_v=g.det_v, detector_pixel_size=g.pixel_u,
                        bright_field=self.bright_field, beam_hardening=self.beam_hardening)
        if self.composite:   # the 2W-wide, mirrored filter input the compositing stage builds
            sc.filter_input_width = 2 * g.det_u
            sc.detector_on_right = self.detector_on_right
        return sc

    def phantom(self):
        r = self.recon
        extent = (r.num_pixels_x * r.pitch_xy, r.num_pixels_y * r.pitch_xy, r.num_pixels_z * r.pitch_z)
        return random_phantom(self.geom.seed + 1, extent, self.n_ellipsoids, n_metal=self.n_metal)

    @property
    def updates(self) -> int:
        """Voxel-view updates of one reconstruction (the GUPS numerator)."""
        r = self.recon
        return r.num_pixels_x * r.num_pixels_y * r.num_pixels_z * self.geom.n_views

    def raw_numpy(self):
        from .phantom import line_integrals, raw_frames
        return raw_frames(line_integrals(self.geom, self.phantom()), self.geom.seed + 2, i0=self.i0,
                          bright_field=self.bright_field, gain_spread=self.gain_spread,
                          offset_max=self.offset_max)

    def raw_torch(self, device="cuda"):
        from .phantom import raw_frames_torch
        return raw_frames_torch(self.geom, self.phantom(), self.geom.seed + 2, self.i0, self.bright_field,
                                self.gain_spread, self.offset_max, device=device)


def c1() -> Workload:
    return Workload("c1", ScanGeometry(360, 500.0, 800.0, 256, 256, 0.5, 0.5, seed=101),
                    ReconConfig(128, 128, 128, 0.5, 0.5, ct_norm0=1.0, ct_norm1=1.0), 10, 0, 1e5)


def c2() -> Workload:
    return Workload("c2", ScanGeometry(600, 500.0, 800.0, 768, 768, 0.2, 0.2, flex_shift_px=0.5,
                                       flex_tilt_deg=0.2, seed=202),
                    ReconConfig(640, 640, 480, 0.125, 0.125, ct_norm0=1.0, ct_norm1=1.0), 20, 3, 5e4)


def c3() -> Workload:
    """Differentiation: 360 views of 512 x 512 (0.5 mm) -> 256^3 at 0.4 mm,
    10-ellipsoid phantom; per-view rigid motion (jenhine_b200.motion) of
    +/- 0.5 mm / +/- 0.3 deg is the geometry the gradient is taken at."""
    return Workload("c3", ScanGeometry(360, 500.0, 800.0, 512, 512, 0.5, 0.5, seed=303),
                    ReconConfig(256, 256, 256, 0.4, 0.4, ct_norm0=1.0, ct_norm1=1.0), 10, 0, 1e5)


BATCH_VOLUMES = ((128, 128, 128), (256, 256, 256), (384, 384, 256), (512, 512, 400))
BATCH_VIEWS = (180, 360, 600, 720)
BATCH_DETECTORS = (256, 512, 768, 1024)


def batch(n: int = 16, seed: int = 404) -> list:
    """Batching: n scans of uneven size, each drawn by seed -- volume from
    BATCH_VOLUMES, views from BATCH_VIEWS, square detector from
    BATCH_DETECTORS, SID 450-600 mm, SDD 700-900 mm.  The detector is 200 mm
    wide (pixel = 200 / width mm) and the volume 100 mm across in x and y
    (cubic voxels); neither is given for this case.  10-ellipsoid phantoms."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        X, Y, Z = BATCH_VOLUMES[rng.integers(len(BATCH_VOLUMES))]
        views = int(BATCH_VIEWS[rng.integers(len(BATCH_VIEWS))])
        det = int(BATCH_DETECTORS[rng.integers(len(BATCH_DETECTORS))])
        sid = float(rng.uniform(450.0, 600.0))
        sdd = float(rng.uniform(700.0, 900.0))
        pix = 200.0 / det
        vox = 100.0 / X
        out.append(Workload(f"batch{i}", ScanGeometry(views, sid, sdd, det, det, pix, pix, seed=seed * 100 + i),
                            ReconConfig(X, Y, Z, vox, vox, ct_norm0=1.0, ct_norm1=1.0), 10, 0, 1e5))
    return out


def c2_slab() -> Workload:
    """c2's scan backprojected into a 16-slice central slab (profiling case:
    same projections and kernels, 1/30 of the volume)."""
    w = c2()
    w.name = "c2_slab"
    w.recon.num_pixels_z = 16
    return w


def c2_chunks() -> Workload:
    """c2's detector, orbit and voxels with 96 views (three 32-view chunks)
    into a 16-slice slab: the per-chunk kernels (preprocess + pre-weight,
    ramp product, packing) at c2's sizes with ~1.2 GB on the device, for
    multi-pass profiling."""
    w = c2()
    w.name = "c2_chunks"
    w.geom.n_views = 96
    w.recon.num_pixels_z = 16
    return w


def c2_offset() -> Workload:
    """c2 with an offset detector: the principal point 100 columns from the
    detector's left edge, read with conjugate-view compositing (2 x 768-wide
    filter input) and the z-filter, as the reference application's offset
    scans run (CompositeAgent, FilterAgent, ZFilterAgent)."""
    w = c2()
    w.name = "c2_offset"
    w.geom.offset_u_px = 100.0 - (w.geom.det_u / 2.0 - 1.0)
    w.composite = True
    w.recon.z_filter = True
    return w


def c2_offset_chunks() -> Workload:
    """c2_offset with 96 views into a 16-slice slab (multi-pass profiling of
    the compositing filter stage at c2's frame size)."""
    w = c2_offset()
    w.name = "c2_offset_chunks"
    w.geom.n_views = 96
    w.recon.num_pixels_z = 16
    return w


def c2_tilt() -> Workload:
    """c2 with the orbit plane tilted 1 deg about x.  Projection matrices
    from a calibration, like these, have P[10] != 0: W then depends on z and
    the backprojectors take their W(z) form (a reciprocal per sample)."""
    w = c2()
    w.name = "c2_tilt"
    w.geom.gantry_tilt_deg = 1.0
    return w


def mini_c1() -> Workload:
    return Workload("mini_c1", ScanGeometry(48, 500.0, 800.0, 64, 56, 2.0, 2.0, seed=5),
                    ReconConfig(40, 40, 32, 1.6, 1.6, ct_norm0=1.2, ct_norm1=1.0), 10, 0, 1e5)


def mini_c2() -> Workload:
    return Workload("mini_c2", ScanGeometry(60, 500.0, 800.0, 96, 80, 1.6, 1.6, flex_shift_px=0.5,
                                            flex_tilt_deg=0.2, seed=6),
                    ReconConfig(64, 64, 48, 1.25, 1.25, ct_norm0=1.2, ct_norm1=0.9), 20, 3, 5e4,
                    beam_hardening=(1.0, 0.05, 0.01))


WORKLOADS = {"c1": c1, "c2": c2, "c2_slab": c2_slab, "c2_chunks": c2_chunks, "c2_offset": c2_offset,
             "c2_offset_chunks": c2_offset_chunks, "c2_tilt": c2_tilt, "c3": c3, "mini_c1": mini_c1, "mini_c2": mini_c2}
