"""FP64 FDK on the CPU, built from the oracle's double-precision pieces, for
stating the error of the engine's forms (rel-L2 and max HU).

Steps: preprocessing and the pre-weight table as the reference computes them
(float; identical input to every form), then the filter
(oracle.filter_rows_f64), the taper product, sample coordinates, lerps,
sums and CT numbers in double (oracle.bp_points_f64, ctnum_f64).  Voxels are
given as a list of (x, y, z) indices, so a large volume is checked on a
sample of its voxels.  Test infrastructure only."""
from __future__ import annotations

import json
import os

import numpy as np


def case_from_workload(w, raw_u16: np.ndarray) -> dict:
    """The keys of a golden case, for a benchmark workload."""
    r = w.recon
    return {
        "raw": raw_u16, "ptms": w.geom.ptms(), "dso": w.geom.sid, "hsr": w.geom.half_sample_rate,
        "bright_field": w.bright_field, "bhc": np.array(w.beam_hardening, np.float32),
        "vol": (r.num_pixels_x, r.num_pixels_y, r.num_pixels_z), "pitch": (r.pitch_xy, r.pitch_z),
        "norm": (r.ct_norm0, r.ct_norm1), "cut": (r.filter_cutoff_start, r.filter_cutoff_end),
        "adj_pts": np.array(r.adjust_points, np.float32), "adj_db": np.array(r.adjust_level_db, np.float32),
    }


def project_points(g: dict, pts: np.ndarray):
    """(u, v) of every point in every view, in double: arrays [views][n]."""
    X, Y, Z = (int(v) for v in g["vol"])
    pxy, pz = (float(v) for v in g["pitch"])
    P = np.asarray(g["ptms"], np.float64).reshape(-1, 3, 4)
    xyz1 = np.stack([(pts[:, 0] - (X - 1) / 2.0) * pxy, (pts[:, 1] - (Y - 1) / 2.0) * pxy,
                     (pts[:, 2] - (Z - 1) / 2.0) * pz, np.ones(len(pts))], 1)
    uvw = np.einsum("vij,nj->vin", P, xyz1)
    return uvw[:, 0] / uvw[:, 2] + 0.5, uvw[:, 1] / uvw[:, 2] + 0.5


def survey(g: dict, pts: np.ndarray, margin: float = 1.0):
    """(interior, vrange) of the points (oracle.points_survey, in double):
    interior[i] when every view samples point i at least `margin` pixels
    inside the detector; vrange the least and largest detector row (as
    floats) of the samples inside the detector, or None."""
    from oracle.pyoracle import Oracle
    X, Y, Z = (int(v) for v in g["vol"])
    pxy, pz = (float(v) for v in g["pitch"])
    V, U = g["raw"].shape[1:]
    return Oracle().points_survey(g["ptms"], pts, X, Y, Z, pxy, pz, U, V, margin)


def interior(g: dict, pts: np.ndarray, margin: float = 1.0) -> np.ndarray:
    """Points that every view samples at least `margin` pixels inside the
    detector: their sample set does not depend on how u, v are rounded."""
    return survey(g, pts, margin)[0]


def all_points(X: int, Y: int, Z: int, z0: int = 0, nz: int | None = None, stride: int = 1) -> np.ndarray:
    nz = Z - z0 if nz is None else nz
    z, y, x = np.meshgrid(np.arange(z0, z0 + nz), np.arange(0, Y, stride), np.arange(0, X, stride), indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.int32)


def fdk_f64(oracle, g: dict, pts: np.ndarray) -> np.ndarray:
    """HU (double) of the points."""
    raw = g["raw"]
    nv, Hh, W = raw.shape
    X, Y, Z = (int(v) for v in g["vol"])
    pxy, pz = (float(v) for v in g["pitch"])
    # detector rows the points sample (+1 for the lower neighbour)
    band = survey(g, pts)[1]
    r0 = max(int(np.floor(band[0])) - 1, 0) if band else 0
    r1 = min(int(np.floor(band[1])) + 3, Hh) if band else Hh
    pre = np.stack([oracle.preprocess(raw[i], float(g["bright_field"]), tuple(g["bhc"])) for i in range(nv)])
    L = oracle.fft_length(W)
    H = oracle.filter_spectrum(L, float(g["hsr"]), float(g["cut"][0]), float(g["cut"][1]), g["adj_pts"],
                               g["adj_db"])
    filt = oracle.filter_projections_f64(pre, g["ptms"], H, float(g["dso"]), rows=(r0, r1))
    s, c = oracle.bp_points_f64(filt, g["ptms"], pts, X, Y, Z, pxy, pz, row0=r0, det_rows=Hh)
    with np.errstate(invalid="ignore", divide="ignore"):
        mu = s / c
    return oracle.ctnum_f64(mu, float(g["norm"][0]), float(g["norm"][1]))


def errors(hu: np.ndarray, ref: np.ndarray, inside: np.ndarray) -> dict:
    """rel-L2 of the attenuation (HU + 1000) and max |dHU|, over the interior
    voxels and over all voxels both volumes see."""
    hu = np.asarray(hu, np.float64)
    both = np.isfinite(hu) & np.isfinite(ref)
    d = np.abs(hu - ref)

    def rl2(m):
        a, b = hu[m] + 1000.0, ref[m] + 1000.0
        return float(np.linalg.norm(a - b) / np.linalg.norm(b)) if m.any() else 0.0

    return {
        "rel_l2_interior": rl2(both & inside),
        "rel_l2_all": rl2(both),
        "max_hu_interior": float(d[both & inside].max()) if (both & inside).any() else 0.0,
        "max_hu_all": float(d[both].max()) if both.any() else 0.0,
        "seen_mismatch": int(np.count_nonzero(np.isfinite(hu) != np.isfinite(ref))),
        "voxels": int(hu.size),
        "interior_voxels": int(np.count_nonzero(inside)),
    }


def report(name: str, form: str, err: dict) -> None:
    """Append a JSON line to $JFDK_ERROR_REPORT when it is set."""
    path = os.environ.get("JFDK_ERROR_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"case": name, "form": form, **err}) + "\n")
