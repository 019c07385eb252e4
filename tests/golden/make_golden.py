"""Generate tests/golden/*.npz from the reference's own Core classes.

Runs the JEngine PreProcessingCore / PreFilterWeightGenerator / FilterCore /
BPCore / CTNumCore compiled from source (oracle/_ref, built by
oracle/build.py with the project's IPP/MKL shims) on small seeded inputs and
stores inputs and outputs.  The GPU parity tests and the CPU oracle tests read
these files; nothing at test time needs the reference tree.

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from jenhine_b200.phantom import ScanGeometry, line_integrals, random_phantom, raw_frames  # noqa: E402
from oracle.pyoracle import RefCores  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# Small cases of the two benchmark geometries (same orbit and magnification,
# fewer views, coarser detector and volume so each file stays small).
CASES = {
    "mini_c1": dict(geom=dict(n_views=36, sid=500.0, sdd=800.0, det_u=48, det_v=40, pixel_u=2.0,
                              pixel_v=2.0, seed=11),
                    vol=(24, 24, 20, 2.5, 2.5), phantom=dict(n=10), i0=1e5, bf=50000.0,
                    bhc=(1.0, 0.0, 0.0), norm=(1.2, 1.0)),
    "mini_c2": dict(geom=dict(n_views=40, sid=500.0, sdd=800.0, det_u=56, det_v=44, pixel_u=2.6,
                              pixel_v=2.6, flex_shift_px=0.5, flex_tilt_deg=0.2, seed=22),
                    vol=(32, 32, 24, 2.5, 2.5), phantom=dict(n=20, n_metal=3), i0=5e4,
                    bf=50000.0, bhc=(1.0, 0.05, 0.01), norm=(1.2, 0.9),
                    filt=dict(cut_start=0.0, cut_end=0.0, adj_pts=(0.05, 0.1), adj_db=(1.0, -1.0))),
    # offset detector (principal point 10 columns from its left edge) read
    # with conjugate-view compositing, as the reference application does
    # (CompositeAgent before a 2W-wide, mirrored FilterAgent)
    "mini_comp": dict(geom=dict(n_views=40, sid=500.0, sdd=800.0, det_u=48, det_v=36, pixel_u=2.6,
                                pixel_v=2.6, offset_u_px=-13.0, seed=44),
                      vol=(32, 32, 20, 2.5, 2.5), phantom=dict(n=10), i0=1e5, bf=50000.0,
                      bhc=(1.0, 0.0, 0.0), norm=(1.0, 1.0), composite=dict(det_right=True)),
    # ragged sizes: an odd detector (33 x 17), a view count that is not a
    # multiple of the 9-view pre-weight group, a volume that fills no BP tile
    # (13 x 37 x 5 against tiles of 4 x 32 x 8)
    "mini_odd": dict(geom=dict(n_views=11, sid=500.0, sdd=800.0, det_u=33, det_v=17, pixel_u=2.6,
                               pixel_v=2.6, flex_shift_px=0.5, flex_tilt_deg=0.2, seed=55),
                     vol=(13, 37, 5, 1.4, 2.5), phantom=dict(n=8, n_metal=1), i0=5e4, bf=50000.0,
                     bhc=(1.0, 0.05, 0.01), norm=(1.2, 0.9)),
    # orbit plane tilted 15 deg about x: the projection matrices' P[10] is
    # not zero, so W depends on z (the backprojectors' W(z) instantiations)
    "mini_tilt": dict(geom=dict(n_views=24, sid=500.0, sdd=800.0, det_u=40, det_v=36, pixel_u=2.6,
                                pixel_v=2.6, flex_shift_px=0.5, gantry_tilt_deg=15.0, seed=66),
                      vol=(24, 24, 16, 2.5, 2.5), phantom=dict(n=10, n_metal=1), i0=5e4, bf=50000.0,
                      bhc=(1.0, 0.0, 0.0), norm=(1.0, 1.0)),
}


def make(name: str, c: dict, ref: RefCores) -> str:
    g = ScanGeometry(**c["geom"])
    X, Y, Z, pxy, pz = c["vol"]
    ph = random_phantom(c["geom"]["seed"] + 1, (X * pxy, Y * pxy, Z * pz), **c["phantom"])
    raw = raw_frames(line_integrals(g, ph), c["geom"]["seed"] + 2, i0=c["i0"], bright_field=c["bf"])
    ptms = g.ptms()
    dso = np.float32(g.sid)
    hsr = g.half_sample_rate
    f = c.get("filt", {})
    prep = ref.preprocess(raw, c["bf"], c["bhc"])
    comp = c.get("composite")
    extra = {}
    if comp:   # CompositeCore, then the 2W-wide FilterCore (mirrored when the detector is on the right)
        cmp_ = ref.composite(prep, ptms, float(dso), comp["det_right"], nthreads=4)
        filt = ref.filter(cmp_, ptms, hsr, float(dso), f.get("cut_start", 0.0), f.get("cut_end", 0.0),
                          f.get("adj_pts", ()), f.get("adj_db", ()), mirror=comp["det_right"], w_out=g.det_u,
                          nthreads=4)
        extra = dict(comp=cmp_, det_right=np.int32(comp["det_right"]))
    else:
        filt = ref.filter(prep, ptms, hsr, float(dso), f.get("cut_start", 0.0), f.get("cut_end", 0.0),
                          f.get("adj_pts", ()), f.get("adj_db", ()), nthreads=4)
    bp = ref.bp(filt, ptms, X, Y, Z, pxy, pz, nthreads=4)
    hu = ref.ctnum(bp, *c["norm"])
    pw0 = ref.preweight(ptms, g.det_u, g.det_v, float(dso), 4)
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(
        path, raw=raw, ptms=ptms, dso=dso, hsr=np.float32(hsr), bright_field=np.float32(c["bf"]),
        bhc=np.asarray(c["bhc"], np.float32), vol=np.asarray([X, Y, Z], np.int32),
        pitch=np.asarray([pxy, pz], np.float32), norm=np.asarray(c["norm"], np.float32),
        cut=np.asarray([f.get("cut_start", 0.0), f.get("cut_end", 0.0)], np.float32),
        adj_pts=np.asarray(f.get("adj_pts", ()), np.float32),
        adj_db=np.asarray(f.get("adj_db", ()), np.float32),
        prep=prep, preweight_v4=pw0, filt=filt, bp=bp, hu=hu, **extra)
    return path


def main(names=None) -> None:
    ref = RefCores()
    for name, c in CASES.items():
        if names and name not in names:
            continue
        print(make(name, c, ref))


if __name__ == "__main__":
    main(sys.argv[1:])
