"""ctypes bindings for the parity oracles (TEST INFRASTRUCTURE ONLY).

``Oracle`` wraps ``libjfdk_oracle.so`` (the C restatement, fdk_oracle.c).
``RefCores`` wraps ``_ref/libjref.so`` (the reference's own Core classes
compiled from source with IPP/MKL shims); it is absent where the reference
tree was never available to build it.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module.  The engine in ``jenhine_b200`` never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build  # noqa: F401  (package-relative when imported as oracle.pyoracle)

HERE = os.path.dirname(os.path.abspath(__file__))

_f32 = np.float32
_P = C.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Oracle:
    """FP32 restatement of the reference hot path plus its FP64 twin."""

    def __init__(self, path: str | None = None):
        path = path or _build.build_oracle()
        self.lib = C.CDLL(path)
        L = self.lib
        I, F = C.c_int, C.c_float
        sig = {
            "jo_ptm_move_u": [_P, F], "jo_ptm_move_v": [_P, F], "jo_ptm_reverse_x": [_P],
            "jo_ptm_reverse_y": [_P], "jo_ptm_move_z": [_P, F], "jo_ptm2tm": [_P, _P, F],
            "jo_solve_f32": [I, I, _P, _P], "jo_solve_f64": [I, I, _P, _P],
            "jo_preprocess": [_P, _P, I, I, I, I, I, I, I, I, F, _P],
            "jo_preweight_generate": [_P, _P, I, I, I],
            "jo_preweight_for_view": [_P, _P, F, I, I, I],
            "jo_preweight_source_view": [I, I], "jo_fft_length": [I],
            "jo_rfft_forward": [_P, _P, I], "jo_rfft_backward": [_P, _P, I],
            "jo_filter_spectrum": [_P, I, F, F, F, _P, _P, I],
            "jo_filter_rows": [_P, _P, _P, I, I, I, I, _P, I],
            "jo_filter_rows_f64": [_P, _P, _P, I, I, I, I, _P, I],
            "jo_composite": [_P, _P, _P, _P, _P, F, I, I, I],
            "jo_bp_points_f64": [_P, _P, _P, _P, _P, I, I, I, I, _P, I, I, I, I, F, F, I],
            "jo_bp_points_f64d": [_P, _P, _P, _P, _P, I, I, I, I, _P, I, I, I, I, F, F, I],
            "jo_points_survey": [_P, _P, _P, I, _P, I, I, I, I, C.c_double, C.c_double, I, I, C.c_double, I],
            "jo_filter_kernel_f64": [_P, _P, I], "jo_bp_uweights": [_P, _P, I, I],
            "jo_bp_accumulate": [_P, _P, _P, _P, _P, I, I, I, I, I, I, I, F, F, I, I, I],
            "jo_bp_accumulate_f64": [_P, _P, _P, _P, _P, I, I, I, I, I, I, I, F, F, I, I, I],
            "jo_bp_finalize": [_P, _P, _P, C.c_size_t],
            "jo_ctnum": [_P, C.c_size_t, F, F, F], "jo_to_int16": [_P, _P, C.c_size_t],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = I if name in ("jo_solve_f32", "jo_solve_f64", "jo_preprocess",
                                       "jo_preweight_source_view", "jo_fft_length") else None

    # -- geometry -----------------------------------------------------------
    def ptm_modify(self, ptm, op: str, a: float = 0.0) -> np.ndarray:
        p = _c(ptm, _f32).copy()
        fn = {"move_u": self.lib.jo_ptm_move_u, "move_v": self.lib.jo_ptm_move_v,
              "move_z": self.lib.jo_ptm_move_z}.get(op)
        if fn is not None:
            fn(_ptr(p), a)
        elif op == "reverse_x":
            self.lib.jo_ptm_reverse_x(_ptr(p))
        elif op == "reverse_y":
            self.lib.jo_ptm_reverse_y(_ptr(p))
        else:
            raise ValueError(op)
        return p

    def ptm2tm(self, ptm, dso: float) -> np.ndarray:
        tm = np.zeros(16, _f32)
        self.lib.jo_ptm2tm(_ptr(tm), _ptr(_c(ptm, _f32)), dso)
        return tm

    def solve_f32(self, A, B):
        A = _c(A, _f32).copy(); B = _c(B, _f32).copy()
        m = A.shape[0]; p = B.shape[1] if B.ndim == 2 else 1
        info = self.lib.jo_solve_f32(m, p, _ptr(A), _ptr(B))
        if info:
            raise np.linalg.LinAlgError(f"singular pivot {info}")
        return B

    # -- preprocessing ------------------------------------------------------
    def preprocess(self, raw, bright_field, bhc=(1.0, 0.0, 0.0), borders=(0, 0, 0, 0)):
        raw = _c(raw, np.uint16)
        views = raw.reshape(-1, raw.shape[-2], raw.shape[-1])
        inH, inW = views.shape[1:]
        bu, bd, bl, br = borders
        outH, outW = inH - bu - bd, inW - bl - br
        out = np.empty((views.shape[0], outH, outW), _f32)
        b = np.asarray(bhc, _f32)
        for i in range(views.shape[0]):
            r = self.lib.jo_preprocess(_ptr(out[i]), _ptr(views[i]), inW, inH, bu, bd, bl, br,
                                       outW, outH, bright_field, _ptr(b))
            if r:
                raise ValueError("only the identity resize is restated")
        return out.reshape(raw.shape[:-2] + (outH, outW))

    # -- pre-weight ---------------------------------------------------------
    def fft_length(self, w: int) -> int:
        return self.lib.jo_fft_length(w)

    def preweight_for_view(self, ptm, dso, input_width, height, det_on_right=False):
        L = self.fft_length(input_width)
        w = np.empty((height, L), _f32)
        self.lib.jo_preweight_for_view(_ptr(w), _ptr(_c(ptm, _f32)), dso, input_width, height,
                                       int(det_on_right))
        return w

    def preweight_source_view(self, v, n):
        return self.lib.jo_preweight_source_view(v, n)

    # -- FFT / filter -------------------------------------------------------
    def rfft_forward(self, x):
        x = _c(x, _f32); n = x.size
        ccs = np.zeros(n // 2 * 2 + 2, _f32)
        self.lib.jo_rfft_forward(_ptr(ccs), _ptr(x), n)
        return ccs

    def rfft_backward(self, ccs, n):
        x = np.zeros(n, _f32)
        self.lib.jo_rfft_backward(_ptr(x), _ptr(_c(ccs, _f32)), n)
        return x

    def filter_spectrum(self, L, hsr, cut_start=0.0, cut_end=0.0, adj_pts=(), adj_db=()):
        H = np.zeros(L // 2 + 1, _f32)
        ap = _c(np.asarray(adj_pts, _f32).reshape(-1), _f32)
        ad = _c(np.asarray(adj_db, _f32).reshape(-1), _f32)
        self.lib.jo_filter_spectrum(_ptr(H), L, hsr, cut_start, cut_end, _ptr(ap), _ptr(ad), ap.size)
        return H

    def filter_kernel_f64(self, H, L):
        h = np.zeros(L, np.float64)
        self.lib.jo_filter_kernel_f64(_ptr(h), _ptr(_c(H, _f32)), L)
        return h

    def filter_rows(self, rows, H, L, w_out=None, mirror=False, preweight=None):
        rows = _c(rows, _f32)
        R, W = rows.reshape(-1, rows.shape[-1]).shape
        w_out = W if w_out is None else w_out
        out = np.empty((R, w_out), _f32)
        pw = None if preweight is None else _c(preweight, _f32)
        self.lib.jo_filter_rows(_ptr(out), _ptr(rows), None if pw is None else _ptr(pw), R, W,
                                w_out, int(mirror), _ptr(_c(H, _f32)), L)
        return out.reshape(rows.shape[:-1] + (w_out,))

    def composite(self, pre, ptms, dso, det_right, v0=0, nv=None):
        """The restated CompositeCore over views [v0, v0 + nv) of the
        rotation pre [N][H][W]: [nv][H][2W]."""
        pre = _c(pre, _f32)
        N, H, W = pre.shape
        ptms = _c(ptms, _f32).reshape(-1, 12)
        nv = N - v0 if nv is None else nv
        out = np.empty((nv, H, 2 * W), _f32)
        for i in range(nv):
            k = (v0 + i) % N
            kc = (k + N // 2) % N
            self.lib.jo_composite(_ptr(out[i]), _ptr(pre[k]), _ptr(pre[kc]), _ptr(ptms[k]), _ptr(ptms[kc]), dso, W,
                                  H, int(det_right))
        return out

    def filter_rows_f64(self, rows, H, L, w_out=None, mirror=False, preweight=None):
        rows = _c(rows, _f32)
        R, W = rows.reshape(-1, rows.shape[-1]).shape
        w_out = W if w_out is None else w_out
        out = np.empty((R, w_out), np.float64)
        pw = None if preweight is None else _c(preweight, _f32)
        self.lib.jo_filter_rows_f64(_ptr(out), _ptr(rows), None if pw is None else _ptr(pw), R, W,
                                    w_out, int(mirror), _ptr(_c(H, _f32)), L)
        return out.reshape(rows.shape[:-1] + (w_out,))

    def filter_projections_f64(self, proj, ptms, H, dso, mirror=False, rows=None):
        """FP64 FilterAgent over views 0..N-1 (9-view pre-weight grouping, the
        pre-weight table itself as the reference computes it), restricted to
        detector rows [rows[0], rows[1]) when given."""
        proj = _c(proj, _f32)
        V, Hh, W = proj.shape
        r0, r1 = (0, Hh) if rows is None else rows
        L = self.fft_length(W)
        out = np.empty((V, r1 - r0, W), np.float64)
        cache = {}
        for v in range(V):
            s = self.preweight_source_view(v, V)
            if s not in cache:
                cache.clear()
                cache[s] = self.preweight_for_view(ptms[s], dso, W, Hh, mirror)[r0:r1]
            out[v] = self.filter_rows_f64(proj[v, r0:r1], H, L, W, mirror, cache[s])
        return out

    def filter_projections(self, proj, ptms, H, dso, mirror=False, w_out=None):
        """FilterAgent over views 0..N-1: the 9-view pre-weight grouping;
        rows of width W in, w_out (default W) out."""
        proj = _c(proj, _f32)
        V, Hh, W = proj.shape
        w_out = W if w_out is None else w_out
        L = self.fft_length(W)
        out = np.empty((V, Hh, w_out), _f32)
        cache = {}
        for v in range(V):
            s = self.preweight_source_view(v, V)
            if s not in cache:
                cache.clear()
                cache[s] = self.preweight_for_view(ptms[s], dso, W, Hh, mirror)
            out[v] = self.filter_rows(proj[v], H, L, w_out, mirror, cache[s])
        return out

    # -- backprojection -----------------------------------------------------
    def bp_uweights(self, ptms, U):
        ptms = _c(ptms, _f32).reshape(-1, 12)
        w = np.empty((ptms.shape[0], U), _f32)
        self.lib.jo_bp_uweights(_ptr(w), _ptr(ptms), ptms.shape[0], U)
        return w

    def bp(self, proj, ptms, X, Y, Z, pitch_xy, pitch_z, z0=0, nz=None, nthreads=None,
           f64=False, return_parts=False):
        proj = _c(proj, _f32)
        nv, V, U = proj.shape
        ptms = _c(ptms, _f32).reshape(-1, 12)
        uw = self.bp_uweights(ptms, U)
        nz = Z - z0 if nz is None else nz
        nthreads = nthreads or os.cpu_count() or 1
        dt = np.float64 if f64 else _f32
        s = np.zeros((nz, Y, X), dt); c = np.zeros((nz, Y, X), dt)
        fn = self.lib.jo_bp_accumulate_f64 if f64 else self.lib.jo_bp_accumulate
        fn(_ptr(s), _ptr(c), _ptr(proj), _ptr(ptms), _ptr(uw), 0, nv, U, V, X, Y, Z,
           pitch_xy, pitch_z, z0, nz, nthreads)
        if return_parts:
            return s, c
        if f64:
            with np.errstate(invalid="ignore", divide="ignore"):
                return s / c
        out = np.empty_like(s)
        self.lib.jo_bp_finalize(_ptr(out), _ptr(s), _ptr(c), out.size)
        return out

    def bp_points_f64(self, proj, ptms, pts, X, Y, Z, pitch_xy, pitch_z, row0=0, det_rows=None,
                      nthreads=None):
        """FP64 backprojection of voxels pts[n][3] = (x, y, z).  proj holds
        detector rows [row0, row0 + proj.shape[1]) of a detector det_rows high
        (default: all rows given); a voxel that samples a row outside the
        given band raises.  Returns (sum, weight) per point."""
        proj = _c(proj, np.float64)
        nv, Vb, U = proj.shape
        det_rows = Vb if det_rows is None else det_rows
        ptms = _c(ptms, _f32).reshape(-1, 12)
        uw = self.bp_uweights(ptms, U)
        pts = _c(pts, np.int32).reshape(-1, 3)
        if row0 or Vb != det_rows:
            # embed the band in a full-height detector (zeros elsewhere) and
            # check that every sample used lies inside the band
            full = np.zeros((nv, det_rows, U), np.float64)
            full[:, row0:row0 + Vb] = proj
            self._check_band(ptms, pts, X, Y, Z, pitch_xy, pitch_z, U, det_rows, row0, row0 + Vb)
            proj = full
        s = np.zeros(len(pts), np.float64)
        c = np.zeros(len(pts), np.float64)
        self.lib.jo_bp_points_f64(_ptr(s), _ptr(c), _ptr(proj), _ptr(ptms), _ptr(uw), 0, nv, U,
                                  det_rows, _ptr(pts), len(pts), X, Y, Z, pitch_xy, pitch_z,
                                  nthreads or os.cpu_count() or 1)
        return s, c

    def bp_points_f64d(self, proj, ptms64, uw, pts, X, Y, Z, pitch_xy, pitch_z, nthreads=None):
        """FP64 backprojection of voxels pts with FP64 projection matrices
        ptms64 (n x 12) and a given u-taper uw (n x U, float32)."""
        proj = _c(proj, np.float64)
        nv, V, U = proj.shape
        pts = _c(pts, np.int32).reshape(-1, 3)
        s = np.zeros(len(pts), np.float64)
        c = np.zeros(len(pts), np.float64)
        self.lib.jo_bp_points_f64d(_ptr(s), _ptr(c), _ptr(proj), _ptr(_c(ptms64, np.float64)), _ptr(_c(uw, _f32)),
                                   0, nv, U, V, _ptr(pts), len(pts), X, Y, Z, pitch_xy, pitch_z,
                                   nthreads or os.cpu_count() or 1)
        return s, c

    def points_survey(self, ptms, pts, X, Y, Z, pitch_xy, pitch_z, U, V, margin=1.0, nthreads=None):
        """(interior, vrange) of voxels pts[n][3] in double: interior[i] when
        every view samples point i at least `margin` pixels inside the U x V
        detector; vrange = (least, largest) v over the samples inside the
        detector, or None when no sample is."""
        P = _c(np.asarray(ptms, np.float64).reshape(-1, 12), np.float64)
        pts = _c(pts, np.int32).reshape(-1, 3)
        inside = np.zeros(len(pts), np.uint8)
        vr = np.zeros(2, np.float64)
        self.lib.jo_points_survey(_ptr(inside), _ptr(vr), _ptr(pts), len(pts), _ptr(P), P.shape[0], X, Y, Z,
                                  float(pitch_xy), float(pitch_z), U, V, float(margin),
                                  nthreads or os.cpu_count() or 1)
        return inside.astype(bool), (None if vr[0] > vr[1] else (float(vr[0]), float(vr[1])))

    def _check_band(self, ptms, pts, X, Y, Z, pitch_xy, pitch_z, U, V, r0, r1):
        _, vr = self.points_survey(ptms, pts, X, Y, Z, pitch_xy, pitch_z, U, V)
        if vr is not None:
            lo, hi = np.floor(vr[0]), np.floor(vr[1]) + 1
            if lo < r0 or hi >= r1:
                raise ValueError(f"samples rows {lo:.0f}..{hi:.0f} outside [{r0}, {r1})")

    @staticmethod
    def ctnum_f64(mu, norm0, norm1, mu_water=0.02):
        """CTNumCore::Process in double."""
        h = np.asarray(mu, np.float64) * (norm0 * 1000.0 / mu_water) - 1000.0
        hi = h > 300.0
        h[hi] = np.minimum(8191.0, (h[hi] - 300.0) * norm1 + 300.0)
        return h

    # -- CT numbers ---------------------------------------------------------
    def ctnum(self, vol, norm0, norm1, mu_water=0.02):
        v = _c(vol, _f32).copy()
        self.lib.jo_ctnum(_ptr(v), v.size, norm0, norm1, mu_water)
        return v

    def to_int16(self, vol):
        v = _c(vol, _f32)
        o = np.empty(v.shape, np.int16)
        self.lib.jo_to_int16(_ptr(o), _ptr(v), v.size)
        return o


class RefCores:
    """The reference's Core classes compiled from source (oracle/_ref)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "_ref", "libjref.so")
        if not os.path.exists(path):
            path = _build.build_ref()
        if not path or not os.path.exists(path):
            raise FileNotFoundError("oracle/_ref/libjref.so is not built")
        self.lib = C.CDLL(path)
        I, F = C.c_int, C.c_float
        sig = {
            "jref_ptm2tm": [_P, _P, F], "jref_ptm_modify": [_P, I, F],
            "jref_preprocess": [_P, _P, I, I, I, I, I, I, I, I, I, F, _P, I],
            "jref_preweight": [_P, _P, I, I, I, I, F, I],
            "jref_filter": [_P, _P, I, I, I, I, I, F, F, F, _P, _P, I, _P, I, F, I],
            "jref_filter_rows_noweight": [_P, _P, I, I, I, I, F, F, F, _P, _P, I],
            "jref_bp": [_P, _P, _P, I, I, I, I, I, I, F, F, I],
            "jref_ctnum": [_P, I, I, I, F, F, F], "jref_fft_length": [I],
            "jref_composite": [_P, _P, I, I, _P, I, I, I, I, F, I],
        }
        for name, args in sig.items():
            fn = getattr(self.lib, name)
            fn.argtypes = args
            fn.restype = I

    def ptm2tm(self, ptm, dso):
        tm = np.zeros(16, _f32)
        self.lib.jref_ptm2tm(_ptr(tm), _ptr(_c(ptm, _f32)), dso)
        return tm

    def ptm_modify(self, ptm, op: str, a: float = 0.0):
        p = _c(ptm, _f32).copy()
        code = {"move_u": 0, "move_v": 1, "reverse_x": 2, "reverse_y": 3, "move_z": 4}[op]
        self.lib.jref_ptm_modify(_ptr(p), code, a)
        return p

    def preprocess(self, raw, bright_field, bhc=(1.0, 0.0, 0.0), borders=(0, 0, 0, 0), nthreads=1):
        raw = _c(raw, np.uint16)
        views = raw.reshape(-1, raw.shape[-2], raw.shape[-1])
        inH, inW = views.shape[1:]
        bu, bd, bl, br = borders
        outH, outW = inH - bu - bd, inW - bl - br
        out = np.empty((views.shape[0], outH, outW), _f32)
        self.lib.jref_preprocess(_ptr(out), _ptr(views), views.shape[0], inW, inH, bu, bd, bl, br,
                                 outW, outH, bright_field, _ptr(np.asarray(bhc, _f32)), nthreads)
        return out.reshape(raw.shape[:-2] + (outH, outW))

    def preweight(self, ptms, input_width, height, dso, view, det_on_right=False):
        ptms = _c(ptms, _f32).reshape(-1, 12)
        L = self.lib.jref_fft_length(input_width)
        w = np.empty((height, L), _f32)
        self.lib.jref_preweight(_ptr(w), _ptr(ptms), ptms.shape[0], input_width, height,
                                int(det_on_right), dso, view)
        return w

    def filter(self, proj, ptms, hsr, dso, cut_start=0.0, cut_end=0.0, adj_pts=(), adj_db=(),
               mirror=False, w_out=None, nthreads=1):
        proj = _c(proj, _f32)
        V, H, W = proj.shape
        w_out = W if w_out is None else w_out
        ptms = _c(ptms, _f32).reshape(-1, 12)
        out = np.empty((V, H, w_out), _f32)
        ap = _c(np.asarray(adj_pts, _f32).reshape(-1), _f32)
        ad = _c(np.asarray(adj_db, _f32).reshape(-1), _f32)
        self.lib.jref_filter(_ptr(out), _ptr(proj), V, W, H, w_out, int(mirror), hsr, cut_start,
                             cut_end, _ptr(ap), _ptr(ad), ap.size, _ptr(ptms), ptms.shape[0], dso,
                             nthreads)
        return out

    def composite(self, pre, ptms, dso, det_right, v0=0, nv=None, nthreads=1):
        """CompositeCore over views [v0, v0 + nv) of the rotation pre
        [N][H][W]: [nv][H][2W]."""
        pre = _c(pre, _f32)
        N, H, W = pre.shape
        nv = N - v0 if nv is None else nv
        out = np.empty((nv, H, 2 * W), _f32)
        self.lib.jref_composite(_ptr(out), _ptr(pre), v0, nv, _ptr(_c(ptms, _f32)), N, W, H, int(det_right),
                                dso, nthreads)
        return out

    def filter_rows_noweight(self, rows, hsr, cut_start=0.0, cut_end=0.0, adj_pts=(), adj_db=(),
                             mirror=False, w_out=None):
        rows = _c(rows, _f32)
        R, W = rows.shape
        w_out = W if w_out is None else w_out
        out = np.empty((R, w_out), _f32)
        ap = _c(np.asarray(adj_pts, _f32).reshape(-1), _f32)
        ad = _c(np.asarray(adj_db, _f32).reshape(-1), _f32)
        self.lib.jref_filter_rows_noweight(_ptr(out), _ptr(rows), R, W, w_out, int(mirror), hsr,
                                           cut_start, cut_end, _ptr(ap), _ptr(ad), ap.size)
        return out

    def bp(self, proj, ptms, X, Y, Z, pitch_xy, pitch_z, nthreads=None):
        proj = _c(proj, _f32)
        nv, V, U = proj.shape
        out = np.empty((Z, Y, X), _f32)
        self.lib.jref_bp(_ptr(out), _ptr(proj), _ptr(_c(ptms, _f32).reshape(-1, 12)), nv, U, V,
                         X, Y, Z, pitch_xy, pitch_z, nthreads or os.cpu_count() or 1)
        return out

    def ctnum(self, vol, norm0, norm1, mu_water=0.02):
        v = _c(vol, _f32).copy()
        Z = v.shape[0] if v.ndim == 3 else 1
        self.lib.jref_ctnum(_ptr(v), v.shape[-1], v.shape[-2], Z, norm0, norm1, mu_water)
        return v
