"""Python host API over libjfdk.so.

``FDKEngine`` mirrors the per-stage interface of the reference's agents:

=====================  ===========================================  ==============================
method                 reference                                    C ABI
=====================  ===========================================  ==============================
``preprocess``         PreProcessingCore::Process                   jfdk_preprocess_frames
``filter``             FilterAgent::ProcessTask / FilterCore         jfdk_filter_frames
``zfilter``            ZFilterAgent::ProcessTask                    jfdk_zfilter_frames
``bp_reset``           BPCUDACore::InitShot_Synced / BPCore::InitShot jfdk_bp_reset
``bp_accumulate``      BPCUDACore::DeployBackProj (BPCore semantics) jfdk_bp_accumulate
``finalize``           BPCore::DoneSlice (+ CTNumCore::Process)     jfdk_finalize
``ctnum``              CTNumCore::Process                           jfdk_ctnum
``reconstruct``        the whole Proj -> Slice pipeline             jfdk_reconstruct
=====================  ===========================================  ==============================

Device buffers are torch CUDA tensors (torch provides allocation and streams
only); every computation runs in libjfdk.so.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional, Sequence

import numpy as np

from . import _lib


@dataclasses.dataclass
class ScanConfig:
    """Config/ScanParams.h fields (snake case)."""
    num_views: int
    dso: float
    dsd: float
    num_dets_u: int
    num_dets_v: int
    detector_pixel_size: float
    border_up: int = 0
    border_down: int = 0
    border_left: int = 0
    border_right: int = 0
    bright_field: float = 50000.0
    beam_hardening: Sequence[float] = (1.0, 0.0, 0.0)
    half_sample_rate: float = 0.0       # 0: derived as Config/ConfigHelper.cpp:52-53
    detector_on_right: bool = False
    filter_input_width: int = 0          # 0: the used detector width


@dataclasses.dataclass
class ReconConfig:
    """Config/ReconParams.h fields (snake case)."""
    num_pixels_x: int
    num_pixels_y: int
    num_pixels_z: int
    pitch_xy: float
    pitch_z: float
    ct_norm0: float = 1.0
    ct_norm1: float = 1.0
    mu_water: float = 0.02
    filter_cutoff_start: float = 0.0
    filter_cutoff_end: float = 0.0
    adjust_points: Sequence[float] = ()
    adjust_level_db: Sequence[float] = ()
    z_filter: bool = False


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


class FDKEngine:
    """One reconstruction context (one CUDA stream) on the current device."""

    def __init__(self, scan: ScanConfig, recon: ReconConfig, ptms, precision: str = "fp32",
                 stream=None, bp_exact: bool = False, view_chunk: Optional[int] = None):
        self.lib = _lib.load()
        self.scan, self.recon = scan, recon
        self.ptms = np.ascontiguousarray(np.asarray(ptms, np.float32).reshape(-1, 12))
        if self.ptms.shape[0] != scan.num_views:
            raise ValueError("need one 3x4 projection matrix per view")
        sp = _lib.ScanParams()
        for f in ("num_views", "dso", "dsd", "num_dets_u", "num_dets_v", "detector_pixel_size",
                  "border_up", "border_down", "border_left", "border_right", "bright_field",
                  "half_sample_rate", "filter_input_width"):
            setattr(sp, f, getattr(scan, f))
        sp.beam_hardening[:] = [float(x) for x in scan.beam_hardening]
        sp.detector_on_right = int(bool(scan.detector_on_right))
        self._adj = (np.ascontiguousarray(recon.adjust_points, np.float32),
                     np.ascontiguousarray(recon.adjust_level_db, np.float32))
        if self._adj[0].size != self._adj[1].size:
            raise ValueError("adjust points and levels differ in length")
        rp = _lib.ReconParams()
        for f in ("num_pixels_x", "num_pixels_y", "num_pixels_z", "pitch_xy", "pitch_z", "ct_norm0",
                  "ct_norm1", "mu_water", "filter_cutoff_start", "filter_cutoff_end"):
            setattr(rp, f, getattr(recon, f))
        rp.num_adjust = self._adj[0].size
        fp = C.POINTER(C.c_float)
        rp.adjust_points = self._adj[0].ctypes.data_as(fp)
        rp.adjust_level_db = self._adj[1].ctypes.data_as(fp)
        rp.z_filter = int(bool(recon.z_filter))
        prec = {"fp32": _lib.PRECISION_FP32, "mixed": _lib.PRECISION_MIXED}[precision]
        if stream is None:
            # bind to torch's current stream so torch copies and the engine's
            # kernels are ordered (0 is the legacy default stream)
            import torch
            stream = torch.cuda.current_stream().cuda_stream if torch.cuda.is_available() else 0
        self.stream_handle = int(stream)
        ctx = C.c_void_p()
        st = self.lib.jfdk_create(C.byref(ctx), C.byref(sp), C.byref(rp),
                                  self.ptms.ctypes.data_as(C.c_void_p), prec,
                                  C.c_void_p(self.stream_handle) if self.stream_handle else None)
        if st != _lib.JFDK_OK:
            msg = self.lib.jfdk_last_error(ctx).decode() if ctx.value else ""
            if ctx.value:
                self.lib.jfdk_destroy(ctx)
            raise _lib.JfdkError(st, msg)
        self.ctx = ctx
        if bp_exact:
            self._check(self.lib.jfdk_set_option(ctx, _lib.OPT_BP_EXACT, 1))
        if view_chunk:
            self._check(self.lib.jfdk_set_option(ctx, _lib.OPT_VIEW_CHUNK, int(view_chunk)))
        dims = [C.c_int() for _ in range(4)]
        self._check(self.lib.jfdk_get_dims(ctx, *[C.byref(d) for d in dims]))
        self.filter_in_w, self.filter_out_w, self.fft_length, self.rows = [d.value for d in dims]

    # -- plumbing -------------------------------------------------------------
    def _check(self, st):
        _lib.check(self.ctx, st)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.jfdk_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sync(self):
        self._check(self.lib.jfdk_sync(self.ctx))

    @property
    def kernel_launches(self) -> int:
        return self.lib.jfdk_kernel_launches(self.ctx)

    @property
    def device_bytes(self) -> int:
        """Device memory the context holds now."""
        return self.lib.jfdk_device_bytes(self.ctx)

    def autotune(self, force: bool = False):
        """Pick slices per thread and views per chunk for this shape (timed on
        the device; cached per shape)."""
        self._check(self.lib.jfdk_autotune(self.ctx, _lib.AUTOTUNE_FORCE if force else 0))

    def set_option(self, key: int, value: int):
        self._check(self.lib.jfdk_set_option(self.ctx, key, int(value)))

    def get_option(self, key: int) -> int:
        """The option's value in effect (defaults resolved, jfdk_get_option)."""
        v = C.c_longlong(0)
        self._check(self.lib.jfdk_get_option(self.ctx, key, C.byref(v)))
        return int(v.value)

    @property
    def tile_depth(self) -> int:
        """Slices per backprojection thread in effect: z-slabs that start at
        multiples of it reproduce the whole volume bit for bit."""
        return self.get_option(_lib.OPT_BP_ZPT)

    def stage_times(self):
        """ms of [prep + filter, z-filter, backprojection] of the last
        reconstruct (needs set_option(OPT_STAGE_TIMING, 1))."""
        ms = (C.c_float * 3)()
        self._check(self.lib.jfdk_stage_times(self.ctx, ms))
        return list(ms)

    def uweights(self) -> np.ndarray:
        w = np.empty((self.scan.num_views, self.filter_out_w), np.float32)
        self._check(self.lib.jfdk_get_uweights(self.ctx, w.ctypes.data_as(C.c_void_p)))
        return w

    def ramp_operator(self):
        T = np.empty((self.filter_out_w, self.filter_in_w), np.float32)
        c = np.empty(self.filter_out_w, np.float32)
        self._check(self.lib.jfdk_get_ramp_operator(self.ctx, T.ctypes.data_as(C.c_void_p),
                                                    c.ctypes.data_as(C.c_void_p)))
        return T, c

    # -- stages (torch CUDA tensors in and out) ----------------------------------
    def preprocess(self, raw, out=None):
        import torch
        nv = raw.shape[0]
        used_v = self.scan.num_dets_v - self.scan.border_up - self.scan.border_down
        used_u = self.scan.num_dets_u - self.scan.border_left - self.scan.border_right
        out = out if out is not None else torch.empty((nv, used_v, used_u), dtype=torch.float32, device=raw.device)
        self._check(self.lib.jfdk_preprocess_frames(self.ctx, _ptr(raw), nv, _ptr(out)))
        return out

    def _filter_buffers(self, frames, out):
        """Checks frames (nv, rows, filter_in_w) and out (nv, rows,
        filter_out_w): contiguous float32 CUDA tensors; out is made when not
        given.  The C ABI takes raw pointers and would read or write past a
        tensor of another shape."""
        import torch

        def check(t, w, what):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
                raise ValueError(f"{what} must be a contiguous float32 CUDA tensor")
            if t.dim() != 3 or tuple(t.shape[1:]) != (self.rows, w):
                raise ValueError(f"{what} must be (views, {self.rows}, {w}), got {tuple(t.shape)}")
        check(frames, self.filter_in_w, "frames")
        nv = frames.shape[0]
        if out is None:
            out = torch.empty((nv, self.rows, self.filter_out_w), dtype=torch.float32, device=frames.device)
        check(out, self.filter_out_w, "out")
        if out.shape[0] != nv:
            raise ValueError(f"out holds {out.shape[0]} views, frames {nv}")
        return nv, out

    def filter(self, frames, v0: int = 0, out=None):
        nv, out = self._filter_buffers(frames, out)
        self._check(self.lib.jfdk_filter_frames(self.ctx, _ptr(frames), v0, nv, _ptr(out)))
        return out

    def filter_noalloc(self, frames, v0: int = 0, out=None):
        """``filter`` through jfdk_filter_frames_noalloc: working rows in the
        library's fixed 4 MiB device array, no allocation by the library (out
        must be given by callers that cannot allocate); the ramp product on
        FP32 CUDA cores whatever the context's form."""
        nv, out = self._filter_buffers(frames, out)
        self._check(self.lib.jfdk_filter_frames_noalloc(self.ctx, _ptr(frames), v0, nv, _ptr(out)))
        return out

    def composite(self, dirc, conj, v0: int = 0, out=None):
        """CompositeCore on pairs of preprocessed frames (views v0.. and their
        conjugates): (nv, rows, 2 width)."""
        import torch
        nv, H, W = dirc.shape
        out = out if out is not None else torch.empty((nv, H, 2 * W), dtype=torch.float32, device=dirc.device)
        self._check(self.lib.jfdk_composite_frames(self.ctx, _ptr(dirc), _ptr(conj), v0, nv, _ptr(out)))
        return out

    def zfilter(self, frames):
        self._check(self.lib.jfdk_zfilter_frames(self.ctx, _ptr(frames), frames.shape[0]))
        return frames

    def bp_reset(self):
        self._check(self.lib.jfdk_bp_reset(self.ctx))

    def bp_set_slab(self, z0: int, nz: int):
        """Accumulate (and finalize) slices [z0, z0 + nz) only: one z-part of a
        volume reconstructed in parts."""
        self._check(self.lib.jfdk_bp_set_slab(self.ctx, int(z0), int(nz)))

    def bp_accumulate(self, frames, v0: int):
        self._check(self.lib.jfdk_bp_accumulate(self.ctx, _ptr(frames), v0, frames.shape[0]))

    def finalize(self, apply_ctnum: bool = True, z0: int = 0, nz: Optional[int] = None, out=None,
                 out16=None, device="cuda"):
        import torch
        nz = self.recon.num_pixels_z - z0 if nz is None else nz
        shape = (nz, self.recon.num_pixels_y, self.recon.num_pixels_x)
        if out is None and out16 is None:
            out = torch.empty(shape, dtype=torch.float32, device=device)
        self._check(self.lib.jfdk_finalize(self.ctx, z0, nz, int(apply_ctnum), _ptr(out), _ptr(out16)))
        return out if out is not None else out16

    def ctnum(self, vol):
        self._check(self.lib.jfdk_ctnum(self.ctx, _ptr(vol), vol.numel()))
        return vol

    def reconstruct(self, raw, out=None, out16=None):
        import torch
        shape = (self.recon.num_pixels_z, self.recon.num_pixels_y, self.recon.num_pixels_x)
        if out is None and out16 is None:
            out = torch.empty(shape, dtype=torch.float32, device=raw.device)
        self._check(self.lib.jfdk_reconstruct(self.ctx, _ptr(raw), _ptr(out), _ptr(out16)))
        return out if out is not None else out16

    def reconstruct_host(self, raw: np.ndarray, out: Optional[np.ndarray] = None) -> np.ndarray:
        raw = np.ascontiguousarray(raw, np.uint16)
        shape = (self.recon.num_pixels_z, self.recon.num_pixels_y, self.recon.num_pixels_x)
        out = out if out is not None else np.empty(shape, np.float32)
        self._check(self.lib.jfdk_reconstruct_host(self.ctx, raw.ctypes.data_as(C.c_void_p),
                                                   out.ctypes.data_as(C.c_void_p)))
        return out

    # -- derivatives of the FP32 form (torch CUDA tensors) ------------------------
    # -- one volume over several GPUs (z-slabs; jenhine_b200.zslab) -------------
    def filter_raw(self, raw, v0: int, nv: int, out=None):
        """Filtered frames (nv, rows, filter_out_w) of views [v0, v0 + nv)
        from raw, the rotation's frames on the device (jfdk_filter_raw)."""
        import torch
        if out is None:
            out = torch.empty((nv, self.rows, self.filter_out_w), dtype=torch.float32, device=raw.device)
        if not (out.is_cuda and out.dtype == torch.float32 and out.is_contiguous()
                and tuple(out.shape) == (nv, self.rows, self.filter_out_w)):
            raise ValueError(f"out must be a contiguous float32 CUDA tensor ({nv}, {self.rows}, {self.filter_out_w})")
        self._check(self.lib.jfdk_filter_raw(self.ctx, _ptr(raw), int(v0), int(nv), _ptr(out)))
        return out

    def filter_to_store(self, raw, v0: int, nv: int):
        """Filter views [v0, v0 + nv) of raw (the rotation's frames, device) into
        the projection store."""
        self._check(self.lib.jfdk_filter_to_store(self.ctx, _ptr(raw), int(v0), int(nv)))

    def store_range(self, v0: int, nv: int):
        """(device address, bytes) of the store's records of views [v0, v0+nv),
        and (address, bytes) of their scales (mixed form) or None."""
        rec, nbytes, sc = C.c_void_p(), C.c_size_t(), C.c_void_p()
        self._check(self.lib.jfdk_store_range(self.ctx, int(v0), int(nv), C.byref(rec), C.byref(nbytes),
                                              C.byref(sc)))
        return (rec.value, nbytes.value), ((sc.value, 4 * int(nv)) if sc.value else None)

    def backproject_store(self, z0: int, nz: int, out=None, device="cuda"):
        """HU of slices [z0, z0 + nz) from every view in the store."""
        import torch
        if out is None:
            out = torch.empty((nz, self.recon.num_pixels_y, self.recon.num_pixels_x), dtype=torch.float32,
                              device=device)
        self._check(self.lib.jfdk_backproject_store(self.ctx, int(z0), int(nz), _ptr(out), None))
        return out

    def set_bp_geometry(self, ptms):
        """Projection matrices the backprojector uses from now on (the filter's
        pre-weight and the u-taper keep the creation geometry)."""
        p = np.ascontiguousarray(np.asarray(ptms, np.float32).reshape(self.scan.num_views, 12))
        self._check(self.lib.jfdk_set_bp_geometry(self.ctx, p.ctypes.data_as(C.c_void_p)))

    def bp_adjoint(self, vol_bar, v0: int = 0, nv: Optional[int] = None, out=None):
        """S^T (vol_bar / C) for views [v0, v0 + nv), C from the last
        bp_accumulate sequence."""
        import torch
        nv = self.scan.num_views - v0 if nv is None else nv
        out = out if out is not None else torch.empty((nv, self.rows, self.filter_out_w), dtype=torch.float32,
                                                      device=vol_bar.device)
        self._check(self.lib.jfdk_bp_adjoint(self.ctx, _ptr(vol_bar), v0, nv, _ptr(out)))
        return out

    def filter_adjoint(self, q_bar, v0: int = 0, out=None):
        import torch
        nv = q_bar.shape[0]
        out = out if out is not None else torch.empty((nv, self.rows, self.filter_in_w), dtype=torch.float32,
                                                      device=q_bar.device)
        self._check(self.lib.jfdk_filter_adjoint(self.ctx, _ptr(q_bar), v0, nv, _ptr(out)))
        return out

    def geometry_gradient(self, q, v0: int, vol, vol_bar, dptm, out=None):
        """dL/dtheta (nv x 6, float64) for views [v0, v0 + q.shape[0]) given
        dP/dtheta (nv x 6 x 12, float32 CUDA)."""
        import torch
        nv = q.shape[0]
        out = out if out is not None else torch.empty((nv, 6), dtype=torch.float64, device=q.device)
        self._check(self.lib.jfdk_geometry_gradient(self.ctx, _ptr(q), v0, nv, _ptr(vol), _ptr(vol_bar),
                                                    _ptr(dptm), _ptr(out)))
        return out


class FDKBatch:
    """Scans of uneven size reconstructed together, recorded as a CUDA graph on
    the first run with a set of buffers and replayed after.  schedule:
    "persistent" (each scan's filter stage, then one persistent backprojection
    launch over the tiles of up to 8 scans), "pipelined" (each scan's own
    backprojection beside the next scan's filter stage), or None: the faster
    of the two, timed on the first run when autotune is on (else persistent).

        batch = FDKBatch([engine_0, ..., engine_n], autotune=True)
        batch.run([raw_0, ...], [vol_0, ...])   # torch CUDA tensors
    """

    def __init__(self, engines, autotune: bool = True, graph: bool = True, stream=None,
                 schedule: Optional[str] = None):
        import torch
        self.lib = _lib.load()
        self.h = None
        self.engines = list(engines)
        self.stream = stream if stream is not None else torch.cuda.Stream()
        arr = (C.c_void_p * len(self.engines))(*[e.ctx for e in self.engines])
        h = C.c_void_p()
        flags = (_lib.BATCH_AUTOTUNE if autotune else 0) | (_lib.BATCH_GRAPH if graph else 0)
        flags |= {None: 0, "persistent": _lib.BATCH_PERSISTENT, "pipelined": _lib.BATCH_PIPELINED}[schedule]
        st = self.lib.jfdk_batch_create(C.byref(h), arr, len(self.engines), flags,
                                        C.c_void_p(self.stream.cuda_stream))
        self.h = h.value
        if st != _lib.JFDK_OK:
            msg = self.lib.jfdk_batch_last_error(self.h).decode() if self.h else ""
            self.close()
            raise _lib.JfdkError(st, msg)

    def run(self, raws, outs):
        """Reconstruct every scan (HU volumes into outs), ordered after the
        caller's current stream, and the caller's stream after it."""
        import torch
        cur = torch.cuda.current_stream()
        self.stream.wait_stream(cur)
        r = (C.c_void_p * len(raws))(*[x.data_ptr() for x in raws])
        o = (C.c_void_p * len(outs))(*[x.data_ptr() for x in outs])
        st = self.lib.jfdk_batch_run(self.h, r, o)
        if st != _lib.JFDK_OK:
            raise _lib.JfdkError(st, self.lib.jfdk_batch_last_error(self.h).decode())
        cur.wait_stream(self.stream)
        return outs

    @property
    def launches(self) -> int:
        return self.lib.jfdk_batch_launches(self.h)

    @property
    def schedule(self) -> Optional[str]:
        """The schedule in use (None before the first run picks one)."""
        return {0: None, _lib.BATCH_PERSISTENT: "persistent",
                _lib.BATCH_PIPELINED: "pipelined"}[self.lib.jfdk_batch_schedule(self.h)]

    def close(self):
        if getattr(self, "h", None):
            self.lib.jfdk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
