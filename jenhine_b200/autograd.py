"""Thin torch.autograd binding of the FP32 form's derivatives.

    vol = FDKFunction.apply(p, theta, engine, P0)

p: (views, rows, filter_in_w) float32 CUDA, preprocessed projections (line
integrals); theta: (views, 6) rigid motion per view (jenhine_b200.motion),
any device / dtype; engine: an FP32-form FDKEngine created with the nominal
matrices P0 (views x 12).  The filter, its cosine pre-weight and the u-taper
use P0; the backprojection uses P0 M(theta).  vol is the attenuation volume
(no CT numbers; NaN where no view sees a voxel).  backward returns dL/dp
(adjoint backprojection, then adjoint filter) and dL/dtheta (geometry
gradient).  The engine keeps the weights of the last forward, so each
backward must follow its own forward on that engine.  Meant for tests and
small problems; large problems call the engine's entry points directly.
"""
from __future__ import annotations

import numpy as np
import torch

from .motion import moved_ptms, ptm_derivatives


class FDKFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p, theta, engine, P0, chunk: int = 64):
        th = theta.detach().to("cpu", torch.float64).numpy()
        engine.set_bp_geometry(moved_ptms(P0, th).astype(np.float32))
        p = p.contiguous()
        nv = p.shape[0]
        q = torch.empty((nv, engine.rows, engine.filter_out_w), dtype=torch.float32, device=p.device)
        for v0 in range(0, nv, chunk):
            engine.filter(p[v0:v0 + chunk], v0, out=q[v0:v0 + chunk])
        engine.bp_reset()
        for v0 in range(0, nv, chunk):
            engine.bp_accumulate(q[v0:v0 + chunk], v0)
        vol = engine.finalize(apply_ctnum=False, device=p.device)
        ctx.engine, ctx.chunk = engine, chunk
        ctx.dptm = torch.from_numpy(ptm_derivatives(P0, th).astype(np.float32)).to(p.device)
        ctx.theta_like = (theta.device, theta.dtype)
        ctx.save_for_backward(q, vol)
        return vol

    @staticmethod
    def backward(ctx, vol_bar):
        q, vol = ctx.saved_tensors
        e, chunk = ctx.engine, ctx.chunk
        vol_bar = torch.where(torch.isfinite(vol), vol_bar.to(torch.float32), 0.0).contiguous()
        nv = q.shape[0]
        p_bar = torch.empty((nv, e.rows, e.filter_in_w), dtype=torch.float32, device=q.device)
        g = torch.empty((nv, 6), dtype=torch.float64, device=q.device)
        for v0 in range(0, nv, chunk):
            n = min(chunk, nv - v0)
            e.filter_adjoint(e.bp_adjoint(vol_bar, v0, n), v0, out=p_bar[v0:v0 + n])
            e.geometry_gradient(q[v0:v0 + n], v0, vol, vol_bar, ctx.dptm[v0:v0 + n], out=g[v0:v0 + n])
        dev, dt = ctx.theta_like
        return p_bar, g.to(dev, dt), None, None, None
