"""One volume over several GPUs: z-slabs.

Each rank (one process per GPU, torch.distributed over NCCL) filters its
share of the views into FP32 filtered frames (jfdk_filter_raw), the frames of
every view reach every rank by one broadcast per rank (over NVLink; 4 bytes a
pixel, each view's frames crossing each link once), and each rank
backprojects every view into its own slab of slices (jfdk_bp_set_slab,
jfdk_bp_reset, jfdk_bp_accumulate, jfdk_finalize).  The broadcasts are all
issued up front and run on the collective stream while the backprojection
of the views already present runs on the compute stream; the views are
accumulated in order, rank by rank as their frames arrive, so each rank's
slab equals one GPU's jfdk_reconstruct on those slices bit for bit (the
partial sums are stored and reloaded exactly).  The slabs start at
multiples of the backprojection's tile depth for the same reason.  Per GPU:
V/N views of preprocessing and ramp filtering, 1/N of the voxel-view
updates, no reduction; each rank packs the backprojection's store from the
exchanged frames itself.
"""
from __future__ import annotations

from typing import Optional


def view_ranges(n_views: int, world: int) -> list[tuple[int, int]]:
    """(first view, views) of each rank: contiguous, sizes differing by one."""
    base, extra = divmod(n_views, world)
    out, v = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((v, n))
        v += n
    return out


def slab_ranges(n_slices: int, world: int, tile_depth: int = 8) -> list[tuple[int, int]]:
    """(first slice, slices) of each rank: contiguous slabs of whole tiles
    (tile_depth slices; the volume's last tile may be short), the tile counts
    differing by one at most (a rank may get none)."""
    tiles = -(-n_slices // tile_depth)
    base, extra = divmod(tiles, world)
    out, t = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        z0 = min(t * tile_depth, n_slices)
        out.append((z0, min((t + n) * tile_depth, n_slices) - z0))
        t += n
    return out


class _DeviceBytes:
    """A device byte range as a tensor source (__cuda_array_interface__)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3}


def device_bytes(ptr: int, nbytes: int, device):
    import torch
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=device)


def exchange(parts, rank: int, group=None) -> None:
    """Complete every rank's copy of a partitioned buffer: parts[r] is this
    rank's tensor for rank r's range (its own is filled, the others are
    overwritten); one broadcast per rank."""
    import torch.distributed as dist
    for src, t in enumerate(parts):
        if t is not None and t.numel():
            dist.broadcast(t, src=src, group=group)


def reconstruct_zslab(engine, raw, rank: int, world: int, group=None, out=None, tile_depth: Optional[int] = None,
                      frames=None):
    """This rank's slab of the HU volume: (z0, tensor of nz x Y x X, or None
    when the rank has no slices).  raw: the rotation's frames on this rank's
    GPU (only this rank's views -- and their conjugates when compositing --
    are read); frames: an optional (views, rows, filter_out_w) float32 device
    buffer for the filtered frames of every view; tile_depth: the slabs'
    granularity (default: the engine's backprojection tile depth)."""
    import torch
    V = engine.scan.num_views
    views = view_ranges(V, world)
    if tile_depth is None:
        tile_depth = engine.tile_depth
    slabs = slab_ranges(engine.recon.num_pixels_z, world, tile_depth)
    if frames is None:
        frames = torch.empty((V, engine.rows, engine.filter_out_w), dtype=torch.float32, device=raw.device)
    v0, nv = views[rank]
    if nv:
        engine.filter_raw(raw, v0, nv, out=frames[v0:v0 + nv])
    works = [None] * world
    if world > 1:
        import torch.distributed as dist
        # every rank issues the same broadcasts in the same order, all at once
        for s, (a, n) in enumerate(views):
            if n:
                works[s] = dist.broadcast(frames[a:a + n], src=s, group=group, async_op=True)
    z0, nz = slabs[rank]
    if nz:
        engine.bp_set_slab(z0, nz)
        engine.bp_reset()
    for s, (a, n) in enumerate(views):
        if works[s] is not None:
            works[s].wait()          # the compute stream waits for rank s's frames
        if nz and n:
            engine.bp_accumulate(frames[a:a + n], a)
    if not nz:
        return z0, None
    return z0, engine.finalize(apply_ctnum=True, z0=z0, nz=nz, out=out, device=raw.device)
