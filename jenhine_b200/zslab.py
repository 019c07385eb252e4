"""One volume over several GPUs: z-slabs.

Each rank (one process per GPU, torch.distributed over NCCL) filters its
share of the views into its engine's projection store, the stores are
completed by one broadcast per rank of that rank's records (over NVLink; the
records of all views, 16 bytes a pixel, cross each link once), and each rank
backprojects its own slab of slices from every view.  Per GPU: V/N views of
preprocessing and ramp filtering, 1/N of the voxel-view updates, no
reduction.  The slabs start at multiples of the backprojection's tile depth,
so the slab volumes equal one GPU's jfdk_reconstruct bit for bit.

The engine's steps (FDKEngine.filter_to_store, store_range,
backproject_store) are the C ABI's jfdk_filter_to_store, jfdk_store_range
and jfdk_backproject_store; this module adds the partition and the exchange.
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


def reconstruct_zslab(engine, raw, rank: int, world: int, group=None, out=None, tile_depth: int = 8):
    """This rank's slab of the HU volume: (z0, tensor of nz x Y x X).  raw:
    the rotation's frames on this rank's GPU (only this rank's views -- and
    their conjugates when compositing -- are read)."""
    views = view_ranges(engine.scan.num_views, world)
    slabs = slab_ranges(engine.recon.num_pixels_z, world, tile_depth)
    v0, nv = views[rank]
    engine.filter_to_store(raw, v0, nv)
    if world > 1:
        recs, scales = [], []
        for (a, n) in views:
            rec, sc = engine.store_range(a, n)
            recs.append(device_bytes(*rec, raw.device))
            scales.append(device_bytes(*sc, raw.device) if sc else None)
        exchange(recs, rank, group)
        if scales[0] is not None:
            exchange(scales, rank, group)
    z0, nz = slabs[rank]
    if nz == 0:
        return z0, None
    return z0, engine.backproject_store(z0, nz, out=out, device=raw.device)
