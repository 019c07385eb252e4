"""Host logic of the multi-GPU paths, on CPU with world_size-2 gloo process
groups: the z-slab partition (jenhine_b200.zslab), its exchange (one
broadcast per rank), the z-slab reconstruction's order of steps over a
stand-in engine (filtered frames exchanged, every view accumulated in order
into each rank's slab), and the bench's max-over-ranks timing reduction."""
import os
import socket
import sys

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_view_and_slab_partitions():
    from jenhine_b200.zslab import slab_ranges, view_ranges
    for n, world in ((600, 8), (10, 3), (7, 4), (3, 4)):
        vr = view_ranges(n, world)
        assert [a for a, _ in vr] == [sum(k for _, k in vr[:i]) for i in range(world)]
        assert sum(k for _, k in vr) == n and max(k for _, k in vr) - min(k for _, k in vr) <= 1
    for z, world, td in ((480, 8, 8), (20, 3, 8), (20, 4, 8), (5, 4, 8), (33, 2, 4)):
        sr = slab_ranges(z, world, td)
        assert sum(k for _, k in sr) == z
        assert all(a % td == 0 or k == 0 for a, k in sr)
        ends = [a + k for a, k in sr]
        assert all(sr[i + 1][0] == ends[i] for i in range(world - 1) if sr[i + 1][1])
        tiles = [-(-k // td) for _, k in sr]
        assert max(tiles) - min(tiles) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
        sys.path.insert(0, ROOT)
        import bench
        from jenhine_b200 import zslab
        dist = bench.init_dist(world, 0, backend="gloo")
        # each rank owns one range of a 10-view "store" of 6 values a view
        views = zslab.view_ranges(10, world)
        store = torch.full((10, 6), -1.0)
        a, n = views[rank]
        store[a:a + n] = torch.arange(a * 6, (a + n) * 6, dtype=torch.float32).reshape(n, 6)
        zslab.exchange([store[s:s + k] for s, k in views], rank)
        ok_store = torch.equal(store, torch.arange(60, dtype=torch.float32).reshape(10, 6))
        # the job's time is its slowest rank's
        got = bench.max_over_ranks(dist, 10.0 + rank, device="cpu")
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok_store, got))
    except Exception as e:  # reported to the test, never left hanging
        q.put((rank, False, repr(e)))


def test_zslab_exchange_and_rank_max_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for rank, ok_store, got in sorted(results):
        assert ok_store, (rank, got)
        assert got == 10.0 + world - 1, (rank, got)


class _FakeEngine:
    """The engine steps reconstruct_zslab calls, on CPU: filtered frames are
    the view index in every pixel; bp_accumulate checks that the frames it
    is given are those of its views and records the order."""

    class _C:
        pass

    def __init__(self, views, slices):
        self.scan, self.recon = self._C(), self._C()
        self.scan.num_views = views
        self.recon.num_pixels_z, self.recon.num_pixels_y, self.recon.num_pixels_x = slices, 2, 2
        self.rows, self.filter_out_w = 2, 3
        self.log = []

    def filter_raw(self, raw, v0, nv, out):
        out.copy_(torch.arange(v0, v0 + nv, dtype=torch.float32).view(nv, 1, 1).expand_as(out))
        self.log.append(("filter", v0, nv))

    def bp_set_slab(self, z0, nz):
        self.log.append(("slab", z0, nz))

    def bp_reset(self):
        self.log.append(("reset",))

    def bp_accumulate(self, frames, v0):
        n = frames.shape[0]
        ok = torch.equal(frames[:, 0, 0], torch.arange(v0, v0 + n, dtype=torch.float32))
        self.log.append(("acc", v0, n, ok))

    def finalize(self, apply_ctnum, z0, nz, out=None, device="cpu"):
        self.log.append(("finalize", z0, nz))
        return torch.zeros((nz, 2, 2))


def _zslab_worker(rank, world, port, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
        sys.path.insert(0, ROOT)
        import bench
        from jenhine_b200 import zslab
        dist = bench.init_dist(world, 0, backend="gloo")
        e = _FakeEngine(10, 20)
        z0, vol = zslab.reconstruct_zslab(e, torch.zeros(1), rank, world, tile_depth=8)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, e.log, z0, None if vol is None else tuple(vol.shape)))
    except Exception as ex:  # reported to the test, never left hanging
        q.put((rank, repr(ex), None, None))


def test_zslab_reconstruction_steps_gloo():
    from jenhine_b200.zslab import slab_ranges, view_ranges
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_zslab_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    views, slabs = view_ranges(10, world), slab_ranges(20, world, 8)
    for rank, log, z0, shape in sorted(results):
        assert isinstance(log, list), log
        a, n = views[rank]
        sz0, snz = slabs[rank]
        assert log[0] == ("filter", a, n)
        assert log[1:3] == [("slab", sz0, snz), ("reset",)]
        accs = [x for x in log if x[0] == "acc"]
        # every view, in order, each chunk carrying its own views' frames
        assert [(x[1], x[2]) for x in accs] == views and all(x[3] for x in accs), accs
        assert log[-1] == ("finalize", sz0, snz) and z0 == sz0 and shape == (snz, 2, 2)
