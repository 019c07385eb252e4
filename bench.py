#!/usr/bin/env python
"""FDK reconstruction throughput on B200: GUPS (voxel-view updates / s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--workload c2] [--precision both|fp32|mixed] [--no-cpu-baseline]

A step is one full reconstruction of the workload (raw uint16 frames ->
preprocess -> cosine pre-weight -> ramp filter -> backprojection -> CT
numbers) with the raw frames already resident in HBM.  Under torchrun each
rank reconstructs its own seeded scan (independent objects, no data-path
collective): weak scaling.  value = updates of all ranks / max over ranks of
the device-timed K steps.  By default both forms run back to back: the line's
value, e2e and roofline are the plain FP32 form's, forms.mixed holds the
mixed-precision form's numbers and its speed-up over the plain form.

e2e: the same metric through the C ABI's host-buffer call
(jfdk_reconstruct_host): every step copies the raw frames in from pinned
host memory and the HU volume back out.

--impl reference times the reference's own CPU Cores (PreProcessingCore,
FilterAgent/FilterCore + PreFilterWeightGenerator, BPAgent/BPCore,
CTNumCore compiled from source into oracle/_ref) on the host cores, each step
a bounded sample of the same workload extrapolated to one volume.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GUPS (voxel·view/s) & s/volume, 640²×480 from 600 views: mixed vs plain FP32"
DATA = "synthetic: seeded ellipsoid phantom, analytic line integrals, Poisson noise, per-pixel gain/offset"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "mixed"],
                    help="both: the plain FP32 form is the line's value, the mixed form under forms.mixed")
    ap.add_argument("--exact", action="store_true", help="BPCore-exact backprojection rounding")
    ap.add_argument("--zpt", type=int, default=0, help="slices per backprojection thread (0: form default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the default c2 line's batch key (the 16-scan batch, mixed form)")
    ap.add_argument("--no-gpu-baseline", action="store_true",
                    help="skip timing the reference's own GPU backprojector (baseline/_ref)")
    ap.add_argument("--split", default="scans", choices=["scans", "zslab"],
                    help="scans: one independent scan per GPU (weak scaling); zslab: one volume, each GPU "
                         "filters 1/N of the views and backprojects 1/N of the slices (strong scaling)")
    return ap.parse_args()


def init_dist(world, local, backend="nccl"):
    """The job's process group (None for one process); a short timeout so
    ranks that wait for one another end with an error."""
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
    return dist


def max_over_ranks(dist, value: float, device="cuda") -> float:
    """The largest of every rank's value (the job's time is its slowest rank's)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def workload_config(w):
    r, g = w.recon, w.geom
    return {"workload": f"{w.name}: {r.num_pixels_x}x{r.num_pixels_y}x{r.num_pixels_z} from {g.n_views} views "
                        f"of {g.det_u}x{g.det_v}",
            "views": g.n_views, "detector": [g.det_u, g.det_v], "volume": [r.num_pixels_x, r.num_pixels_y,
                                                                          r.num_pixels_z],
            "voxel_mm": [r.pitch_xy, r.pitch_z], "sid_sdd_mm": [g.sid, g.sdd],
            "updates_per_volume": w.updates,
            "l2": "inputs larger than L2 (raw frames, filtered store and volume each > 126 MB)"
                  if w.updates > FULL_CPU_UPDATES else "L2 flushed before each timed step (256 MB write)",
            "setup": "per-geometry setup (ramp operator, pre-weight table, u-taper) at context creation and the "
                     "normalisation-weight volume at the first reconstruction (a warm-up step), outside the timed "
                     "step, as the reference's GPU path caches its weight pass in a file"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.idx = gpu_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [l.strip().split(", ") for l in self.f.read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_figure(name: str, key: str):
    """A figure of a committed ncu summary (profiles/<name>.md, line 'key: N')."""
    try:
        for line in open(os.path.join(ROOT, "profiles", f"{name}.md")):
            if line.strip().startswith(key + ":"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def profile_traffic(name: str):
    """dram bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/<name>.md, line 'dram_bytes_per_launch: N')."""
    path = os.path.join(ROOT, "profiles", f"{name}.md")
    try:
        for line in open(path):
            if line.strip().startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


FULL_CPU_UPDATES = 2_000_000_000   # workloads up to this many updates run whole on the CPU


def cpu_full(w) -> bool:
    """The CPU baseline runs the whole workload (not a sample) when it is
    small enough to finish in seconds on the host (c1: 7.6e8 updates)."""
    return w.updates <= FULL_CPU_UPDATES


CPU_NOTES = {"ipp_mkl": "the reference's Cores compiled from source with scalar restatements of its Intel IPP / MKL "
                        "calls (oracle/ref_shims; IPP and MKL are not in the image)",
             "setup": "per-geometry setup (FilterCore spectrum, pre-weight generator, BPCore axes) outside the timed "
                      "run, as the engine's context creation is outside its timed step"}


def cpu_sample(w, raw_np, filt_np, ptms):
    """The reference CPU Cores on the workload: all of it when cpu_full(w)
    (raw_np holds every view), else a bounded sample -- preprocess + filter of
    12 views, BPCore over 60 views of a 16-slice central slab (filt_np: those
    60 views filtered) -- extrapolated linearly to one volume.
    Returns (GUPS, cores, kind, sample description, seconds spent, seconds
    per volume, extrapolated)."""
    import numpy as np
    try:
        from oracle.pyoracle import RefCores
        impl, kind = RefCores(), "reference"
    except (OSError, FileNotFoundError, RuntimeError):
        from oracle.pyoracle import Oracle
        impl, kind = Oracle(), "port"
    cores = os.cpu_count() or 1
    r, g = w.recon, w.geom
    full = cpu_full(w)
    nv_f = g.n_views if full else min(12, g.n_views)
    nv_b = g.n_views if full else min(60, g.n_views)
    nz = r.num_pixels_z if full else min(16, r.num_pixels_z)
    t0 = time.perf_counter()
    if kind == "reference":
        prep = impl.preprocess(raw_np[:nv_f], w.bright_field, w.beam_hardening, nthreads=cores)
        t1 = time.perf_counter()
        filt = impl.filter(prep, ptms, g.half_sample_rate, g.sid, nthreads=cores)
        t2 = time.perf_counter()
        if full:
            vol = impl.bp(filt, ptms, r.num_pixels_x, r.num_pixels_y, r.num_pixels_z, r.pitch_xy, r.pitch_z,
                          nthreads=cores)
        else:
            # BPCore over a central z-slab: the reference backprojects the
            # whole volume, whose cost is linear in slices
            vol = _ref_bp_slab(impl, filt_np[:nv_b], ptms[:nv_b], r, nz, r.num_pixels_z // 2 - nz // 2, cores)
        t3 = time.perf_counter()
        impl.ctnum(vol, r.ct_norm0, r.ct_norm1)
        t4 = time.perf_counter()
    else:
        prep = impl.preprocess(raw_np[:nv_f], w.bright_field, w.beam_hardening)
        t1 = time.perf_counter()
        H = impl.filter_spectrum(impl.fft_length(g.det_u), g.half_sample_rate)
        filt = np.stack([impl.filter_rows(prep[v], H, impl.fft_length(g.det_u)) for v in range(nv_f)])
        t2 = time.perf_counter()
        vol = impl.bp(filt if full else filt_np[:nv_b], ptms[:nv_b], r.num_pixels_x, r.num_pixels_y,
                      r.num_pixels_z, r.pitch_xy, r.pitch_z, z0=r.num_pixels_z // 2 - nz // 2, nz=nz,
                      nthreads=cores)
        t3 = time.perf_counter()
        impl.ctnum(vol, r.ct_norm0, r.ct_norm1)
        t4 = time.perf_counter()
    per_volume = ((t1 - t0) + (t2 - t1)) * g.n_views / nv_f + (t3 - t2) * (g.n_views / nv_b) * (
        r.num_pixels_z / nz) + (t4 - t3) * r.num_pixels_z / nz
    if full:
        sample = f"the whole workload, not extrapolated: {per_volume:.2f} s/volume"
    else:
        sample = (f"preprocess+filter of {nv_f} views (x{g.n_views / nv_f:g}) and BP of {nv_b} views into "
                  f"{nz} of {r.num_pixels_z} slices (x{g.n_views / nv_b * r.num_pixels_z / nz:g}), "
                  f"extrapolated linearly to one volume: {per_volume:.1f} s/volume")
    return w.updates / per_volume / 1e9, cores, kind, sample, t4 - t0, per_volume, not full


def _ref_bp_slab(ref, filt, ptms, r, nz, z0, cores):
    """The reference BPCore on slices [z0, z0+nz): shift the volume centre with
    the reference's own MoveZAxis PTM edit (JEngine/JEngine.cpp:149) so a
    nz-slice BPCore reconstructs exactly that slab."""
    import numpy as np
    zc = (z0 + (nz - 1) / 2.0) - (r.num_pixels_z - 1) / 2.0
    p = np.stack([ref.ptm_modify(ptms[i], "move_z", float(np.float32(zc * r.pitch_z))) for i in range(len(ptms))])
    return ref.bp(filt, p, r.num_pixels_x, r.num_pixels_y, nz, r.pitch_xy, r.pitch_z, nthreads=cores)


def error_sample(w):
    """The voxels each form's error against the FP64 oracle is stated on:
    (first slice, slices, stride in x and y) -- the 8 central slices, every
    4th voxel in x and y (the whole volume for volumes of at most 2^21
    voxels)."""
    r = w.recon
    if r.num_pixels_x * r.num_pixels_y * r.num_pixels_z <= 1 << 21:
        return 0, r.num_pixels_z, 1
    nz = min(8, r.num_pixels_z)
    return r.num_pixels_z // 2 - nz // 2, nz, 4


def fp64_errors(w, raw_np, samples):
    """Error of each form's volume against the FP64 oracle on the error
    sample (tests/fp64_fdk.py: the reference's float preprocessing and
    pre-weight, then filter, backprojection and CT numbers in double):
    rel-L2 of HU + 1000 and max |dHU| over the interior voxels (sampled at
    least a pixel inside the detector by every view) and over all voxels."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from fp64_fdk import all_points, case_from_workload, errors, fdk_f64, survey
    from oracle.pyoracle import Oracle
    r = w.recon
    z0, nz, stride = error_sample(w)
    pts = all_points(r.num_pixels_x, r.num_pixels_y, r.num_pixels_z, z0=z0, nz=nz, stride=stride)
    g = case_from_workload(w, raw_np)
    ref = fdk_f64(Oracle(), g, pts)
    inside = survey(g, pts)[0]
    out = {}
    for form, hu in samples.items():
        e = errors(np.asarray(hu, np.float64).ravel(), ref, inside)
        out[form] = {"rel_l2": e["rel_l2_interior"], "max_hu": e["max_hu_interior"], "rel_l2_all": e["rel_l2_all"],
                     "max_hu_all": e["max_hu_all"], "voxels": e["voxels"], "interior_voxels": e["interior_voxels"]}
    out["sample"] = (f"slices {z0}..{z0 + nz - 1}, every {stride}th voxel in x and y" if stride > 1 else
                     f"slices {z0}..{z0 + nz - 1}, every voxel")
    out["oracle"] = ("FP64 FDK (tests/fp64_fdk.py): float preprocessing and pre-weight as the reference, then "
                     "filter, taper, coordinates, lerps, sums and CT numbers in double; rel_l2 / max_hu over the "
                     "interior voxels, *_all over every voxel")
    return out


def gpu_baseline(w, raw, ptms, local):
    """The reference's own GPU backprojector (BPCUDAAgent/BPCUDACore.cu,
    compiled unchanged for sm_100a into baseline/_ref by oracle/build.py)
    through the host loop BPCUDAAgent drives it with: per view three Scale
    kernels and a stream sync (PreCalculate_Synced), the BackProject kernel
    (a texture fetch and a global read-modify-write of the volume per voxel)
    and a sync; then per slice the host-side FP16 weight expansion, its upload
    and the Div2 kernel.  Fed the engine's own filtered projections, one part
    (the volume fits).  Host-timed: the reference synchronises after every
    kernel.  None when the library is not built."""
    import ctypes as C
    import numpy as np
    from jenhine_b200.fdk import FDKEngine
    path = os.path.join(ROOT, "baseline", "_ref", "libbpcuda_ref.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.jrefgpu_bp.restype = C.c_int
    lib.jrefgpu_last_error.restype = C.c_char_p
    g, r = w.geom, w.recon
    eng = FDKEngine(w.scan, w.recon, ptms)
    filt = np.empty((g.n_views, eng.rows, eng.filter_out_w), np.float32)
    for v0 in range(0, g.n_views, 100):
        filt[v0:v0 + 100] = eng.filter(eng.preprocess(raw[v0:v0 + 100]), v0).cpu().numpy()
    eng.close()
    t = (C.c_double * 3)()
    P = np.ascontiguousarray(ptms, np.float32)
    clocks = ClockSampler(local)
    clocks.start()
    st = lib.jrefgpu_bp(None, filt.ctypes.data_as(C.c_void_p), P.ctypes.data_as(C.c_void_p), g.n_views,
                        eng.filter_out_w, eng.rows, r.num_pixels_x, r.num_pixels_y, r.num_pixels_z,
                        C.c_float(r.pitch_xy), C.c_float(r.pitch_z), 1, 2, t)
    clk = clocks.stop()
    if st != 0:
        return {"unavailable": "reference GPU backprojector failed: " + lib.jrefgpu_last_error().decode()}
    return {"value": w.updates / (t[0] / 1000.0) / 1e9, "unit": "GUPS", "backprojection_ms": t[0],
            "normalise_output_ms": t[1], "setup_ms": t[2],
            "kernel": "reference BPCUDACore (BPCUDAAgent/BPCUDACore.cu) compiled unchanged for sm_100a, driven by "
                      "BPCUDAAgent's loop (oracle/ref_gpu/bpcuda_driver.cpp)",
            "timed": "backprojection_ms: every view (PreCalculate_Synced, DeployBackProj, SyncBackProj); value = "
                     "updates / backprojection_ms, comparable with stages_ms.backprojection_hu; normalise_output_ms: "
                     "every slice (DeployUpdateOutput, SyncUpdateOutput); setup_ms (not in value): texture uploads "
                     "and the weight pass the reference caches in a file",
            "clocks": clk}


def time_zslab(a, w, raw, ptms, precision, dist, rank, world, local):
    """One volume over the job's GPUs (jenhine_b200.zslab): per step each rank
    filters its share of the views, the FP32 filtered frames of every view
    reach every rank by broadcasts over NVLink (overlapped with the
    backprojection of the views already there), and each rank backprojects
    its slab.  Device-timed, max over ranks; value = one volume's updates per
    second."""
    import torch
    from jenhine_b200.fdk import FDKEngine
    from jenhine_b200.zslab import reconstruct_zslab, slab_ranges
    eng = FDKEngine(w.scan, w.recon, ptms, precision=precision, bp_exact=a.exact)
    r = w.recon
    z0, nz = slab_ranges(r.num_pixels_z, world, eng.tile_depth)[rank]
    out = torch.empty((max(nz, 1), r.num_pixels_y, r.num_pixels_x), dtype=torch.float32, device="cuda")
    frames = torch.empty((w.geom.n_views, eng.rows, eng.filter_out_w), dtype=torch.float32, device="cuda")
    for _ in range(a.warmup):
        reconstruct_zslab(eng, raw, rank, world, out=out[:nz] if nz else None, frames=frames)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    l0 = eng.kernel_launches
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start.record()
    for _ in range(a.steps):
        reconstruct_zslab(eng, raw, rank, world, out=out[:nz] if nz else None, frames=frames)
    end.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = max_over_ranks(dist, start.elapsed_time(end) / a.steps)
    launches = eng.kernel_launches - l0
    eng.close()
    return {"value": w.updates / (ms / 1000.0) / 1e9, "ms_per_step": ms, "s_per_volume": ms / 1000.0,
            "gpu_launches": launches, "clocks": clk,
            "exchange_bytes_per_step": int(frames.numel() * 4) if world > 1 else 0}


def run_reference(a, w, rank, world):
    """--impl reference: the reference CPU implementation, rank 0 only."""
    if rank != 0:
        return
    from jenhine_b200.phantom import line_integrals, raw_frames
    g = w.geom
    ptms = g.ptms()
    full = cpu_full(w)
    # inputs: every view (whole run), or the first views (bounded sample)
    nv = g.n_views if full else min(60, g.n_views)
    lint = line_integrals(g, w.phantom(), views=range(nv))
    raw = raw_frames(lint, g.seed + 2, i0=w.i0, bright_field=w.bright_field, gain_spread=w.gain_spread,
                     offset_max=w.offset_max)
    filt = None
    if not full:   # the BP sample's filtered views, from the reference Cores
        from oracle.pyoracle import RefCores
        ref = RefCores()
        prep = ref.preprocess(raw, w.bright_field, w.beam_hardening, nthreads=os.cpu_count() or 1)
        filt = ref.filter(prep, ptms, g.half_sample_rate, g.sid, nthreads=os.cpu_count() or 1)
    vals, secs = [], []
    for i in range(a.warmup + a.steps):
        gups, cores, kind, sample, spent, per_volume, extrap = cpu_sample(w, raw, filt, ptms)
        if i >= a.warmup:
            vals.append(gups)
            secs.append(per_volume)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GUPS", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": statistics.median(secs) * 1000.0,
            "s_per_volume": statistics.median(secs), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": DATA, "config": workload_config(w),
            "cpu_baseline": {"value": value, "unit": "GUPS", "cores": cores, "kind": kind, "sample": sample,
                             "extrapolated": extrap, **CPU_NOTES},
            "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_form(a, w, raw, ptms, precision, dist, world, local):
    """Device-timed steps of one form (raw frames resident in HBM), then the
    same through the host-buffer call.  Returns a dict of the form's numbers."""
    import torch
    from jenhine_b200 import _lib
    from jenhine_b200.fdk import FDKEngine
    eng = FDKEngine(w.scan, w.recon, ptms, precision=precision, bp_exact=a.exact)
    eng.set_option(_lib.OPT_STAGE_TIMING, 1)
    if a.zpt:
        eng.set_option(_lib.OPT_BP_ZPT, a.zpt)
    r = w.recon
    vol = torch.empty((r.num_pixels_z, r.num_pixels_y, r.num_pixels_x), dtype=torch.float32, device="cuda")
    for _ in range(a.warmup):
        eng.reconstruct(raw, vol)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    launches0 = eng.kernel_launches
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stage_ms = []
    # a workload whose inputs partly fit in L2 gets L2 flushed before each
    # step (a 256 MB write, outside the step's events)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if w.updates <= FULL_CPU_UPDATES else None
    step_ms = 0.0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start.record()
    for _ in range(a.steps):
        if flush is not None:
            flush.fill_(1)
            s1, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s1.record()
        eng.reconstruct(raw, vol)
        if flush is not None:
            e1.record()
        stage_ms.append(eng.stage_times())   # events on the engine's stream (synchronises)
        if flush is not None:
            step_ms += s1.elapsed_time(e1)
    end.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = eng.kernel_launches - launches0
    clk = clocks.stop()
    ms = max_over_ranks(dist, (step_ms if flush is not None else start.elapsed_time(end)) / a.steps)
    z0, nz, stride = error_sample(w)
    sample = vol[z0:z0 + nz, ::stride, ::stride].cpu().numpy()
    out = {"value": w.updates * world / (ms / 1000.0) / 1e9, "ms_per_step": ms, "s_per_volume": ms / 1000.0,
           "stages_ms": {"preprocess_weight_filter": statistics.mean(s[0] for s in stage_ms),
                         "backprojection_hu": statistics.mean(s[2] for s in stage_ms)},
           "gpu_launches": launches, "clocks": clk, "tile_depth": eng.tile_depth, "_sample": sample}

    # end to end through the host-buffer call, pinned memory
    if not a.no_e2e:
        raw_h = torch.empty(raw.shape, dtype=torch.uint16, pin_memory=True)
        raw_h.copy_(raw.cpu())
        out_h = torch.empty(vol.shape, dtype=torch.float32, pin_memory=True)
        raw_np, out_np = raw_h.numpy(), out_h.numpy()
        eng.reconstruct_host(raw_np, out_np)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = eng.kernel_launches
        s2.record()
        for _ in range(a.steps):
            eng.reconstruct_host(raw_np, out_np)
        e2.record()
        torch.cuda.synchronize()
        out["gpu_launches"] += eng.kernel_launches - l0
        ems = max_over_ranks(dist, s2.elapsed_time(e2) / a.steps)
        out["e2e"] = {"value": w.updates * world / (ems / 1000.0) / 1e9, "unit": "GUPS",
                      "h2d_bytes_per_step": int(raw.numel() * 2), "d2h_bytes_per_step": int(vol.numel() * 4),
                      "ms_per_step": ems}
    eng.close()
    return out


def gather_ceiling(record_bytes: int, with_taper: bool, distinct: int, warps_per_sm: int = 32):
    """Samples per second the load path delivers for the backprojector's
    fetch pattern (jfdk_measure_gather_rate, measured here on this GPU)."""
    import ctypes as C
    from jenhine_b200 import _lib
    r = C.c_double()
    st = _lib.load().jfdk_measure_gather_rate(record_bytes, int(with_taper), distinct, warps_per_sm, C.byref(r))
    return r.value if st == 0 else None


def roofline(w, bp_ms, form, clocks):
    """The backprojector (the dominant kernel) against the bounds that bind
    it, from its CUDA-event time:
      issue  -- SMs x 4 schedulers x the SM clock sampled during the run,
                over the warp instructions it issues per 32 updates (ncu, the
                same build, profiles/<kernel>_c2_chunks.md);
      gather -- the samples per second the load path delivers for its fetch
                pattern (record bytes, taper pair, records per warp request
                from the same profile), measured live by a microbenchmark;
      hbm    -- algorithmic bytes (filtered projections read once at 4 bytes
                (FP32) or 2 bytes (FP16) a pixel, the normalisation weights
                read and the volume written once)
                against the measured copy bandwidth, with the DRAM traffic
                of a full-size launch (ncu, profiles/<kernel>_c2.md).
    frac is the issue fraction: the kernel's binding bound."""
    import torch
    kernel = "bp_kernel" if form == "fp32" else "bp_mixed_kernel"
    prof = f"{kernel}_{w.name}"
    r, g = w.recon, w.geom
    gups = w.updates / (bp_ms / 1000.0) / 1e9
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    w32 = profile_figure(f"{kernel}_c2_chunks", "warp_instructions_per_32_updates")
    # one record per sample, the weights read once from the per-geometry
    # volume: a 16-byte FP32 quad, or an 8-byte FP16 record (mixed)
    rec = 16 if form == "fp32" else 8
    per_req = profile_figure(f"{kernel}_c2_chunks", "records_per_request") or 6.0
    warps = int(profile_figure(f"{kernel}_c2_chunks", "warps_per_sm") or 32)
    gather = gather_ceiling(rec, False, max(1, min(32, int(round(per_req)))), warps)
    peak, peak_kind = measured_peaks()
    # projections once (4 / 2 bytes a pixel), the weights read and the volume written once
    alg = g.n_views * g.det_v * g.det_u * (4 if form == "fp32" else 2) + 2 * r.num_pixels_x * r.num_pixels_y * \
        r.num_pixels_z * 4
    hbm = alg / (bp_ms / 1000.0) / 1e9
    out = {"kernel": f"{kernel} (backprojection + normalisation + CT numbers)", "bound": "issue",
           "achieved": gups, "unit": "GUPS (voxel-view updates/s)"}
    if w32:
        ceiling = sms * 4 * mhz * 1e6 * 32.0 / w32 / 1e9
        out.update({"peak": ceiling, "frac": gups / ceiling,
                    "peak_source": f"issue ceiling: {sms} SMs x 4 schedulers x {mhz:.0f} MHz (sampled) / {w32:.2f} "
                                   f"warp instructions per 32 updates (ncu, profiles/{kernel}_c2_chunks.md)"})
    else:
        out.update({"peak": None, "frac": None, "peak_source": "no instruction count committed for this kernel"})
    out["gather"] = {"peak": gather / 1e9 if gather else None, "achieved": gups,
                     "frac": gups / (gather / 1e9) if gather else None, "unit": "G samples/s",
                     "pattern": f"one {rec}-byte record per sample, {per_req:g} records per warp request, "
                                f"{warps} warps per SM, L1-resident (jfdk_measure_gather_rate, this run)"}
    out["hbm"] = {"achieved": hbm, "peak": peak, "frac": hbm / peak, "unit": "GB/s",
                  "peak_source": f"{peak_kind} hbm_gbs ({'of measured' if peak_kind == 'measured' else 'of fallback'})",
                  "algorithmic_bytes_per_launch": alg, "traffic": profile_traffic(prof)}
    return out


def run_batch(a, rank, world, local):
    """--workload batch: 16 seeded scans of uneven size (workloads.batch()),
    reconstructed (a) one jfdk_reconstruct launch sequence per scan and (b) as
    one batch -- every scan's filter stage and one persistent backprojection,
    replayed as a CUDA graph.  value = aggregate GUPS of (b)."""
    import torch
    from jenhine_b200.fdk import FDKBatch, FDKEngine
    from jenhine_b200.workloads import batch
    if a.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the batch workload is timed on the GPU engine only; "
                                                                  "the reference arm runs the c2 workload"}), flush=True)
        return
    torch.cuda.set_device(local)
    dist = init_dist(world, local)
    scans = batch()
    for w in scans:
        w.geom.seed += 1000 * rank
    updates = sum(w.updates for w in scans)
    raws = [w.raw_torch() for w in scans]
    forms = ["fp32", "mixed"] if a.precision == "both" else [a.precision]
    res = {}
    def time_schedule(b, outs):
        for _ in range(a.warmup):
            b.run(raws, outs)
        torch.cuda.synchronize()
        s1, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s1.record()
        for _ in range(a.steps):
            b.run(raws, outs)
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(dist, s1.elapsed_time(e1) / a.steps)

    for form in forms:
        engines = [FDKEngine(w.scan, w.recon, w.geom.ptms(), precision=form) for w in scans]
        b = FDKBatch(engines, autotune=True, graph=True)
        outs = [torch.empty((w.recon.num_pixels_z, w.recon.num_pixels_y, w.recon.num_pixels_x), device="cuda")
                for w in scans]
        ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
        # one launch sequence per scan
        for _ in range(a.warmup):
            for e, r, o in zip(engines, raws, outs):
                e.reconstruct(r, o)
        torch.cuda.synchronize()
        s0, e0 = ev(), ev()
        s0.record()
        for _ in range(a.steps):
            for e, r, o in zip(engines, raws, outs):
                e.reconstruct(r, o)
        e0.record()
        torch.cuda.synchronize()
        single_ms = max_over_ranks(dist, s0.elapsed_time(e0) / a.steps)
        # one batch: direct run + graph recording, then replays
        for _ in range(a.warmup):
            b.run(raws, outs)
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.5)
        l0 = b.launches
        s1, e1 = ev(), ev()
        s1.record()
        for _ in range(a.steps):
            b.run(raws, outs)
        e1.record()
        torch.cuda.synchronize()
        clk = clocks.stop()
        batch_ms = max_over_ranks(dist, s1.elapsed_time(e1) / a.steps)
        chosen = b.schedule
        launched = b.launches - l0
        b.close()
        # both schedules, each fixed (the tuned choice above is one of them)
        sched = {}
        for name in ("persistent", "pipelined"):
            bs = FDKBatch(engines, autotune=False, graph=True, schedule=name)
            ms = time_schedule(bs, outs)
            sched[name] = {"value": updates * world / (ms / 1000.0) / 1e9, "ms_per_step": ms}
            bs.close()
        res[form] = {"value": updates * world / (batch_ms / 1000.0) / 1e9, "ms_per_step": batch_ms,
                     "schedule": chosen, "schedules": sched,
                     "one_launch_each": {"value": updates * world / (single_ms / 1000.0) / 1e9,
                                         "ms_per_step": single_ms},
                     "speedup_vs_one_launch_each": single_ms / batch_ms,
                     "gpu_launches": launched, "clocks": clk}
        for e in engines:
            e.close()
    if rank == 0:
        head = res[forms[0]]
        line = {"metric": "aggregate GUPS, 16 seeded scans of uneven size: one graph-replayed batch "
                          "(schedule picked by the autotuner: persistent backprojection or pipelined per-scan "
                          "launches) vs one launch sequence per scan",
                "value": head["value"], "unit": "GUPS", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": DATA,
                "config": {"workload": "batch: " + ", ".join(
                    f"{w.recon.num_pixels_x}x{w.recon.num_pixels_y}x{w.recon.num_pixels_z}/{w.geom.n_views}v/"
                    f"{w.geom.det_u}" for w in scans), "updates_per_step": updates, "precision": forms[0],
                    "l2": "inputs larger than L2"},
                "schedule": head["schedule"], "schedules": head["schedules"],
                "one_launch_each": head["one_launch_each"],
                "speedup_vs_one_launch_each": head["speedup_vs_one_launch_each"],
                "gpu_launches": head["gpu_launches"], "clocks": head["clocks"]}
        if len(forms) == 2:
            line["forms"] = res
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def batch_summary(local, form: str = "mixed", steps: int = 3, warmup: int = 3):
    """The 16-scan batch workload in one form, autotuned and graph-replayed
    (the schedule the autotuner keeps), for the default line's `batch` key;
    the comparison of schedules is `--workload batch`."""
    import torch
    from jenhine_b200.fdk import FDKBatch, FDKEngine
    from jenhine_b200.workloads import batch
    scans = batch()
    updates = sum(w.updates for w in scans)
    raws = [w.raw_torch() for w in scans]
    engines = [FDKEngine(w.scan, w.recon, w.geom.ptms(), precision=form) for w in scans]
    outs = [torch.empty((w.recon.num_pixels_z, w.recon.num_pixels_y, w.recon.num_pixels_x), device="cuda")
            for w in scans]
    b = FDKBatch(engines, autotune=True, graph=True)
    try:
        for _ in range(warmup):   # the first run times both schedules and records the graph
            b.run(raws, outs)
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.5)
        l0 = b.launches
        s1, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s1.record()
        for _ in range(steps):
            b.run(raws, outs)
        e1.record()
        torch.cuda.synchronize()
        clk = clocks.stop()
        ms = s1.elapsed_time(e1) / steps
        return {"value": updates / (ms / 1000.0) / 1e9, "unit": "GUPS", "ms_per_step": ms, "steps": steps,
                "warmup": warmup, "precision": form, "schedule": b.schedule, "gpu_launches": b.launches - l0,
                "clocks": clk, "updates_per_step": updates,
                "workload": "16 seeded scans of uneven size (bench.py --workload batch), one graph-replayed batch"}
    finally:
        b.close()
        for e in engines:
            e.close()


def run_grad(a, rank, world, local):
    """--workload grad: the differentiation case (c3: 256^3 at 0.4 mm from 360
    views of 512^2).  One step = the loss ||FDK(p; theta) - V_target||^2 and
    its gradient with respect to the preprocessed projections p and the 6
    rigid parameters per view theta: forward filter + backprojection under
    the moved geometry, then per chunk of views the adjoint backprojection,
    the adjoint filter and the geometry gradient (jenhine_b200.autograd).
    value = voxel-view updates of the three backprojection-sized passes
    (forward, adjoint, gradient) per second."""
    import numpy as np
    import torch
    from jenhine_b200.autograd import FDKFunction
    from jenhine_b200.fdk import FDKEngine
    from jenhine_b200.motion import seeded_motion
    from jenhine_b200.workloads import c3
    if a.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no derivatives "
                                                                  "(no adjoint backprojector, filter or geometry "
                                                                  "gradient)"}), flush=True)
        return
    torch.cuda.set_device(local)
    dist = init_dist(world, local)
    w = c3()
    w.geom.seed += 1000 * rank
    P0 = np.asarray(w.geom.ptms(), np.float32)
    eng = FDKEngine(w.scan, w.recon, P0)
    p = eng.preprocess(w.raw_torch()).contiguous()
    nv = p.shape[0]
    target = FDKFunction.apply(p, torch.zeros((nv, 6), dtype=torch.float64), eng, P0).detach().clone()
    seen = torch.isfinite(target)
    target = torch.nan_to_num(target)
    theta = torch.from_numpy(seeded_motion(nv, 303)).requires_grad_()
    pp = p.clone().requires_grad_()

    def step():
        vol = FDKFunction.apply(pp, theta, eng, P0)
        loss = torch.where(seen & torch.isfinite(vol), vol - target, 0.0).square().sum()
        pp.grad = None
        theta.grad = None
        loss.backward()
        return loss

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    l0 = eng.kernel_launches
    s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(a.steps):
        loss = step()
    e0.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(dist, s0.elapsed_time(e0) / a.steps)
    g_theta = theta.grad.detach().cpu().numpy()
    if rank == 0:
        upd = 3 * w.updates * world
        print(json.dumps({
            "metric": "gradient of ||FDK(p; theta) - V_target||^2 w.r.t. projections and 6 rigid parameters "
                      "per view: voxel-view updates/s of forward + adjoint + geometry-gradient passes",
            "value": upd / (ms / 1000.0) / 1e9, "unit": "GUPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": DATA,
            "config": {"workload": "c3: 256x256x256 at 0.4 mm from 360 views of 512x512, seeded rigid motion "
                                   "+/-0.5 mm / +/-0.3 deg", "updates_per_pass": w.updates, "passes": 3,
                       "l2": "inputs larger than L2 (projections 377 MB, quad store 1.5 GB)"},
            "loss": float(loss.item()), "grad_theta_norm": float(np.linalg.norm(g_theta)),
            "gpu_launches": eng.kernel_launches - l0, "clocks": clk}), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from jenhine_b200.workloads import WORKLOADS
    if a.workload == "batch":
        run_batch(a, rank, world, local)
        return
    if a.workload == "grad":
        run_grad(a, rank, world, local)
        return
    w = WORKLOADS[a.workload]()
    if a.impl == "reference":
        run_reference(a, w, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = init_dist(world, local)
    forms = ["fp32", "mixed"] if a.precision == "both" else [a.precision]
    if a.split == "zslab":
        # one volume shared by all ranks
        raw = w.raw_torch()
        ptms = w.geom.ptms()
        res = {f: time_zslab(a, w, raw, ptms, f, dist, rank, world, local) for f in forms}
        if rank == 0:
            head = res[forms[0]]
            line = {"metric": METRIC, "value": head["value"], "unit": "GUPS", "n_gpus": world,
                    "steps": a.steps, "warmup": a.warmup, "ms_per_step": head["ms_per_step"],
                    "s_per_volume": head["s_per_volume"], "higher_is_better": True, "scaling": "strong",
                    "vs_baseline": None, "dtype": "f32", "data": DATA,
                    "config": dict(workload_config(w), precision=forms[0],
                                   parallelism=f"one volume in z-slabs over {world} GPUs"),
                    "gpu_launches": sum(r["gpu_launches"] for r in res.values()), "clocks": head["clocks"]}
            if len(forms) == 2:
                line["forms"] = res
            print(json.dumps(line), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    # each rank reconstructs its own scan
    w.geom.seed += 1000 * rank
    raw = w.raw_torch()
    ptms = w.geom.ptms()
    res = {f: time_form(a, w, raw, ptms, f, dist, world, local) for f in forms}
    samples = {f: res[f].pop("_sample") for f in forms}

    if rank == 0:
        head = res[forms[0]]
        line = {
            "metric": METRIC, "value": head["value"], "unit": "GUPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": head["ms_per_step"], "s_per_volume": head["s_per_volume"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA,
            "config": dict(workload_config(w), precision=forms[0],
                           forms="value/e2e: the plain FP32 form; forms.mixed: the mixed-precision form"
                           if len(forms) == 2 else forms[0],
                           bp_rounding="bpcore-exact" if a.exact else "fast",
                           parallelism=f"{world} independent scans, one per GPU"),
            "stages_ms": head["stages_ms"],
            "roofline": roofline(w, head["stages_ms"]["backprojection_hu"], forms[0], head["clocks"]),
            "gpu_launches": sum(r["gpu_launches"] for r in res.values()),
            "clocks": head["clocks"],
        }
        if "e2e" in head:
            line["e2e"] = head["e2e"]
        if len(forms) == 2:
            m = dict(res["mixed"])
            m["roofline"] = roofline(w, m["stages_ms"]["backprojection_hu"], "mixed", m["clocks"])
            m["speedup_vs_fp32"] = head["ms_per_step"] / m["ms_per_step"]
            line["forms"] = {"fp32": {k: v for k, v in head.items()}, "mixed": m}
        if not a.no_gpu_baseline and world == 1 and not w.composite:
            gb = gpu_baseline(w, raw, ptms, local)
            if gb is not None:
                line["gpu_baseline"] = gb
        if not a.no_batch and world == 1 and a.workload == "c2" and "mixed" in forms:
            try:
                line["batch"] = batch_summary(local)
            except Exception as ex:   # the extra key must not cost the line
                line["batch"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
        if not a.no_cpu_baseline and world == 1 and not w.composite:
            # the CPU leg (rank 0, one GPU): the reference Cores timed on the
            # host, and each form's error against the FP64 oracle
            from jenhine_b200.fdk import FDKEngine
            g = w.geom
            full = cpu_full(w)
            nvb = g.n_views if full else min(60, g.n_views)
            raw_np = raw.cpu().numpy() if full else raw[:12].cpu().numpy()
            filt = None
            if not full:
                eng = FDKEngine(w.scan, w.recon, ptms)
                filt = eng.filter(eng.preprocess(raw[:nvb]), 0).cpu().numpy()
                eng.close()
            gups, cores, kind, sample, spent, _, extrap = cpu_sample(w, raw_np, filt, ptms)
            line["cpu_baseline"] = {"value": gups, "unit": "GUPS", "cores": cores, "kind": kind,
                                    "sample": sample, "seconds": spent, "extrapolated": extrap, **CPU_NOTES}
            errs = fp64_errors(w, raw.cpu().numpy(), samples)
            line["error_vs_fp64"] = {"sample": errs["sample"], "oracle": errs["oracle"], **errs[forms[0]]}
            if len(forms) == 2:
                line["forms"]["mixed"]["error_vs_fp64"] = errs["mixed"]
                line["forms"]["fp32"]["error_vs_fp64"] = errs["fp32"]
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
