#!/usr/bin/env python
"""bench.py — FBP voxel-angle updates/s of the B200 backend (one JSON line).

Workload (default, "large"): a 512^3 float32 phantom of 32 seeded random
ellipsoids (rotated, summed inside the unit sphere), 720 angles on [0, pi),
Nd = ceil(sqrt(2) 512) rounded up to odd = 725 detector bins, Shepp-Logan
filter. One step = the whole reconstructVolume path on the device: per-slice
statistics, forward projection of all 512 slices, ramp filtering, backprojection
and denormalisation. updates = N^2 * slices * angles per volume. Synthetic
data (no dataset involved); the volume (0.54 GB) exceeds the 126 MB L2, so no
flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config small|large|medium|precision|tcprof|batch|serving]

N > 1 runs under torch.distributed.run, one rank per GPU, each rank
reconstructing its own volume (weak scaling; no data-path collective).
--impl reference times the reference's own CPU implementation of the path
(OpenMPBackend built from its sources, oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "small": dict(n=128, nz=128, na=180, ellipsoids=10, filter=0, seed=1,
                  name="128^3 phantom (10 ellipsoids), 180 angles, Ram-Lak"),
    "large": dict(n=512, nz=512, na=720, ellipsoids=32, filter=1, seed=2,
                  name="512^3 phantom (32 ellipsoids), 720 angles, Shepp-Logan"),
    "medium": dict(n=384, nz=384, na=540, ellipsoids=24, filter=1, seed=4,
                   name="384^3 phantom (24 ellipsoids), 540 angles, Shepp-Logan (profiling size)"),
    "precision": dict(n=1024, nz=256, na=1440, ellipsoids=64, filter=4, seed=3,
                      name="1024^2 x 256 phantom (64 ellipsoids), 1440 angles, Hann"),
    "tcprof": dict(n=1024, nz=16, na=1440, ellipsoids=64, filter=4, seed=3,
                   name="1024^2 x 16 slices, 1440 angles, Hann (profiling size of the filter kernels)"),
    "batch": dict(jobs=64, seed=4,
                  name="64 uneven FBP jobs: N in {64..768}, 16-256 slices, round(pi/2 N) angles, "
                       "Ram-Lak/Shepp-Logan/Hann, sinograms of seeded 10-ellipsoid phantoms"),
    "serving": dict(requests=48, seed=5, big_fraction=0.1, budget_gb=120, copy_threads=4, rates=[0.5, 1.0, 2.0, 4.0],
                    name="Poisson stream of FBP requests: 90% the batch mix, 10% 1024^2 x 64 x 1440 angles; "
                         "host sinograms in, host volumes out; 120 GB device budget"),
}
FILTER_NAMES = ["ramlak", "shepp-logan", "hamming", "cosine", "hann", "bartlett"]
METRIC = "FBP voxel-angle updates/s"
UNIT = "updates/s"


def odd_nd(n: int) -> int:
    nd = math.ceil(math.sqrt(2.0) * n)
    return nd + 1 if nd % 2 == 0 else nd


def image_support(vol):
    """Pixels the forward projector must read, from the host volume (z, y, x):
    the non-zero normalised pixels (raw != 0 and raw != the slice minimum;
    every other pixel contributes an exact zero, as the reference's skip of
    raw == 0 does), and the pixels of the per-8-slice-group bounding boxes of
    those, an upper bound of what the projector walks."""
    import numpy as np
    nz = vol.shape[0]
    lo = vol.reshape(nz, -1).min(axis=1)
    nnz = 0
    walked = 0
    for g in range(0, nz, 8):
        blk = vol[g:g + 8]
        m = (blk != 0) & (blk != lo[g:g + 8, None, None])
        nnz += int(m.sum())
        u = m.any(axis=0)
        rows, cols = np.flatnonzero(u.any(axis=1)), np.flatnonzero(u.any(axis=0))
        if rows.size:
            walked += (rows[-1] - rows[0] + 1) * (cols[-1] - cols[0] + 1) * blk.shape[0]
    return nnz, walked


def circle_voxels(n: int) -> int:
    """Voxels the reference reconstructs: xx^2 + yy^2 <= r^2 with r = n//2."""
    r = n // 2
    c = 0
    for y in range(n):
        yy = y - r
        rem = r * r - yy * yy
        if rem < 0:
            continue
        s = math.isqrt(rem)
        c += max(0, min(n - 1, r + s) - max(0, r - s) + 1)
    return c


# ---------------------------------------------------------------- accuracy
ACC_GATE = {"rel_l2": 1e-5, "max_abs": 1e-4}


def accuracy_slices(nz: int, n: int):
    """Slices whose output is checked: both sides of the first and last slab
    boundaries of the host pipeline's schedule (8, 24, 64, ..., 64, 24, 8
    slices at 512), which are 8-slice group boundaries too, the middle and the
    ends (fewer at n >= 1024, where one FP64 slice takes seconds)."""
    if n >= 1024:
        zs = [0, 15, 16, nz // 2 - 1, nz // 2, nz - 1]
    else:
        zs = [0, 7, 8, 31, 32, 95, 96, nz // 2 - 1, nz // 2, nz - 33, nz - 32, nz - 9, nz - 8, nz - 1]
    return sorted({z for z in zs if 0 <= z < nz})


def accuracy_report(vol_host, outputs: dict, na: int, nd: int, kind: int, zs):
    """Error of each reconstructed volume in `outputs` (name -> (nz, n, n)
    array) on the slices `zs` against the FP64 rerun of SerialBackend's
    reconstructVolume (oracle, per slice: slices are independent), and against
    SerialBackend's own float path (reported, not gated: at n = 512 the float
    reference itself is ~3e-5 from FP64). Worst slice of each. The oracle
    calls run in threads (they release the GIL)."""
    import concurrent.futures as cf

    import numpy as np

    import oracle as O

    def one(z, f64):
        v = np.ascontiguousarray(vol_host[z:z + 1])
        return (O.reconstruct_volume_f64 if f64 else O.reconstruct_volume_f32)(v, na, nd, kind)[0]

    with cf.ThreadPoolExecutor(max_workers=max(1, min(2 * len(zs), os.cpu_count() or 1))) as ex:
        f64 = dict(zip(zs, ex.map(lambda z: one(z, True), zs)))
        f32 = dict(zip(zs, ex.map(lambda z: one(z, False), zs)))
    rep = {"slices": list(zs), "gate_vs_fp64": ACC_GATE,
           "reference": "FP64 rerun of SerialBackend::reconstructVolume (oracle); serial = its float path",
           "serial_vs_fp64": {"rel_l2": max(O.rel_l2(f32[z], f64[z]) for z in zs),
                              "max_abs": max(O.max_abs_rel(f32[z], f64[z]) for z in zs)}}
    for name, out in outputs.items():
        r = {"rel_l2_vs_fp64": max(O.rel_l2(out[z], f64[z]) for z in zs),
             "max_abs_vs_fp64": max(O.max_abs_rel(out[z], f64[z]) for z in zs),
             "rel_l2_vs_serial": max(O.rel_l2(out[z], f32[z]) for z in zs),
             "max_abs_vs_serial": max(O.max_abs_rel(out[z], f32[z]) for z in zs)}
        r["pass"] = r["rel_l2_vs_fp64"] <= ACC_GATE["rel_l2"] and r["max_abs_vs_fp64"] <= ACC_GATE["max_abs"]
        rep[name] = r
    return rep


def fft_fp32_roofline(nd: int, sq: int, nz: int, na: int, ms: float):
    """The filter's arithmetic against the FP32 pipe: the nominal 5 L log2 L
    flops of a complex FFT of the convolution length L = nextPow2(sq + nd - 1),
    a forward and an inverse transform plus the 6 L of the spectrum product per
    pair of rows (two real rows travel as one complex sequence), against
    148 SMs x 128 lanes x 2 flops x 1.965 GHz (the B200's FP32 FMA peak at its
    maximum clock; packed FP32x2 instructions do not raise it)."""
    L = 64
    while L < sq + nd - 1:
        L *= 2
    flops = ((nz + 1) // 2) * na * (2 * 5 * L * math.log2(L) + 6 * L)
    peak = 148 * 128 * 2 * 1.965e9 / 1e12
    achieved = flops / (ms * 1e-3) / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "algorithmic": f"nominal FFT flops: 2 x 5 L log2 L + 6 L per row pair, L = {L}",
            "peak_source": "nominal FP32 FMA peak of a B200 at 1965 MHz (148 SMs)"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str, period_ms: int = 100):
        self.rows = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(period_ms)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        if not self.rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def gpu_id_for(device: int) -> str:
    import torch
    try:
        u = str(torch.cuda.get_device_properties(device).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        return vis.split(",")[device] if vis else str(device)


def load_profile_traffic(kernel: str, config: str):
    """DRAM bytes per launch of `kernel` ("forward", "backproject") from the
    committed ncu summary (JSON text), if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{config}_traffic.txt")
    try:
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


# Peaks measured earlier on B200s of the same configuration, used only when
# MEASURED_PEAKS.json is absent (a STREAM-style copy; a cuBLAS bf16 GEMM as a
# burst and under the power cap in a seconds-long loop).
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def measured_peaks():
    """The measured denominators, with "_label" = "of measured"; the recipe's
    fallback figures, labelled "of fallback", when the file is absent."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        d["_label"] = "MEASURED_PEAKS.json (of measured)"
        return d
    except (OSError, ValueError):
        d = dict(FALLBACK_PEAKS)
        d["_label"] = "fallback peaks, MEASURED_PEAKS.json absent (of fallback)"
        return d


# ------------------------------------------------------------------ ranks
def max_over_ranks(dist, values, device):
    """Element-wise maximum of per-rank timings; every rank calls it at the
    same point (a no-op without a process group)."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_throughput(world: int, units_per_rank: float, ms: float) -> float:
    """Whole-job rate of `world` replicas, each processing `units_per_rank`
    in at most `ms` (the max over ranks)."""
    return world * units_per_rank / (ms * 1e-3)


# ------------------------------------------------------------- CPU baseline
def cpu_reference_rate(cfg: dict, slices: int, params, repeats: int = 3):
    """The reference's OpenMPBackend per-slice path (computeSinogram with the
    config's odd detector + reconstructSlice) on `slices` central slices of the
    phantom, all host threads, after one warm-up slice; the median of
    `repeats` timed runs. Returns (updates/s, threads, kind, isa, sample)."""
    import numpy as np

    import oracle as O
    from oracle import reference as R
    n, nz, na, kind = cfg["n"], cfg["nz"], cfg["na"], cfg["filter"]
    nd = odd_nd(n)
    z0 = nz // 2 - slices // 2
    vol = O.phantom_sum_slab(params, n, n, nz, z0, slices)
    lib, isa = R.timing_lib()
    if lib is None:
        # reference not built: the float restatement of SerialBackend (1 thread)
        t0 = time.perf_counter()
        for z in range(slices):
            s, a, mm = O.sinogram_f32(vol[z], na, nd)
            O.reconstruct_slice_f32(s, a, n, kind)
        dt = time.perf_counter() - t0
        return n * n * slices * na / dt, 1, "port", "x86-64", f"{slices} slices (SerialBackend restatement)"
    threads = os.cpu_count() or 1
    lib.ref_set_threads(threads)
    # warm-up on one slice
    s, a, mm = R.compute_sinogram(R.OPENMP, vol[0], na, nd, lib=lib)
    R.reconstruct_slice(R.OPENMP, s, a, n, kind, mm[0], mm[1], lib=lib)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        for z in range(slices):
            s, a, mm = R.compute_sinogram(R.OPENMP, vol[z], na, nd, lib=lib)
            R.reconstruct_slice(R.OPENMP, s, a, n, kind, mm[0], mm[1], lib=lib)
        times.append(time.perf_counter() - t0)
    sample = (f"{slices} central of {nz} slices, OpenMPBackend computeSinogram(nd={nd}) + reconstructSlice, "
              f"{isa}, median of {repeats} runs")
    return n * n * slices * na / statistics.median(times), threads, "reference", isa, sample


def cpu_native_rate(cfg: dict, slices: int, params, repeats: int = 3):
    """The reference OpenMPBackend's own reconstructVolume (its native volume
    path: detector bins = N, symmetric-z SIMD backprojection) on `slices`
    slices of the phantom, all host threads; the median of `repeats` runs.
    Returns (updates/s, threads) or None when the reference build is absent."""
    import oracle as O
    from oracle import reference as R
    lib, _ = R.timing_lib()
    if lib is None:
        return None
    n, nz, na, kind = cfg["n"], cfg["nz"], cfg["na"], cfg["filter"]
    vol = O.phantom_sum_slab(params, n, n, nz, nz // 2 - slices // 2, slices)
    threads = os.cpu_count() or 1
    lib.ref_set_threads(threads)
    R.reconstruct_volume(R.OPENMP, vol[:2], na, kind, lib=lib)  # warm-up
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        R.reconstruct_volume(R.OPENMP, vol, na, kind, lib=lib)
        times.append(time.perf_counter() - t0)
    return n * n * slices * na / statistics.median(times), threads


def cpu_serial_rate(cfg: dict, slices: int, params, repeats: int = 3):
    """The reference SerialBackend's own reconstructVolume (one thread, its
    native path with detector bins = N) on `slices` central slices of the
    phantom, median of `repeats` runs. Returns updates/s or None when the
    reference build is absent."""
    import oracle as O
    from oracle import reference as R
    lib, _ = R.timing_lib()
    if lib is None:
        return None
    n, nz, na, kind = cfg["n"], cfg["nz"], cfg["na"], cfg["filter"]
    vol = O.phantom_sum_slab(params, n, n, nz, nz // 2 - slices // 2, slices)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        R.reconstruct_volume(R.SERIAL, vol, na, kind, lib=lib)
        times.append(time.perf_counter() - t0)
    return n * n * slices * na / statistics.median(times)


def run_reference(args, cfg, rank: int, world: int):
    """--impl reference: the reference's CPU path, rank 0 only."""
    if rank != 0:
        return 0
    import oracle as O  # the phantom's seeded parameter draw; the product library is never loaded
    params = O.phantom_params(cfg["seed"], cfg["ellipsoids"])
    n, nz, na = cfg["n"], cfg["nz"], cfg["na"]
    slices = args.ref_slices
    for _ in range(args.warmup if args.warmup < 2 else 1):
        cpu_reference_rate(cfg, 1, params)
    rates = []
    threads, kind, isa, sample = 1, "port", "", ""
    for _ in range(args.steps):
        r, threads, kind, isa, sample = cpu_reference_rate(cfg, slices, params, repeats=1)
        rates.append(r)
    sample = sample.replace("median of 1 runs", f"median over {args.steps} steps")
    value = statistics.median(rates)
    step_ms = n * n * slices * na / value * 1e3
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": args.config, "description": cfg["name"], "n": n, "slices": nz,
                   "angles": na, "detector_bins": odd_nd(n), "filter": FILTER_NAMES[cfg["filter"]],
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- ours
def run_ours(args, cfg, rank: int, world: int, local: int):
    import numpy as np
    import torch

    import qtctreconstruction_b200 as ctb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device(f"cuda:{local}"))
    n, nz, na, kind = cfg["n"], cfg["nz"], cfg["na"], cfg["filter"]
    nd = odd_nd(n)
    updates = n * n * nz * na
    be = ctb.B200Backend(local)
    # a dedicated (non-legacy) stream: the library and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    be.set_stream(stream.cuda_stream)
    be.set_profiling(True)

    params = ctb.phantom_params(cfg["seed"], cfg["ellipsoids"])
    vol = torch.empty((nz, n, n), dtype=torch.float32, device="cuda")
    out = torch.empty_like(vol)
    be.phantom_d(params, n, n, nz, vol.data_ptr())
    # the phantom kernel's own device time (events around its launch), after a warm-up
    phantom_ms = []
    for _ in range(3):
        be.phantom_d(params, n, n, nz, out.data_ptr())
        phantom_ms.append(be.last_phantom_ms())
    phantom_ms = statistics.median(phantom_ms)

    def step():
        be.reconstruct_volume_d(vol.data_ptr(), n, nz, na, nd, kind, out.data_ptr())

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing
    sampler = ClockSampler(gpu_id_for(local))
    barrier()
    l0 = be.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = be.launch_count() - l0
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    stages = np.mean([be.stage_times(back) for back in range(args.steps)], axis=0)
    filt_kernel_ms = float(np.mean([be.filter_kernel_ms(back) for back in range(args.steps)]))

    # ---- end to end through the host-buffer C ABI call (pinned host buffers)
    hin = torch.empty((nz, n, n), dtype=torch.float32, pin_memory=True)
    hin.copy_(vol.cpu())
    hout = torch.empty_like(hin, pin_memory=True)
    vol_host_ptr, out_host_ptr = hin.data_ptr(), hout.data_ptr()

    def e2e_step():
        be.reconstruct_volume_host(vol_host_ptr, n, nz, na, nd, kind, out_host_ptr)

    e2e_step()
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(3, args.steps // 4)
    e2.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e2.elapsed_time(e3) / e2e_steps

    # ---- the forward projector walking the whole image (bounds off), for
    # comparison with the bounded walk timed above; same results
    be.set_forward_bounds(False)
    step()
    nb = 3
    for _ in range(nb):
        step()
    torch.cuda.synchronize()
    fwd_whole_ms = float(np.mean([be.stage_times(back)[1] for back in range(nb)]))
    be.set_forward_bounds(True)

    ms, e2e_ms = max_over_ranks(dist, [ms, e2e_ms], "cuda")

    if rank == 0:
        # accuracy of the timed outputs themselves: the device-resident step's
        # volume and the end-to-end call's host volume
        acc = None
        if not args.no_accuracy:
            acc = accuracy_report(hin.numpy(), {"device": out.cpu().numpy(), "e2e": hout.numpy()}, na, nd, kind,
                                  accuracy_slices(nz, n))
        value = replica_throughput(world, updates, ms)
        smem_gbs = be.probe_smem_bandwidth()
        inside = circle_voxels(n) * nz * na
        bp_ms = float(stages[3])
        achieved = inside * 8.0 / (bp_ms * 1e-3) / 1e9  # two float taps per in-circle update
        fwd_ms = float(stages[1])
        nnz, walked = image_support(hin.numpy())
        # each non-zero pixel read once per angle (the zeros contribute nothing)
        fwd_achieved = 4.0 * nnz * na / (fwd_ms * 1e-3) / 1e9
        peaks = measured_peaks()
        hbm_peak = peaks.get("hbm_gbs")
        sq = math.ceil(math.sqrt(2.0) * nd)
        filt_bytes = 4.0 * (nd + sq) * nz * na
        smem_src = "measured shared-memory load bandwidth (probe kernel, same run)"
        roof_fwd = {"kernel": "k_forward", "bound": "l1", "achieved": fwd_achieved, "peak": smem_gbs,
                    "unit": "GB/s", "frac": fwd_achieved / smem_gbs,
                    "traffic": load_profile_traffic("forward", args.config),
                    "peak_source": smem_src + "; L1 hits use the same data path",
                    "algorithmic": "4 B (one float) per non-zero pixel-angle-slice: each non-zero pixel "
                                    "read once per angle",
                    "nonzero_fraction": nnz / (n * n * nz),
                    "box_fraction": walked / (n * n * nz),
                    "ms": fwd_ms, "ms_whole_image": fwd_whole_ms,
                    "note": "the projector walks, per 8-slice group, only where its intervals meet the "
                            "bounding box, the centred disc and the 8-row-band column ranges of the non-zero "
                            "normalised pixels (at most box_fraction of the pixels); the pixels outside are "
                            "exact zeros"}
        roof_bp = {"kernel": "k_backproject", "bound": "smem", "achieved": achieved,
                   "peak": smem_gbs, "unit": "GB/s", "frac": achieved / smem_gbs,
                   "traffic": load_profile_traffic("backproject", args.config),
                   "peak_source": smem_src,
                   "algorithmic": "8 B (two float taps) per in-circle voxel-angle update"}
        # the dominant kernel of the step carries the contract's "roofline" key
        roof_main, roof_other = (roof_fwd, roof_bp) if fwd_ms >= bp_ms else (roof_bp, roof_fwd)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config, "description": cfg["name"], "n": n, "slices": nz,
                       "angles": na, "detector_bins": nd, "filter": FILTER_NAMES[kind],
                       "parallelism": f"replicas x{world}" if world > 1 else "1 gpu",
                       "l2": "inputs larger than L2 (volume 0.54 GB per step), no flush"
                       if n * n * nz * 4 > 126e6 else "inputs smaller than L2"},
            "gpu_launches": launches,
            "stage_ms": {"stats_normalize": stages[0], "forward": stages[1], "filter": stages[2],
                         "backproject": stages[3]},
            "fbp_only": {"value": updates / ((stages[2] + stages[3]) * 1e-3), "unit": UNIT,
                         "note": "filter + backprojection kernels only"},
            "forward_only": {"value": updates / ((stages[0] + stages[1]) * 1e-3), "unit": UNIT,
                             "note": "statistics, normalisation and forward projection only (N^2 slices angles "
                                     "pixel-angle updates)"},
            "roofline": roof_main,
            "roofline_" + roof_other["kernel"][2:]: roof_other,
            "roofline_phantom": {"kernel": "k_phantom_sum", "bound": "hbm",
                                 "achieved": 4.0 * n * n * nz / (phantom_ms * 1e-3) / 1e9, "peak": hbm_peak,
                                 "unit": "GB/s",
                                 "frac": (4.0 * n * n * nz / (phantom_ms * 1e-3) / 1e9 / hbm_peak) if hbm_peak else None,
                                 "ms": phantom_ms, "ellipsoids": cfg["ellipsoids"],
                                 "algorithmic": "4 B written per voxel (N^3 float32)",
                                 "peak_source": "hbm_gbs, " + peaks["_label"] if hbm_peak else None},
            "roofline_filter": {"kernel": "k_filter", "bound": "hbm",
                                "achieved": filt_bytes / (filt_kernel_ms * 1e-3) / 1e9,
                                "peak": hbm_peak, "unit": "GB/s",
                                "frac": (filt_bytes / (filt_kernel_ms * 1e-3) / 1e9 / hbm_peak) if hbm_peak else None,
                                "peak_source": "hbm_gbs, " + peaks["_label"] if hbm_peak else None,
                                "ms": filt_kernel_ms,
                                "fp32": fft_fp32_roofline(nd, sq, nz, na, filt_kernel_ms)},
            "e2e": {"value": replica_throughput(world, updates, e2e_ms), "unit": UNIT,
                    "h2d_bytes_per_step": 4 * n * n * nz, "d2h_bytes_per_step": 4 * n * n * nz,
                    "ms_per_step": e2e_ms, "api": "ctb_reconstruct_volume (pinned host buffers)"},
            "clocks": clocks,
        }
        if acc is not None:
            for k in ("rel_l2_vs_fp64", "max_abs_vs_fp64", "rel_l2_vs_serial"):
                line[k] = acc["device"][k]
            line["e2e"].update({k: acc["e2e"][k] for k in ("rel_l2_vs_fp64", "max_abs_vs_fp64", "rel_l2_vs_serial")})
            line["accuracy"] = acc
        if args.filter_modes:
            line["filter_modes"] = filter_mode_report(args, cfg, be, stream, vol, out, params, peaks)
        if world == 1 and not args.no_cpu_baseline:
            r, threads, kind_b, isa, sample = cpu_reference_rate(cfg, args.ref_slices, params)
            line["cpu_baseline"] = {"value": r, "unit": UNIT, "cores": threads, "kind": kind_b,
                                    "sample": sample}
            nat = cpu_native_rate(cfg, 2 * args.ref_slices, params)
            if nat:
                line["cpu_baseline_native"] = {
                    "value": nat[0], "unit": UNIT, "cores": nat[1], "kind": "reference",
                    "sample": f"{2 * args.ref_slices} central of {cfg['nz']} slices, "
                              "OpenMPBackend::reconstructVolume (its native volume path, detector bins = N), "
                              "median of 3 runs"}
            ser_slices = cfg["nz"] if n <= 128 else 2
            ser = cpu_serial_rate(cfg, ser_slices, params)
            if ser:
                line["cpu_baseline_serial"] = {
                    "value": ser, "unit": UNIT, "cores": 1, "kind": "reference",
                    "volume_s": n * n * nz * na / ser,
                    "sample": f"{ser_slices} of {cfg['nz']} slices, SerialBackend::reconstructVolume (one thread, "
                              "detector bins = N), median of 3 runs; volume_s scales it to the whole volume"}
        print(json.dumps(line), flush=True)
    be.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------- filter modes
def filter_mode_report(args, cfg, be, stream, vol, out, params, peaks):
    """The two filter implementations on the config's volume: device time of
    the filter stage and of its main kernel (CUDA events, profiled steps),
    the tensor-core product's roofline, and the error of each against the
    FP64 rerun of SerialBackend on two slices (sinograms from the GPU forward
    projector, reconstructed by each filter mode and by the FP64 oracle)."""
    import numpy as np
    import torch

    import oracle as O
    import qtctreconstruction_b200 as ctb
    n, nz, na, kind = cfg["n"], cfg["nz"], cfg["na"], cfg["filter"]
    nd = odd_nd(n)
    sq = math.ceil(math.sqrt(2.0) * nd)
    steps = max(3, args.steps // 2)
    rep = {}
    for name, mode in (("fft", ctb.FILTER_MODE_FFT), ("tc_bf16x3", ctb.FILTER_MODE_TC_BF16X3)):
        be.set_filter_mode(mode)
        for _ in range(2):
            be.reconstruct_volume_d(vol.data_ptr(), n, nz, na, nd, kind, out.data_ptr())
        for _ in range(steps):
            be.reconstruct_volume_d(vol.data_ptr(), n, nz, na, nd, kind, out.data_ptr())
        torch.cuda.synchronize()
        st = np.mean([be.stage_times(b) for b in range(steps)], axis=0)
        km = float(np.mean([be.filter_kernel_ms(b) for b in range(steps)]))
        rep[name] = {"filter_stage_ms": float(st[2]), "main_kernel_ms": km, "step_ms": float(np.sum(st))}
    be.set_filter_mode(ctb.FILTER_MODE_FFT)
    flops = 6 * 2.0 * nz * na * nd * sq
    tc_ms = rep["tc_bf16x3"]["main_kernel_ms"]
    # the sustained GEMM figure for a kernel inside a step of 100 ms or more
    # (the GPU settles under its power cap), the burst figure for a short one
    long_step = rep["tc_bf16x3"]["step_ms"] >= 100.0
    peak_key = "bf16_tflops_sustained" if long_step else "bf16_tflops"
    peak = peaks.get(peak_key)
    rep["tc_bf16x3"]["roofline"] = {
        "kernel": "k_filter_gemm", "bound": "tensor", "achieved": flops / (tc_ms * 1e-3) / 1e12, "peak": peak,
        "unit": "TFLOP/s", "frac": (flops / (tc_ms * 1e-3) / 1e12 / peak) if peak else None,
        "algorithmic": "6 x 2 x rows x nd x sq FLOP (six BF16 products of the three-term Toeplitz filter)",
        "peak_source": (f"{peak_key} (the kernel runs inside a {rep['tc_bf16x3']['step_ms']:.1f} ms step), "
                        + peaks["_label"])}
    # accuracy on two slices against the FP64 rerun
    z0 = nz // 2
    slab = torch.from_numpy(O.phantom_sum_slab(params, n, n, nz, z0, 2)).cuda()
    d_sino = torch.empty((2, na, nd), dtype=torch.float32, device="cuda")
    d_stats = torch.empty((2, 4), dtype=torch.float32, device="cuda")
    be.forward_d(slab.data_ptr(), n, 2, na, nd, d_sino.data_ptr(), d_stats.data_ptr())
    be.synchronize()
    sino = d_sino.cpu().numpy()
    ang = O.uniform_angles_deg(na)
    f64 = [O.reconstruct_slice_f64(sino[z], ang, n, kind) for z in range(2)]
    d_out = torch.empty((2, n, n), dtype=torch.float32, device="cuda")
    for name, mode in (("fft", ctb.FILTER_MODE_FFT), ("tc_bf16x3", ctb.FILTER_MODE_TC_BF16X3)):
        be.set_filter_mode(mode)
        be.fbp_d(d_sino.data_ptr(), 2, na, nd, n, kind, d_out.data_ptr())
        be.synchronize()
        got = d_out.cpu().numpy()
        rep[name]["rel_l2_vs_fp64"] = max(O.rel_l2(got[z], f64[z]) for z in range(2))
        rep[name]["max_abs_vs_fp64"] = max(O.max_abs_rel(got[z], f64[z]) for z in range(2))
    be.set_filter_mode(ctb.FILTER_MODE_FFT)
    rep["default"] = "fft"
    rep["rule"] = "the tensor-core product is used only where it beats the FFT path at <= 1e-5 rel-L2 vs FP64"
    rep["accuracy_sample"] = f"slices {z0}, {z0 + 1}: GPU forward projection, FBP per mode vs FP64 oracle"
    return rep


# ------------------------------------------------------------------ batches
BATCH_FILTERS = (0, 1, 4)  # Ram-Lak, Shepp-Logan, Hann


def batch_shapes(seed: int, count: int):
    """The uneven job mix: N uniform in {64, 96, ..., 768}, slices uniform in
    [16, 256], angles round(pi/2 N), Nd odd >= sqrt(2) N, filter uniform over
    Ram-Lak / Shepp-Logan / Hann."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(np.arange(64, 769, 32)))
        out.append(dict(n=n, nz=int(rng.integers(16, 257)), na=int(round(math.pi / 2 * n)), nd=odd_nd(n),
                        filter=int(rng.choice(BATCH_FILTERS))))
    return out


def make_batch_inputs(be, torch, shapes, seed: int):
    """Device sinograms of seeded random-ellipsoid phantoms (forward-projected
    on the GPU) and output buffers for every job."""
    import qtctreconstruction_b200 as ctb
    jobs, keep = [], []
    for k, s in enumerate(shapes):
        n, nz, na, nd = s["n"], s["nz"], s["na"], s["nd"]
        vol = torch.empty((nz, n, n), dtype=torch.float32, device="cuda")
        be.phantom_d(ctb.phantom_params(seed * 1000 + k, 10), n, n, nz, vol.data_ptr())
        sino = torch.empty((nz, na, nd), dtype=torch.float32, device="cuda")
        stats = torch.empty((nz, 4), dtype=torch.float32, device="cuda")
        be.forward_d(vol.data_ptr(), n, nz, na, nd, sino.data_ptr(), stats.data_ptr())
        be.synchronize()
        del vol
        out = torch.empty((nz, n, n), dtype=torch.float32, device="cuda")
        keep.append((sino, out))
        jobs.append(dict(sino=sino.data_ptr(), depth=nz, num_angles=na, bins=nd, output_size=n,
                         filter=s["filter"], out=out.data_ptr()))
    return jobs, keep


def run_batch(args, cfg, rank: int, world: int, local: int):
    """Config "batch": `jobs` uneven FBP jobs from device-resident sinograms.
    One step = every job filtered and backprojected. Timed four ways on the
    same jobs: the batch replayed from a CUDA graph (the value), the batch
    launched directly, the batch with its backprojection on the persistent work
    queue, and one filter + one backprojection launch per job. Then every
    backprojection shape alone on three of the jobs, and the batch again with
    the shapes the autotuner chose per size bucket."""
    import torch

    import qtctreconstruction_b200 as ctb
    torch.cuda.set_device(local)
    be = ctb.B200Backend(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    be.set_stream(stream.cuda_stream)
    shapes = batch_shapes(cfg["seed"], cfg["jobs"])
    jobs, keep = make_batch_inputs(be, torch, shapes, cfg["seed"])
    updates = sum(s["n"] ** 2 * s["nz"] * s["na"] for s in shapes)
    results, outputs = {}, {}
    for mode, flags in (("graph", ctb.BATCH_GRAPH), ("direct", 0),
                        ("persistent", ctb.BATCH_GRAPH | ctb.BATCH_PERSISTENT), ("per_job", ctb.BATCH_PER_JOB)):
        with be.batch(jobs, flags) as b:
            launches, _, nbytes = b.info()
            for _ in range(args.warmup):
                b.run()
            torch.cuda.synchronize()
            sampler = ClockSampler(gpu_id_for(local)) if mode == "graph" else None
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                b.run()
            e1.record(stream)
            torch.cuda.synchronize()
            be.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            results[mode] = dict(ms_per_step=ms, value=updates / (ms * 1e-3), launches_per_step=launches,
                                 device_bytes=nbytes)
            if sampler:
                results[mode]["clocks"] = sampler.stop()
            outputs[mode] = [o.sum().item() for _, o in keep[:4]]
    same = outputs["graph"] == outputs["direct"] == outputs["persistent"] == outputs["per_job"]
    # every compiled backprojection shape (tile, voxels per thread, angles per
    # chunk) timed alone on the smallest, a middle and the largest job
    def fbp_ms(j, reps=3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        be.fbp_d(j["sino"], j["depth"], j["num_angles"], j["bins"], j["output_size"], j["filter"], j["out"])
        e0.record(stream)
        for _ in range(reps):
            be.fbp_d(j["sino"], j["depth"], j["num_angles"], j["bins"], j["output_size"], j["filter"], j["out"])
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    order = sorted(range(len(shapes)), key=lambda k: shapes[k]["n"] ** 2 * shapes[k]["nz"] * shapes[k]["na"])
    shape_times = []
    for k in (order[0], order[len(order) // 2], order[-1]):
        row = {"job": shapes[k], "default_shape": be.bp_shape_for(shapes[k]["n"], shapes[k]["nz"], shapes[k]["na"])}
        for v in range(6):
            be.set_bp_shape(v)
            row[f"shape{v}_{'x'.join(str(x) for x in ctb.bp_shape_info(v))}_ms"] = fbp_ms(jobs[k])
        be.set_bp_shape(-1)
        shape_times.append(row)
    # the autotuner: the first job of each size bucket times all shapes on its
    # own data; the batch then uses the tuned shape of every tuned bucket
    be.set_autotune(True)
    for j in jobs:
        be.fbp_d(j["sino"], j["depth"], j["num_angles"], j["bins"], j["output_size"], j["filter"], j["out"])
    be.synchronize()
    table = be.autotune_table()
    with be.batch(jobs, ctb.BATCH_GRAPH) as b:
        for _ in range(args.warmup):
            b.run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            b.run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms_t = e0.elapsed_time(e1) / args.steps
    be.set_autotune(False)
    results["graph_autotuned"] = dict(ms_per_step=ms_t, value=updates / (ms_t * 1e-3))
    # accuracy of the batch's outputs at the mix's sizes: the slice with the
    # largest sinogram of the largest and of the middle job against the FP64
    # rerun (sinograms from the device, oracle in threads; a phantom of 10
    # ellipsoids leaves many slices empty)
    import concurrent.futures as cf

    import oracle as O
    with be.batch(jobs, ctb.BATCH_GRAPH) as b:
        b.run()
        torch.cuda.synchronize()

    def check(k):
        s = shapes[k]
        sino, out = keep[k]
        z = int(torch.argmax(sino.abs().sum(dim=(1, 2))))  # the slice with the most signal
        ang = O.uniform_angles_deg(s["na"])
        f64 = O.reconstruct_slice_f64(sino[z].double().cpu().numpy(), ang, s["n"], s["filter"])
        got = out[z].cpu().numpy()
        return {"job": s, "slice": z, "max_abs_fp64": float(abs(f64).max()),
                "rel_l2_vs_fp64": O.rel_l2(got, f64), "max_abs_vs_fp64": O.max_abs_rel(got, f64)}
    with cf.ThreadPoolExecutor(max_workers=2) as ex:
        accuracy = list(ex.map(check, (order[-1], order[len(order) // 2])))
    g = results["graph"]
    line = {
        "metric": METRIC, "value": g["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": g["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batch", "description": cfg["name"], "jobs": len(shapes),
                   "voxels": sum(s["n"] ** 2 * s["nz"] for s in shapes),
                   "sinogram_bytes": sum(4 * s["nz"] * s["na"] * s["nd"] for s in shapes),
                   "l2": "inputs larger than L2, no flush"},
        "gpu_launches": g["launches_per_step"] * args.steps,
        "modes": results,
        "batched_vs_per_job": results["per_job"]["ms_per_step"] / g["ms_per_step"],
        "outputs_identical_across_modes": same,
        "accuracy": accuracy,
        "autotune_table": [dict(zip(("n_bucket", "angle_bucket", "depth_bucket", "shape"), e)) for e in table],
        "shape_times": shape_times,
        "clocks": g.get("clocks"),
    }
    print(json.dumps(line), flush=True)
    be.close()
    return 0


# ------------------------------------------------------------------ serving
def serving_shapes(seed: int, count: int, big_fraction: float):
    """Request mix: (1 - big_fraction) drawn from the batch distribution, the
    rest 1024^2 x 64 slices with 1440 angles (Nd 1449), filter as the batch's."""
    import numpy as np
    rng = np.random.default_rng(seed)
    small = batch_shapes(seed + 1, count)
    out = []
    for k in range(count):
        if rng.random() < big_fraction:
            out.append(dict(n=1024, nz=64, na=1440, nd=odd_nd(1024), filter=int(rng.choice(BATCH_FILTERS))))
        else:
            out.append(small[k])
    return out


def run_plain_stream(be, reqs, arrivals):
    """One request per call (ctb_fbp on host buffers: slab-streamed copies
    overlapped with the request's own compute), in arrival order."""
    lat, t0 = [], time.perf_counter()
    for r, a in zip(reqs, arrivals):
        now = time.perf_counter() - t0
        if now < a:
            time.sleep(a - now)
        s = r["shape"]
        be.fbp_host_ptr(r["sino"].ctypes.data, s["nz"], s["na"], s["nd"], s["n"], s["filter"], r["out"].ctypes.data)
        lat.append((time.perf_counter() - t0 - a) * 1e3)
    span = time.perf_counter() - t0 - arrivals[0]
    return lat, span


def run_served_stream(ctb, reqs, arrivals, budget: int, copy_threads: int):
    """The same requests through ctb_server: a submitter follows the arrival
    times; latency is measured by the server from submission to completion."""
    with ctb.Server(0, memory_budget=budget, copy_threads=copy_threads) as srv:
        t0 = time.perf_counter()
        ids = []
        for r, a in zip(reqs, arrivals):
            now = time.perf_counter() - t0
            if now < a:
                time.sleep(a - now)
            ids.append(srv.submit(r["sino"], r["shape"]["n"], r["shape"]["filter"], out=r["out"]))
        status = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(s == 0 for s in status), status
    return st


def run_plain_device(be, dev):
    """Device-resident requests, one per call: ctb_fbp_d then a synchronise
    (the call returns when the request is done), back to back."""
    import torch
    lat = []
    t0 = time.perf_counter()
    for d in dev:
        s = d["shape"]
        t1 = time.perf_counter()
        be.fbp_d(d["sino"].data_ptr(), s["nz"], s["na"], s["nd"], s["n"], s["filter"], d["out"].data_ptr())
        be.synchronize()
        lat.append((time.perf_counter() - t1) * 1e3)
    torch.cuda.synchronize()
    return lat, time.perf_counter() - t0


def run_served_device(ctb, dev, budget: int):
    """The same device-resident requests submitted at once to ctb_server
    (CTB_REQ_DEVICE: nothing is staged; requests are batched)."""
    with ctb.Server(0, memory_budget=budget) as srv:
        ids = [srv.submit_device(d["sino"].data_ptr(), d["shape"]["nz"], d["shape"]["na"], d["shape"]["nd"],
                                 d["shape"]["n"], d["shape"]["filter"], d["out"].data_ptr()) for d in dev]
        status = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(s == 0 for s in status), status
    return st


def percentile(v, p):
    v = sorted(v)
    return v[min(len(v) - 1, max(0, math.ceil(p * len(v)) - 1))]


def run_serving(args, cfg, rank: int, world: int, local: int):
    """Config "serving": a Poisson stream of FBP requests (90 % the batch mix,
    10 % 1024^2 x 64 x 1440) served two ways on the same GPU from the same
    page-locked host buffers: the plain backend (ctb_fbp, one request per
    call, each call streaming its own slabs with copies overlapped) and
    ctb_server (continuous batching, memory-budgeted admission, copies of
    other requests overlapped). First both at saturation (all requests present
    at t = 0), then at arrival rates given as multiples of the plain backend's
    saturated rate. Then the same requests device-resident (sinograms already
    in HBM, volumes left there): one ctb_fbp_d call per request against the
    server's batches, which isolates what batching itself gains from what
    overlapping the host copies gains."""
    import numpy as np
    import torch

    import qtctreconstruction_b200 as ctb
    torch.cuda.set_device(local)
    be = ctb.B200Backend(local)
    shapes = serving_shapes(cfg["seed"], cfg["requests"], cfg["big_fraction"])
    # sinograms of seeded phantoms, forward-projected on the GPU, kept in
    # page-locked host memory (both arms read and write the same buffers)
    reqs, pinned = [], []
    for k, s in enumerate(shapes):
        n, nz, na, nd = s["n"], s["nz"], s["na"], s["nd"]
        vol = torch.empty((nz, n, n), dtype=torch.float32, device="cuda")
        be.phantom_d(ctb.phantom_params(cfg["seed"] * 1000 + k, 10), n, n, nz, vol.data_ptr())
        sino = torch.empty((nz, na, nd), dtype=torch.float32, device="cuda")
        stats = torch.empty((nz, 4), dtype=torch.float32, device="cuda")
        be.forward_d(vol.data_ptr(), n, nz, na, nd, sino.data_ptr(), stats.data_ptr())
        be.synchronize()
        hs = torch.empty((nz, na, nd), dtype=torch.float32, pin_memory=True)
        hs.copy_(sino)
        ho = torch.zeros((nz, n, n), dtype=torch.float32, pin_memory=True)  # pages touched now
        pinned.append((hs, ho))
        reqs.append(dict(shape=s, sino=hs.numpy(), out=ho.numpy()))
        del vol, sino
    torch.cuda.empty_cache()
    count = len(reqs)
    vol_bytes = sum(4 * s["nz"] * s["n"] ** 2 for s in shapes)
    sino_bytes = sum(4 * s["nz"] * s["na"] * s["nd"] for s in shapes)
    updates = sum(s["n"] ** 2 * s["nz"] * s["na"] for s in shapes)
    budget = cfg["budget_gb"] << 30
    # warm-up both paths: the plain backend's workspaces grow to the largest
    # request first (they are reused, never shrunk), then a few requests each
    big_s = max(range(count), key=lambda k: reqs[k]["sino"].nbytes)
    big_o = max(range(count), key=lambda k: reqs[k]["out"].nbytes)
    for r in [reqs[big_s], reqs[big_o]] + reqs[:args.warmup]:
        s = r["shape"]
        be.fbp_host_ptr(r["sino"].ctypes.data, s["nz"], s["na"], s["nd"], s["n"], s["filter"], r["out"].ctypes.data)
    run_served_stream(ctb, reqs[:args.warmup], [0.0] * args.warmup, budget, cfg["copy_threads"])

    sampler = ClockSampler(gpu_id_for(local))
    zeros = [0.0] * count
    lat_p, span_p = run_plain_stream(be, reqs, zeros)
    plain_sat = count / span_p
    ref_out = [r["out"].copy() for r in reqs[:3]]
    st = run_served_stream(ctb, reqs, zeros, budget, cfg["copy_threads"])
    served_sat = st["volumes_per_s"]
    same = all(np.array_equal(a, r["out"]) for a, r in zip(ref_out, reqs[:3]))
    sweep = []
    rng = np.random.default_rng(cfg["seed"] + 7)
    for mult in cfg["rates"]:
        rate = mult * plain_sat
        arrivals = list(np.cumsum(rng.exponential(1.0 / rate, count)) - 0.0)
        arrivals = [a - arrivals[0] for a in arrivals]
        lp, sp = run_plain_stream(be, reqs, arrivals)
        ss = run_served_stream(ctb, reqs, arrivals, budget, cfg["copy_threads"])
        sweep.append({"rate_per_s": rate, "rate_x_plain": mult,
                      "plain": {"volumes_per_s": count / sp, "p50_ms": percentile(lp, 0.5),
                                "p99_ms": percentile(lp, 0.99)},
                      "served": {"volumes_per_s": ss["volumes_per_s"], "p50_ms": ss["p50_ms"],
                                 "p99_ms": ss["p99_ms"], "mean_batch": ss["mean_batch"]}})
    # device-resident: the same requests with sinograms and volumes in HBM
    dev = [dict(shape=r["shape"], sino=torch.from_numpy(r["sino"]).cuda(),
                out=torch.zeros(r["out"].shape, dtype=torch.float32, device="cuda")) for r in reqs]
    run_plain_device(be, dev[:args.warmup])
    run_served_device(ctb, dev[:args.warmup], budget)
    lat_d, span_d = run_plain_device(be, dev)
    ref_d = [d["out"].cpu() for d in dev[:3]]
    st_d = run_served_device(ctb, dev, budget)
    same_d = all(torch.equal(a, d["out"].cpu()) for a, d in zip(ref_d, dev[:3]))
    clocks = sampler.stop()
    line = {
        "metric": "volumes/s (mixed FBP request stream)", "value": served_sat, "unit": "volumes/s",
        "n_gpus": 1, "steps": count, "warmup": args.warmup, "ms_per_step": 1e3 / served_sat,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving", "description": cfg["name"], "requests": count,
                   "voxels": vol_bytes // 4, "sinogram_bytes": sino_bytes, "budget_bytes": budget,
                   "copy_threads": cfg["copy_threads"], "host_buffers": "page-locked, shared by both arms",
                   "l2": "inputs larger than L2, no flush"},
        "served": {"volumes_per_s": served_sat, "updates_per_s": st["updates_per_s"], "p50_ms": st["p50_ms"],
                   "p99_ms": st["p99_ms"], "batches": st["batches"], "mean_batch": st["mean_batch"],
                   "memory_peak": st["memory_peak"]},
        "plain": {"volumes_per_s": plain_sat, "updates_per_s": updates / span_p,
                  "p50_ms": percentile(lat_p, 0.5), "p99_ms": percentile(lat_p, 0.99),
                  "api": "ctb_fbp, one request per call, slab-streamed copies overlapped with its compute"},
        "served_vs_plain": served_sat / plain_sat,
        "outputs_identical": same,
        "sweep": sweep,
        "device_resident": {
            "plain": {"volumes_per_s": count / span_d, "p50_ms": percentile(lat_d, 0.5),
                      "p99_ms": percentile(lat_d, 0.99), "api": "ctb_fbp_d + synchronise per request"},
            "served": {"volumes_per_s": st_d["volumes_per_s"], "p50_ms": st_d["p50_ms"], "p99_ms": st_d["p99_ms"],
                       "batches": st_d["batches"], "mean_batch": st_d["mean_batch"]},
            "served_vs_plain": st_d["volumes_per_s"] / (count / span_d),
            "outputs_identical": same_d},
        "e2e": {"value": served_sat, "unit": "volumes/s", "h2d_bytes_per_step": sino_bytes // count,
                "d2h_bytes_per_step": vol_bytes // count},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    be.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="large")
    ap.add_argument("--ref-slices", type=int, default=16, help="central slices per CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the check of the timed outputs against the FP64 oracle")
    ap.add_argument("--filter-modes", action="store_true",
                    help="also time the tensor-core filter and compare both filters with FP64 (default for precision)")
    args = ap.parse_args()
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = CONFIGS[args.config]
    if args.config == "precision":
        args.filter_modes = True
    if args.config in ("batch", "serving"):
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference",
                                  "unavailable": f"the reference has no {args.config} entry point"}))
            return 0
        run = run_batch if args.config == "batch" else run_serving
        return run(args, cfg, rank, world, local) if rank == 0 else 0
    if args.impl == "reference":
        return run_reference(args, cfg, rank, world)
    return run_ours(args, cfg, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
