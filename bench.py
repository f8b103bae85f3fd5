#!/usr/bin/env python
"""Benchmark: TOD samples/s of the beam-convolution path on B200.

Workload (config 2, plain method on GPU): HEALPix RING nside 1024 float64
I/Q/U sky, circular Gaussian beam FWHM 30' at beam nside 2048 with a 0.99
power cut (S = 1512 beam pixels), one 24 h batch of a 100 Hz spin scan
(8.64e6 samples), one beam entry carrying I, Q and U (spin-2 on), bilinear
interpolation (``--mode nearest`` makes nearest the headline mode).

A step is one pass of the fused kernel over the whole batch.

* ``value``: samples/s with the kernel inputs (float32 rotation parameters,
  boresight longitudes, beam, map) resident in HBM; the step zeroes the
  float64 (3, B) accumulator and runs the kernel.  Inputs (~1 GB) exceed L2.
* ``roofline``: the gather view of the kernel -- S x K stencil pixels of R =
  32-byte float64 records per sample -- against the L2 read bandwidth
  measured live by ``todgpu_l2_probe``.
* ``parity``: both modes of the timed configuration (same beam order, same
  map records, same float32 parameters) against the CPU oracle on a subset of
  samples spread over the day; nearest-pixel identity by an index map.
* ``nearest`` (or ``bilinear`` under ``--mode nearest``): the other mode,
  timed on the same workload.
* ``e2e``: the day driver with host float32 scan in and host float64 (3, n)
  out, copies inside the timed region; ``e2e_drop_in``: the drop-in
  ``tod_core.beam_tod_batch`` from host arrays.
* ``cpu_baseline``: the CPU oracle (a C/OpenMP restatement of the reference's
  Numba kernel) on the host cores, on a bounded sample of the same workload.
* ``mixed``, ``precision`` (config 3), ``batched`` (config 4), ``learned``
  (config 5): the other forms, each as value, time and error only.

``--impl reference`` times the CPU implementation as the benchmark itself
(rank 0 only, bounded sample per step) on a sky built on the CPU: nothing of
the GPU library is loaded in that arm.

Multi-GPU (torchrun): each rank runs its own day of samples (weak scaling, no
collective on the data path); timings are max-reduced over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TOD samples/s, 1 B200: FP64 plain vs mixed/learned-tail at fixed RMS error"

# FP64 flops per (sample, beam pixel) evaluation of the reference algorithm,
# counted by ncu (dadd + dmul + 2 * dfma) on the direct-evaluation path
# (TODGPU_FLAG_NO_TABLES) of the config-2 workload.  The timed kernel takes
# spin-2 angles from per-sample tables, so it executes fewer: the rate below
# is reference-equivalent work per second, not pipe utilisation.
REF_FLOPS_PER_EVAL = {"bilinear": 853.0, "nearest": 500.0}
STENCIL = {"bilinear": 4, "nearest": 1}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--mode", choices=["bilinear", "nearest"], default="bilinear")
    p.add_argument("--samples", type=int, default=8_640_000)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-parity", action="store_true", help="skip the oracle parity of the timed day")
    p.add_argument("--parity-samples", type=int, default=200_000,
                   help="samples of the timed day compared with the CPU oracle (spread over the day)")
    p.add_argument("--no-other-mode", action="store_true", help="skip the timed leg of the other mode")
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision forms")
    p.add_argument("--no-learned", action="store_true", help="skip the learned-tail form (config 5)")
    p.add_argument("--no-precision", action="store_true", help="skip the nside 2048 precision form (config 3)")
    p.add_argument("--no-batched", action="store_true", help="skip the 64-detector batched form (config 4)")
    p.add_argument("--learned-train", type=int, default=1 << 18,
                   help="training pointings of the learned tail (plain-method targets)")
    p.add_argument("--learned-steps", type=int, default=4000, help="training steps of the learned tail")
    p.add_argument("--learned-curve", type=str, default=None,
                   help="comma-separated training-set sizes: print the learned tail's held-out error per size "
                        "(targets of the largest, nested subsets) instead of the benchmark")
    p.add_argument("--no-tables", action="store_true",
                   help="evaluate ring data and spin-2 angles directly (A/B comparison)")
    p.add_argument("--no-beam-stage", action="store_true",
                   help="read the beam from global memory instead of shared memory (A/B comparison)")
    p.add_argument("--cpu-seconds", type=float, default=10.0,
                   help="target CPU time of the bounded CPU-baseline sample")
    return p.parse_args()


def g4(x):
    """x rounded to 4 significant digits (keeps the JSON line short)."""
    if x is None:
        return None
    if isinstance(x, (list, tuple, np.ndarray)):
        return [g4(v) for v in np.asarray(x).reshape(-1)]
    return float(f"{float(x):.4g}")


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(
        os.environ.get("LOCAL_RANK", 0))


class Dist:
    def __init__(self):
        import torch

        self.torch = torch
        self.rank, self.world, self.local = dist_env()
        self.pg = None
        if self.world > 1:
            import torch.distributed as td

            torch.cuda.set_device(self.local)
            td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                  device_id=torch.device("cuda", self.local))
            self.pg = td

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device="cuda")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def _numpy_modules():
    from tod_generation_mapbased_beam_b200 import tod_rotations as R
    from tod_generation_mapbased_beam_b200 import workloads as W

    return R, W


def make_workload(n_samples, rank, gpu_sky=True):
    """Config-2 workload of one rank.  The sky is synthesised on the GPU
    (synfast-like: C_l^TT ~ (l+10)^-2 at 100 uK RMS, EE/BB at 10%/1%, seed 1);
    with ``gpu_sky=False`` (the CPU arm) it is a seeded Gaussian sky of the
    same RMS built on the CPU -- the CPU path's cost does not depend on the
    sky's content, and that arm then loads nothing of the GPU library."""
    R, W = _numpy_modules()
    beam = W.pole_gaussian_beam(30.0, 2048, 0.99, search_fwhm=1.5)
    # each rank scans its own day (weak scaling): shift the start longitude
    theta, phi, psi = W.spin_scan(n_samples, 100.0, phi0=0.7 * rank)
    if gpu_sky:
        from tod_generation_mapbased_beam_b200 import sky as SKY

        sky = SKY.synfast_iqu(1024, seed=1).cpu().numpy()
    else:
        sky = W.white_sky(1024, seed=1)
    rot, beta = R.precompute_rotation_vector_batch(beam.ra, beam.dec, phi, theta)
    psis = -beta + psi
    return dict(nside=1024, beam=beam, theta=theta, phi=phi, psi=psi, psis=psis, rot=rot, sky=sky)


def bench_config(args, S, world):
    return {"workload": f"config2 FP64 {args.mode}: nside 1024 IQU sky, 30' beam @2048 0.99 cut, 100 Hz scan, "
                        "spin-2",
            "samples_per_gpu": args.samples, "S": S, "mode": args.mode,
            "l2": "inputs > L2, no flush", "params": "reference f32",
            "parallelism": f"samples x{world}"}


# ---------------------------------------------------------------------------
# CPU (oracle) timing and parity
# ---------------------------------------------------------------------------

def oracle_fn(mode):
    import oracle

    return oracle.gather_accum_fused if mode == "bilinear" else oracle.gather_accum_nearest


def cpu_rate(wl, mode, target_seconds):
    """Samples/s of the CPU oracle on a bounded sample; returns (rate, n, threads)."""
    R, _ = _numpy_modules()
    threads = len(os.sched_getaffinity(0))
    beam = wl["beam"]
    fn = oracle_fn(mode)

    def run(lo, n):
        sl = slice(lo, lo + n)
        params = R._rotation_params(wl["rot"][sl], wl["phi"][sl], wl["theta"][sl], wl["psis"][sl])
        tod = np.zeros((3, n))
        t0 = time.perf_counter()
        fn(beam.vec_orig, *params, wl["nside"], wl["sky"], beam.beam_vals, n, beam.S, tod, 1, 2,
           nthreads=threads)
        return time.perf_counter() - t0

    run(0, 64)  # page in the library and the map
    n0 = max(threads * 16, 512)
    dt = run(1000, n0)
    n = int(min(len(wl["theta"]) - 2000, max(n0, n0 * target_seconds / max(dt, 1e-6))))
    best = float("inf")
    for rep in range(2):
        best = min(best, run(2000 + rep * 7, n))
    return n / best, n, threads


def index_map(npix, device):
    """(2, npix) float64 map whose values identify the pixel: p and a hash of
    p below 2^20.  Summed with unit beam weights, every TOD value is an exact
    integer (below 2^53), so two engines agree on it exactly only if they
    picked the same pixels."""
    import torch

    p = torch.arange(npix, dtype=torch.int64, device=device)
    return torch.stack([p.double(), ((p * 2654435761) % 1048573).double()]).contiguous()


def oracle_parity(wl, params_h, order, gpu_tod, mode, idx, nthreads):
    """Max |GPU - oracle| / max |oracle| over the subset idx of the day, for
    the timed kernel's inputs (the beam in the same pixel order)."""
    beam = wl["beam"]
    sub = [np.ascontiguousarray(p[idx]) for p in params_h]
    ref = np.zeros((3, idx.size))
    oracle_fn(mode)(beam.vec_orig[order], *sub, wl["nside"], wl["sky"], beam.beam_vals[order], idx.size,
                    beam.S, ref, 1, 2, nthreads=nthreads)
    scale = float(np.abs(ref).max())
    return float(np.abs(gpu_tod - ref).max()) / scale


def nearest_pixel_identity(wl, params_h, idx, nthreads, dev):
    """Nearest pixels of the GPU kernel and the oracle on the subset idx: the
    index map with unit beam weights, compared exactly."""
    import torch

    from tod_generation_mapbased_beam_b200 import _native
    from tod_generation_mapbased_beam_b200.kernels import gather_accum

    beam = wl["beam"]
    n = idx.size
    sub = [np.ascontiguousarray(p[idx]) for p in params_h]
    ones = np.ones(beam.S, np.float32)
    imap = index_map(12 * wl["nside"] ** 2, dev)
    got = torch.zeros((2, n), dtype=torch.float64, device=dev)
    gather_accum(_native.NEAREST, beam.vec_orig, *sub, wl["nside"], imap, ones, n, beam.S, got)
    ref = np.zeros((2, n))
    oracle_fn("nearest")(beam.vec_orig, *sub, wl["nside"], imap.cpu().numpy(), ones, n, beam.S, ref,
                         nthreads=nthreads)
    got = got.cpu().numpy()
    return bool(np.array_equal(got, ref)), int(np.count_nonzero(got != ref))


# ---------------------------------------------------------------------------
# GPU timing helpers
# ---------------------------------------------------------------------------

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_peak_tflops():
    """FP64 FMA throughput of this GPU, measured with the library's probe."""
    import torch

    from tod_generation_mapbased_beam_b200 import _native

    lib = _native.lib()
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    blocks = sms * 16
    sink = torch.zeros(blocks, dtype=torch.float64, device="cuda")
    flops = ctypes.c_double()
    stream = torch.cuda.current_stream()
    best = 0.0
    for _ in range(4):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _native.check(lib.todgpu_fp64_probe(blocks, 4096, sink.data_ptr(), ctypes.byref(flops),
                                            stream.cuda_stream))
        e1.record(stream)
        e1.synchronize()
        best = max(best, flops.value / (e0.elapsed_time(e1) / 1e3) / 1e12)
    return best


def l2_peak_gbs():
    """L2 read bandwidth of this GPU, measured with the library's probe over a
    64 MiB buffer (inside the 126 MB L2)."""
    import torch

    from tod_generation_mapbased_beam_b200 import _native

    lib = _native.lib()
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    blocks = sms * 8
    buf = torch.ones(64 << 20, dtype=torch.uint8, device="cuda")
    sink = torch.zeros(blocks, dtype=torch.int32, device="cuda")
    nbytes = ctypes.c_double()
    stream = torch.cuda.current_stream()
    best = 0.0
    for _ in range(4):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _native.check(lib.todgpu_l2_probe(buf.data_ptr(), buf.numel(), 8, sink.data_ptr(), blocks,
                                          ctypes.byref(nbytes), stream.cuda_stream))
        e1.record(stream)
        e1.synchronize()
        best = max(best, nbytes.value / (e0.elapsed_time(e1) / 1e3) / 1e9)
    return best


def _evt_ms(fn, stream):
    import torch

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _err_uk(a, b):
    d = (a - b) * 1e6
    return {"rms_uK": g4(np.sqrt((d ** 2).mean(axis=1))), "max_uK": g4(np.abs(d).max(axis=1))}


def gather_frac(B, S, mode, rec_bytes, ms, l2_peak):
    gb = float(B) * S * STENCIL[mode] * rec_bytes / (ms / 1e3) / 1e9
    return gb, gb / l2_peak


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, dist):
    import torch

    from tod_generation_mapbased_beam_b200 import _native, tod_core
    from tod_generation_mapbased_beam_b200 import tod_rotations as R
    from tod_generation_mapbased_beam_b200.kernels import (beam_order, beam_reach, boresight_phi_host, make_args,
                                                           pack_map, ring_table)

    dev = torch.device("cuda", dist.local)
    torch.cuda.set_device(dev)
    wl = make_workload(args.samples, dist.rank)
    beam = wl["beam"]
    B, S, nside = args.samples, beam.S, wl["nside"]
    params_h = R._rotation_params(wl["rot"], wl["phi"], wl["theta"], wl["psis"])
    bore_h = boresight_phi_host(params_h[3])
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731

    # the beam's pixels in the library's gather order (as every beam-level entry
    # point uploads them; only the order of the pixel sum changes)
    order = beam_order(beam.vec_orig)
    params = [to(beam.vec_orig[order])] + [to(p) for p in params_h]
    bore = to(bore_h)
    bv = to(beam.beam_vals[order])
    sky = to(wl["sky"])
    # float64 map as float64 records {I, Q, U, 0}: the library's layout for the
    # float64 path (packed on upload; TOD bit-identical to the planar map)
    sky_rec = pack_map(sky, "f64")
    table = None if args.no_tables else ring_table(nside, beam_reach(beam.vec_orig, nside), dev)
    lib = _native.lib()
    stream = torch.cuda.current_stream(dev)
    modes = [args.mode] + ([] if args.no_other_mode else [m for m in STENCIL if m != args.mode])
    interp = {"bilinear": _native.BILINEAR, "nearest": _native.NEAREST}
    tods = {m: torch.zeros((3, B), dtype=torch.float64, device=dev) for m in modes}
    flags = _native.FLAG_NO_BEAM_STAGE if args.no_beam_stage else 0
    cargs = {m: make_args(interp[m], nside, B, S, 3, 1, 2, params, np.float32, bore, bv, sky_rec, tods[m],
                          table=table, flags=flags) for m in modes}

    def launch(m):
        _native.check(lib.todgpu_gather_accum(ctypes.byref(cargs[m]), stream.cuda_stream))

    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)

    def step():
        tods[args.mode].zero_()
        torch.cuda.nvtx.range_push("plain_step")
        k0.record(stream)
        launch(args.mode)
        k1.record(stream)
        torch.cuda.nvtx.range_pop()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kern_ms = []
    dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        k1.synchronize()
        kern_ms.append(k0.elapsed_time(k1))
    ev1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    total_ms = dist.max(ev0.elapsed_time(ev1))
    kernel_ms = dist.max(statistics.mean(kern_ms))
    value = B * dist.world * args.steps / (total_ms / 1e3)

    # roofline: the gather view of the kernel -- S x K stencil pixels of R = 32
    # byte float64 records per sample -- against the L2 read bandwidth measured
    # now.  Beside it: the reference-equivalent FP64 rate (ncu-counted flops of
    # the reference algorithm on this GPU) against the FP64 FMA peak measured
    # now, and the compulsory HBM bytes against the measured HBM peak.
    peaks, peak_src = measured_peaks()
    l2_peak = l2_peak_gbs()
    g_gbs, g_frac = gather_frac(B, S, args.mode, 32, kernel_ms, l2_peak)
    fp64_peak = fp64_peak_tflops()
    ref_tflops = float(B) * S * REF_FLOPS_PER_EVAL[args.mode] / (kernel_ms / 1e3) / 1e12
    hbm_bytes = B * (4 * 11 + 8 * 3 * 2) + S * 16
    roofline = {"bound": "l2", "achieved": g4(g_gbs), "peak": g4(l2_peak), "unit": "GB/s", "frac": g4(g_frac),
                "traffic": None, "kernel": "gather_accum_kernel", "kernel_ms": g4(kernel_ms),
                "bytes_per_sample": S * STENCIL[args.mode] * 32,
                "peak_source": "todgpu_l2_probe, this run",
                "fp64_peak_tflops": g4(fp64_peak),
                "ref_equiv_fp64_frac": g4(ref_tflops / fp64_peak),
                "hbm_frac": g4(hbm_bytes / (kernel_ms / 1e3) / 1e9 / peaks["hbm_gbs"])}
    result = {"value": value, "ms_per_step": total_ms / args.steps, "roofline": roofline, "clocks": clk,
              "gpu_launches": args.steps}

    # the other mode on the same workload (same buffers, its own output)
    for m in modes[1:]:
        launch(m)
        torch.cuda.synchronize()
        times = []
        for _ in range(args.steps):
            tods[m].zero_()
            times.append(_evt_ms(lambda: launch(m), stream))
        ms = dist.max(statistics.mean(times))
        _, fr = gather_frac(B, S, m, 32, ms, l2_peak)
        result[m] = {"value": g4(B * dist.world / (ms / 1e3)), "kernel_ms": g4(ms), "gather_frac": g4(fr)}

    # parity of the timed day: both modes against the CPU oracle on a subset
    # spread over the day (same float32 parameters, same beam order, the
    # float64 map), and the nearest pixels compared exactly by an index map
    if not args.no_parity and dist.rank == 0:
        t0 = time.perf_counter()
        nthreads = len(os.sched_getaffinity(0))
        n_sub = min(args.parity_samples, B)
        idx = np.unique(np.linspace(0, B - 1, n_sub).astype(np.int64))
        par = {"samples": int(idx.size)}
        idx_d = to(idx)
        for m in modes:
            rel = oracle_parity(wl, params_h, order, tods[m][:, idx_d].cpu().numpy(), m, idx, nthreads)
            par[f"rel_err_{m}"] = g4(rel)
        if "nearest" in modes:
            same, ndiff = nearest_pixel_identity(wl, params_h, idx, nthreads, dev)
            par["nearest_pixels_identical"] = same
            if not same:
                par["nearest_pixel_sums_differing"] = ndiff
        par["tolerance"] = 1e-12
        par["seconds"] = g4(time.perf_counter() - t0)
        result["parity"] = par

    # mixed precision forms on the same workload: packed float32 / bfloat16
    # records, float32 spin-2 table, float32 Kahan sum, float64 decisions;
    # error against the FP64 oracle on a bounded subset of samples
    if not args.no_mixed:
        mixed = {}
        tod = tods[args.mode]
        tod_rec = tod.clone()  # the float64 result of the last timed step
        sub_ref = None
        if dist.rank == 0 and not args.no_cpu_baseline:
            n_sub = 2000
            sub = [p[:n_sub] for p in params_h]
            sub_ref = np.zeros((3, n_sub))
            oracle_fn(args.mode)(beam.vec_orig, *sub, nside, wl["sky"], beam.beam_vals, n_sub, S, sub_ref, 1, 2,
                                 nthreads=len(os.sched_getaffinity(0)))
        for kind in ("planar_f64", "f32", "bf16"):
            pm = sky if kind == "planar_f64" else pack_map(sky, kind)
            margs = make_args(interp[args.mode], nside, B, S, 3, 1, 2, params, np.float32, bore, bv, pm, tod,
                              table=table, flags=flags)
            for _ in range(2):
                _native.check(lib.todgpu_gather_accum(ctypes.byref(margs), stream.cuda_stream))
            torch.cuda.synchronize()
            times = []
            for _ in range(args.steps):
                tod.zero_()
                times.append(_evt_ms(lambda: _native.check(
                    lib.todgpu_gather_accum(ctypes.byref(margs), stream.cuda_stream)), stream))
            mms = dist.max(statistics.mean(times))
            rec = {"planar_f64": 24, "f32": 16, "bf16": 8}[kind]
            _, fr = gather_frac(B, S, args.mode, rec, mms, l2_peak)
            entry = {"value": g4(B * dist.world / (mms / 1e3)), "gather_frac": g4(fr)}
            if kind == "planar_f64":
                entry["bit_identical"] = bool(torch.equal(tod, tod_rec))
            elif sub_ref is not None:
                err = (tod[:, :sub_ref.shape[1]].cpu().numpy() - sub_ref) * 1e6
                entry["rms_uK"] = g4(float(np.sqrt(np.mean(err ** 2))))
                entry["max_uK"] = g4(float(np.abs(err).max()))
            mixed[kind] = entry
            del pm
        result["mixed"] = mixed

    # end to end with host buffers: the day driver (host float32 scan in,
    # float64 (3, n) day TOD out, device pointing, pipelined copies), and the
    # drop-in beam_tod_batch (host rotation vectors / angles in, float32 dict out)
    if not args.no_e2e:
        from tod_generation_mapbased_beam_b200.driver import DayRunner

        data = dict(vec_orig=beam.vec_orig, beam_vals=beam.beam_vals, comp_indices=[0, 1, 2],
                    mp_stacked=wl["sky"], ra=beam.ra, dec=beam.dec)
        runner = DayRunner({"beam": data}, nside, interp_mode=args.mode, chunk=1 << 20)

        def timed(fn):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                out = fn()
            torch.cuda.synchronize()
            return dist.max(time.perf_counter() - t0), out

        e2e_s, day = timed(lambda: runner.run(wl["theta"], wl["phi"], wl["psi"]))
        assert day.shape == (3, B)
        result["e2e"] = {"value": B * dist.world * args.steps / e2e_s, "unit": "samples/s",
                         "h2d_bytes_per_step": int(B * 3 * 4), "d2h_bytes_per_step": int(B * 3 * 8),
                         "api": "DayRunner.run, host angles -> host f64 TOD"}
        drop_s, res = timed(lambda: tod_core.beam_tod_batch(nside, None, data, wl["rot"], wl["phi"],
                                                            wl["theta"], wl["psis"],
                                                            interp_mode=args.mode))
        assert res[0].shape == (B,)
        result["e2e_drop_in"] = {"value": g4(B * dist.world * args.steps / drop_s),
                                 "h2d_bytes_per_step": int(B * (4 * 10 + 4)), "d2h_bytes_per_step": int(B * 3 * 4)}

    if not args.no_cpu_baseline and dist.rank == 0:
        rate, n, threads = cpu_rate(wl, args.mode, args.cpu_seconds)
        result["cpu_baseline"] = {"value": g4(rate), "unit": "samples/s", "cores": threads, "kind": "port",
                                  "sample": f"{n} consecutive samples, C/OpenMP oracle, best of 2"}
    return result, B, S


def run_precision(args, dist, sky):
    """Precision form (config 3): nside 2048 synfast-like sky (seed 2) as
    float64, packed float32 and bfloat16 records, 30' beam at nside 4096 with
    a 0.999 cut, 8.64e6 scan samples with the rotation derived on the device
    in float64; one timed launch per form after one warm-up.  Errors on a
    subset of samples spread over the day against the FP64 CPU oracle run of
    the same inputs (pointing angles -> float64 rotation parameters -> float64
    gather of the float64 map)."""
    import torch

    import oracle
    from tod_generation_mapbased_beam_b200 import _native
    from tod_generation_mapbased_beam_b200 import workloads as W
    from tod_generation_mapbased_beam_b200.kernels import beam_order, gather_accum_angles, pack_map

    dev = torch.device("cuda", dist.local)
    stream = torch.cuda.current_stream(dev)
    l2_peak = l2_peak_gbs()
    beam = W.pole_gaussian_beam(30.0, 4096, 0.999, search_fwhm=2.0)
    B = args.samples
    th, ph, ps = W.spin_scan(B, 100.0, phi0=0.7 * dist.rank)
    ang = [torch.from_numpy(a).to(dev) for a in (th, ph, ps)]
    order = beam_order(beam.vec_orig)
    vec64 = beam.vec_orig.astype(np.float64)[order]
    bv_h = beam.beam_vals[order]
    vec = torch.from_numpy(vec64).to(dev)
    bv = torch.from_numpy(bv_h).to(dev)
    interp = _native.BILINEAR if args.mode == "bilinear" else _native.NEAREST
    n_sub = 8192
    idx = np.linspace(0, B - 1, n_sub).astype(np.int64)
    idx_d = torch.from_numpy(idx).to(dev)
    out, subs = {}, {}
    for kind in ("f64", "f32", "bf16"):
        mp = pack_map(sky, kind)
        tod = torch.zeros((3, B), dtype=torch.float64, device=dev)

        def launch():
            tod.zero_()
            gather_accum_angles(interp, vec, *ang, 0.0, 0.0, 2048, mp, bv, tod, c_q=1, c_u=2,
                                flags=_native.FLAG_NO_BEAM_STAGE if args.no_beam_stage else 0)

        launch()
        ms = dist.max(_evt_ms(launch, stream))
        subs[kind] = tod[:, idx_d].cpu().numpy()
        rec = {"f64": 32, "f32": 16, "bf16": 8}[kind]
        _, fr = gather_frac(B, beam.S, args.mode, rec, ms, l2_peak)
        out[kind] = {"value": g4(B * dist.world / (ms / 1e3)), "gather_frac": g4(fr)}
        del tod, mp
    if dist.rank == 0 and not args.no_cpu_baseline:
        t0 = time.perf_counter()
        rv, beta = oracle.rotation_vectors_f64(0.0, 0.0, ph[idx], th[idx])
        prm = oracle.rotation_params_f64(rv, ph[idx], th[idx], np.asarray(ps[idx], np.float64) - beta)
        ref = np.zeros((3, n_sub))
        oracle_fn(args.mode)(vec64, *prm, 2048, sky.cpu().numpy(), bv_h, n_sub, beam.S, ref, 1, 2,
                             nthreads=len(os.sched_getaffinity(0)), f64=True)
        for kind in ("f64", "f32", "bf16"):
            out[kind].update(_err_uk(subs[kind], ref))
        oracle_s = time.perf_counter() - t0
    else:
        oracle_s = None
    return {"S": beam.S, "forms": out, "err_vs": f"FP64 oracle, {n_sub} samples"}


def run_batched(args, dist, sky):
    """Batched form (config 4): 64 detectors (FWHM 25-35', ellipticity 0-0.1,
    polarisation angle, boresight offset within 1 deg, scans log-uniform in
    1e5-9e6 samples) on the nside 2048 sky as packed float32 records, one
    persistent graph-captured launch with the autotuned tile, against one
    launch per detector."""
    import torch

    from tod_generation_mapbased_beam_b200 import autotune
    from tod_generation_mapbased_beam_b200 import workloads as W
    from tod_generation_mapbased_beam_b200.batched import DetectorBatch
    from tod_generation_mapbased_beam_b200.kernels import gather_accum_angles, pack_map

    dev = torch.device("cuda", dist.local)
    stream = torch.cuda.current_stream(dev)
    dets, _ = W.config4(seed=4, make_sky=False)
    pm = pack_map(sky, "f32")
    batch = DetectorBatch(2048, pm, dets, interp_mode=args.mode)
    t0 = time.perf_counter()
    batch.tile = autotune.choose_tile(batch, timing_batch=batch.truncated(1.0 / 16))
    tune_s = time.perf_counter() - t0
    batch.run()  # graph capture
    torch.cuda.synchronize()
    times = [_evt_ms(batch.run, stream) for _ in range(args.steps)]
    ms = dist.max(statistics.mean(times))
    n = batch.n_samples

    def loop():
        for vec, bvt, angs, o in zip(batch.vec, batch.beam, batch.angles, batch.out):
            o.zero_()
            gather_accum_angles(batch.interp, vec, *angs, 0.0, 0.0, 2048, pm, bvt, o, c_q=1, c_u=2)

    loop_ms = dist.max(statistics.mean(_evt_ms(loop, stream) for _ in range(2)))
    batch.release()
    return {"value": g4(n * dist.world / (ms / 1e3)), "ms": g4(ms), "samples": n, "tile": batch.tile,
            "per_detector_value": g4(n * dist.world / (loop_ms / 1e3))}


def run_learned(args, dist, sky):
    """Learned-tail form (config 5): nside 2048 synfast-like sky (seed 2),
    30' Gaussian main lobe kept exact within 45' (packed float32 map, Kahan
    sums, float64 decisions) plus a 10-20 deg far-sidelobe annulus with 1% of
    the power replaced by the Fourier-feature network, trained here on
    plain-method tail targets at uniform pointings (seed 6).  Throughput over
    the config-2 scan (8.64e6 samples at 100 Hz) against the plain float64
    path on the whole beam; errors per Stokes component on 4096 held-out scan
    samples against the plain float64 path, with the tail dropped beside it."""
    import torch

    from tod_generation_mapbased_beam_b200 import learned as L
    from tod_generation_mapbased_beam_b200 import workloads as W

    dev = torch.device("cuda", dist.local)
    main, tail = W.config5_beams()
    lt = L.LearnedTailTOD(2048, sky, main, tail)
    info = lt.fit(n_train=args.learned_train, steps=args.learned_steps)
    B = args.samples
    th, ph, ps = W.spin_scan(B, 100.0, phi0=0.7 * dist.rank)
    idx = np.linspace(0, B - 1, 4096).astype(np.int64)
    held = [torch.from_numpy(a[idx].copy()).to(dev) for a in (th, ph, ps)]
    judged = lt.judge(*held, budget_uK=0.1)
    scan = [torch.from_numpy(a).to(dev) for a in (th, ph, ps)]
    tod = torch.zeros((3, B), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    main_ms, net_ms = [], []
    for i in range(args.warmup + args.steps):
        tod.zero_()
        torch.cuda.nvtx.range_push("learned_form")
        ev[0].record(stream)
        lt.main_lobe(*scan, tod)
        ev[1].record(stream)
        lt.learned_tail(*scan, tod)
        ev[2].record(stream)
        torch.cuda.nvtx.range_pop()
        ev[2].synchronize()
        if i >= args.warmup:
            main_ms.append(ev[0].elapsed_time(ev[1]))
            net_ms.append(ev[1].elapsed_time(ev[2]))
    step_ms = dist.max(statistics.mean(m + n for m, n in zip(main_ms, net_ms)))
    net_ms_mean = dist.max(statistics.mean(net_ms))
    sub = [a[:2048] for a in held]
    lt.full_plain(*sub)
    torch.cuda.synchronize()
    plain_ms = dist.max(_evt_ms(lambda: lt.full_plain(*sub), stream))
    plain_rate = 2048 / (plain_ms / 1e3)
    value = B * dist.world / (step_ms / 1e3)
    F, H, D, O = lt.net.dims
    flops = 2.0 * (7 * F + 2 * F * H + (D - 1) * H * H + O * H)
    peaks, _ = measured_peaks()
    net_tflops = B * flops / (net_ms_mean / 1e3) / 1e12
    peak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1400.0))
    return {
        "value": g4(value), "ms": g4(step_ms), "plain_fp64_value": g4(plain_rate),
        "speedup_vs_plain_fp64": g4(value / (plain_rate * dist.world)),
        "err_rms_uK": g4(judged["learned"]["rms_uK"]), "dropped_rms_uK": g4(judged["dropped"]["rms_uK"]),
        "budget_uK": 0.1,
        "within_budget_per_component": bool(judged["use_surrogate"]),
        "dropped_within_budget": bool(max(judged["dropped"]["rms_uK"]) <= 0.1),
        "main_ms": g4(statistics.mean(main_ms)), "net_ms": g4(net_ms_mean),
        "net_tflops": g4(net_tflops), "net_frac_bf16_sustained": g4(net_tflops / peak),
        "n_train": info["n_train"],
    }


def run_learned_curve(args, sizes):
    """Held-out error of the learned tail (config 5) against the training-set
    size: plain-method targets at max(sizes) uniform pointings (seed 6), a
    network trained on each nested prefix (same steps and batch), judged on
    4096 samples of the config-2 scan against the plain float64 path."""
    import torch

    from tod_generation_mapbased_beam_b200 import learned as L
    from tod_generation_mapbased_beam_b200 import sky as SKY
    from tod_generation_mapbased_beam_b200 import workloads as W
    from tod_generation_mapbased_beam_b200.tailnet import TailNet

    dev = torch.device("cuda")
    sky = SKY.synfast_iqu(2048, seed=2)
    main, tail = W.config5_beams()
    lt = L.LearnedTailTOD(2048, sky, main, tail)
    n_max = max(sizes)
    t0 = time.perf_counter()
    th, ph, ps = L.uniform_pointings(n_max, 6)
    ang = [torch.from_numpy(a).to(dev) for a in (th, ph, ps)]
    target = lt.plain_tail(*ang)
    torch.cuda.synchronize()
    target_s = time.perf_counter() - t0
    B = args.samples
    sth, sph, sps = W.spin_scan(B, 100.0)
    idx = np.linspace(0, B - 1, 4096).astype(np.int64)
    held = [torch.from_numpy(a[idx].copy()).to(dev) for a in (sth, sph, sps)]
    out = []
    for n in sorted(sizes):
        lt.net = TailNet(n_out=3)
        x = lt.net.inputs(*[a[:n] for a in ang])
        t1 = time.perf_counter()
        losses = lt.net.fit(x[:n], target[:, :n].T.contiguous(), steps=args.learned_steps, batch=8192)
        torch.cuda.synchronize()
        j = lt.judge(*held, budget_uK=0.1)
        out.append({"n_train": n, "err_rms_uK": g4(j["learned"]["rms_uK"]), "err_max_uK": g4(j["learned"]["max_uK"]),
                    "loss_last": g4(float(losses[-100:].mean())), "train_s": g4(time.perf_counter() - t1)})
    return {"curve": out, "dropped_rms_uK": g4(j["dropped"]["rms_uK"]), "target_s": g4(target_s),
            "targets": n_max, "steps": args.learned_steps, "held_out": 4096}


# ---------------------------------------------------------------------------
# the CPU arm
# ---------------------------------------------------------------------------

def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return None
    wl = make_workload(min(args.samples, 2_000_000), 0, gpu_sky=False)
    rates = []
    per_step = max(2.0, 120.0 / max(1, args.steps + args.warmup))
    for i in range(args.warmup + args.steps):
        rate, n, threads = cpu_rate(wl, args.mode, min(args.cpu_seconds, per_step))
        if i >= args.warmup:
            rates.append((rate, n))
    value = statistics.mean(r for r, _ in rates)
    n = rates[-1][1]
    return {"value": value, "threads": threads, "n": n, "S": wl["beam"].S}


def main():
    args = parse_args()
    base = {"metric": METRIC, "unit": "samples/s", "higher_is_better": True, "steps": args.steps,
            "warmup": args.warmup, "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded spin scan, Gaussian beam, synfast-like I/Q/U sky (GPU; CPU arm: Gaussian "
                    "sky, same RMS)"}
    if args.impl == "reference":
        r = run_reference(args)
        if r is None:
            return
        line = dict(base, impl="reference", value=r["value"], n_gpus=args.gpus,
                    ms_per_step=r["n"] / r["value"] * 1e3, scaling="weak",
                    config=bench_config(args, r["S"], args.gpus),
                    cpu_baseline={"value": r["value"], "unit": "samples/s", "cores": r["threads"],
                                  "kind": "port",
                                  "sample": f"{r['n']} samples per step of the same day, C/OpenMP restatement "
                                            "of the reference Numba kernel, CPU-built sky"},
                    e2e={"value": r["value"], "unit": "samples/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0})
        print(json.dumps(line))
        return

    if args.learned_curve:
        print(json.dumps(run_learned_curve(args, [int(v) for v in args.learned_curve.split(",")]),
                         separators=(",", ":")))
        return
    dist = Dist()
    res, B, S = run_ours(args, dist)
    if not (args.no_learned and args.no_precision and args.no_batched):
        import torch

        from tod_generation_mapbased_beam_b200 import sky as SKY

        torch.cuda.empty_cache()
        sky2048 = SKY.synfast_iqu(2048, seed=2)  # configs 3-5
        torch.cuda.synchronize()
        if not args.no_precision:
            res["precision"] = run_precision(args, dist, sky2048)
        if not args.no_batched:
            res["batched"] = run_batched(args, dist, sky2048)
        if not args.no_learned:
            res["learned"] = run_learned(args, dist, sky2048)
        del sky2048
    if dist.rank == 0:
        line = dict(base, value=res["value"], n_gpus=dist.world, ms_per_step=res["ms_per_step"],
                    scaling="weak", config=bench_config(args, S, dist.world), roofline=res["roofline"],
                    gpu_launches=res["gpu_launches"], clocks=res["clocks"])
        for key in ("cpu_baseline", "e2e", "parity", "nearest", "bilinear", "e2e_drop_in", "mixed", "precision",
                    "batched", "learned"):
            if key in res:
                line[key] = res[key]
        print(json.dumps(line, separators=(",", ":")))
    dist.close()


if __name__ == "__main__":
    main()
