#!/usr/bin/env python
"""Benchmark: TOD samples/s of the beam-convolution path on B200.

Workload (config 2, plain method on GPU): HEALPix RING nside 1024 float64
I/Q/U sky, circular Gaussian beam FWHM 30' at beam nside 2048 with a 0.99
power cut (S = 1512 beam pixels), one 24 h batch of a 100 Hz spin scan
(8.64e6 samples), one beam entry carrying I, Q and U (spin-2 on), bilinear
interpolation (``--mode nearest`` for the other mode).

A step is one pass of the fused kernel over the whole batch.

* ``value``: samples/s with the kernel inputs (float32 rotation parameters,
  boresight longitudes, beam, map) resident in HBM; the step zeroes the
  float64 (3, B) accumulator and runs the kernel.  Inputs (~1 GB) exceed L2.
* ``e2e``: the same metric through the public drop-in
  ``tod_core.beam_tod_batch`` with host numpy inputs (rot_vecs, phi, theta,
  psis) -> float32 host dict: host parameter preparation, host->device copies,
  kernel and device->host copy are all inside the timed region.
* ``cpu_baseline``: the CPU oracle (a C/OpenMP restatement of the reference's
  Numba kernel) on the host cores, on a bounded sample of the same workload.

``--impl reference`` times that CPU implementation as the benchmark itself
(rank 0 only), on a bounded sample per step.

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
# counted by ncu on the direct-evaluation path (TODGPU_FLAG_NO_TABLES) of the
# config-2 workload: dadd + dmul + 2 * dfma per evaluation
# (profiles/gather_accum_{bilinear,nearest}_config2.md).
FLOPS_PER_EVAL = {"bilinear": 853.0, "nearest": 500.0}


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
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision forms")
    p.add_argument("--no-learned", action="store_true", help="skip the learned-tail form (config 5)")
    p.add_argument("--no-precision", action="store_true", help="skip the nside 2048 precision form (config 3)")
    p.add_argument("--no-batched", action="store_true", help="skip the 64-detector batched form (config 4)")
    p.add_argument("--learned-train", type=int, default=1 << 18,
                   help="training pointings of the learned tail (plain-method targets)")
    p.add_argument("--learned-steps", type=int, default=4000, help="training steps of the learned tail")
    p.add_argument("--no-tables", action="store_true",
                   help="evaluate ring data and spin-2 angles directly (A/B comparison)")
    p.add_argument("--cpu-seconds", type=float, default=10.0,
                   help="target CPU time of the bounded CPU-baseline sample")
    return p.parse_args()


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

def make_workload(n_samples, rank):
    from tod_generation_mapbased_beam_b200 import tod_rotations as R
    from tod_generation_mapbased_beam_b200 import workloads as W

    beam = W.pole_gaussian_beam(30.0, 2048, 0.99, search_fwhm=1.5)
    # each rank scans its own day (weak scaling): shift the start longitude
    theta, phi, psi = W.spin_scan(n_samples, 100.0, phi0=0.7 * rank)
    # synfast-like sky: C_l^TT ~ (l+10)^-2 at 100 uK RMS, EE/BB at 10%/1%, seed 1
    # (synthesised on the GPU; a CPU-only run times the CPU path on a seeded
    # Gaussian sky of the same RMS, which does not change its cost)
    import torch

    if torch.cuda.is_available():
        from tod_generation_mapbased_beam_b200 import sky as SKY

        sky = SKY.synfast_iqu(1024, seed=1).cpu().numpy()
    else:
        sky = W.white_sky(1024, seed=1)
    rot, beta = R.precompute_rotation_vector_batch(beam.ra, beam.dec, phi, theta)
    psis = -beta + psi
    return dict(nside=1024, beam=beam, theta=theta, phi=phi, psi=psi, psis=psis, rot=rot, sky=sky)


def map_footprint_bytes(wl, itemsize):
    """Bytes of the map rows the day's scan can touch (the scan sweeps every
    longitude, so whole rings between the extreme colatitudes +- beam radius)."""
    nside = wl["nside"]
    r = wl["beam"].radius + 2 * np.sqrt(4 * np.pi / (12 * nside * nside))
    th_lo = max(0.0, float(wl["theta"].min()) - r)
    th_hi = min(np.pi, float(wl["theta"].max()) + r)
    zs = [np.cos(th_lo), np.cos(th_hi)]

    def first_pix_of_ring(ir):
        if ir < nside:
            return 2 * ir * (ir - 1)
        if ir <= 3 * nside:
            return 2 * nside * (nside - 1) + (ir - nside) * 4 * nside
        i2 = 4 * nside - ir
        return 12 * nside * nside - 2 * i2 * (i2 + 1)

    def ring_of(z):
        az = abs(z)
        if az > 2 / 3:
            ir = int(nside * np.sqrt(3 * (1 - az)))
            return ir if z > 0 else 4 * nside - ir - 1
        return int(nside * (2 - 1.5 * z))

    ir0 = max(1, ring_of(zs[0]))
    ir1 = min(4 * nside - 1, ring_of(zs[1]) + 1)
    npx = first_pix_of_ring(ir1) + (4 * nside) - first_pix_of_ring(ir0)
    npx = min(npx, 12 * nside * nside)
    return npx * 3 * itemsize


# ---------------------------------------------------------------------------
# CPU (oracle) timing
# ---------------------------------------------------------------------------

def cpu_rate(wl, mode, target_seconds):
    """Samples/s of the CPU oracle on a bounded sample; returns (rate, n, threads)."""
    import oracle
    from tod_generation_mapbased_beam_b200 import tod_rotations as R

    threads = len(os.sched_getaffinity(0))
    beam = wl["beam"]

    def run(lo, n):
        sl = slice(lo, lo + n)
        params = R._rotation_params(wl["rot"][sl], wl["phi"][sl], wl["theta"][sl], wl["psis"][sl])
        tod = np.zeros((3, n))
        fn = oracle.gather_accum_fused if mode == "bilinear" else oracle.gather_accum_nearest
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


# ---------------------------------------------------------------------------
# GPU timing
# ---------------------------------------------------------------------------

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


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


def profiled_traffic(mode):
    """dram bytes per launch recorded by the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"gather_accum_{mode}_config2.md")
    try:
        for line in open(path):
            if line.strip().startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def mixed_error_uk(wl, mode, kind, tod, cargs, margs, lib, stream, n_sub=2000):
    """RMS / max error [uK] of a mixed form against the FP64 oracle on the
    first n_sub samples (the same float32 parameters, the float64 map)."""
    import oracle
    from tod_generation_mapbased_beam_b200 import _native
    from tod_generation_mapbased_beam_b200 import tod_rotations as R

    beam = wl["beam"]
    sl = slice(0, n_sub)
    params = R._rotation_params(wl["rot"][sl], wl["phi"][sl], wl["theta"][sl], wl["psis"][sl])
    ref = np.zeros((3, n_sub))
    fn = oracle.gather_accum_fused if mode == "bilinear" else oracle.gather_accum_nearest
    fn(beam.vec_orig, *params, wl["nside"], wl["sky"], beam.beam_vals, n_sub, beam.S, ref, 1, 2,
       nthreads=len(os.sched_getaffinity(0)))
    tod.zero_()
    _native.check(lib.todgpu_gather_accum(ctypes.byref(margs), stream.cuda_stream))
    got = tod[:, :n_sub].cpu().numpy()
    err = (got - ref) * 1e6
    return {"rms_uK": float(np.sqrt(np.mean(err ** 2))), "max_uK": float(np.abs(err).max()),
            "error_sample": f"{n_sub} samples vs FP64 oracle (same float32 parameters, float64 map)"}


def run_ours(args, dist):
    import torch

    from tod_generation_mapbased_beam_b200 import _native, tod_core
    from tod_generation_mapbased_beam_b200 import tod_rotations as R
    from tod_generation_mapbased_beam_b200.kernels import (beam_reach, boresight_phi_host, make_args,
                                                           ring_table)

    dev = torch.device("cuda", dist.local)
    torch.cuda.set_device(dev)
    wl = make_workload(args.samples, dist.rank)
    beam = wl["beam"]
    B, S, nside = args.samples, beam.S, wl["nside"]
    params_h = R._rotation_params(wl["rot"], wl["phi"], wl["theta"], wl["psis"])
    bore_h = boresight_phi_host(params_h[3])
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    from tod_generation_mapbased_beam_b200.kernels import beam_order, pack_map

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
    tod = torch.zeros((3, B), dtype=torch.float64, device=dev)
    interp = _native.BILINEAR if args.mode == "bilinear" else _native.NEAREST
    table = None if args.no_tables else ring_table(nside, beam_reach(beam.vec_orig, nside), dev)
    cargs = make_args(interp, nside, B, S, 3, 1, 2, params, np.float32, bore, bv, sky_rec, tod,
                      table=table)
    lib = _native.lib()
    stream = torch.cuda.current_stream(dev)

    def step():
        tod.zero_()
        torch.cuda.nvtx.range_push("plain_step")
        k0.record(stream)
        _native.check(lib.todgpu_gather_accum(ctypes.byref(cargs), stream.cuda_stream))
        k1.record(stream)
        torch.cuda.nvtx.range_pop()

    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
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

    # roofline of the fused kernel: FP64-pipe bound.  Algorithmic work per
    # (sample, beam pixel) evaluation = the FP64 flops of the reference
    # algorithm executed directly on this GPU (ncu: dadd + dmul + 2 dfma on
    # the direct-evaluation path); peak = FP64 FMA throughput measured now.
    peaks, peak_src = measured_peaks()
    evals = float(B) * S
    flops_per_eval = FLOPS_PER_EVAL[args.mode]
    fp64_peak = fp64_peak_tflops()
    achieved = evals * flops_per_eval / (kernel_ms / 1e3) / 1e12
    bytes_per_launch = (B * (4 * 11 + 8 * 3 * 2) + S * 16 + map_footprint_bytes(wl, 8))
    hbm_achieved = bytes_per_launch / (kernel_ms / 1e3) / 1e9
    # the gather view: S x K stencil pixels of R = 32-byte float64 records per
    # sample (K = 4 bilinear, 1 nearest), against the L2 read bandwidth
    # measured now -- served mostly from L1, so not the bound of this kernel
    gather_bytes = float(B) * S * (4 if args.mode == "bilinear" else 1) * 32
    gather_gbs = gather_bytes / (kernel_ms / 1e3) / 1e9
    l2_peak = l2_peak_gbs()
    roofline = {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(fp64_peak, 3),
                "unit": "TFLOP/s", "frac": round(achieved / fp64_peak, 4),
                "traffic": profiled_traffic(args.mode),
                "peak_source": "measured now (todgpu_fp64_probe: 8 independent FMA chains/thread)",
                "algorithmic_flops_per_eval": flops_per_eval,
                "evals_per_launch": int(evals), "kernel": "gather_accum_kernel",
                "kernel_ms": round(kernel_ms, 3),
                "hbm": {"achieved": round(hbm_achieved, 2), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": round(hbm_achieved / peaks["hbm_gbs"], 5),
                        "algorithmic_bytes_per_launch": int(bytes_per_launch),
                        "peak_source": peak_src},
                "gather": {"achieved": round(gather_gbs, 1), "peak": round(l2_peak, 1), "unit": "GB/s",
                           "frac": round(gather_gbs / l2_peak, 4),
                           "bytes_per_sample": int(gather_bytes / B),
                           "peak_source": "measured now (todgpu_l2_probe: 16-byte L1-bypassing loads over "
                                          "64 MiB)",
                           "note": "logical stencil gathers; 93% are L1 hits, so this is not the bound"}}

    result = {"value": value, "ms_per_step": total_ms / args.steps, "roofline": roofline,
              "clocks": clk, "gpu_launches": args.steps}

    # mixed precision forms on the same workload: packed float32 / bfloat16
    # records, float32 spin-2 table, float32 Kahan sum, float64 decisions;
    # error against the FP64 oracle on a bounded subset of samples
    if not args.no_mixed:
        mixed = {}
        tod_rec = tod.clone()  # the float64 result of the last timed step
        for kind in ("planar_f64", "f32", "bf16"):
            pm = sky if kind == "planar_f64" else pack_map(sky, kind)
            margs = make_args(interp, nside, B, S, 3, 1, 2, params, np.float32, bore, bv, pm, tod,
                              table=table)
            for _ in range(2):
                _native.check(lib.todgpu_gather_accum(ctypes.byref(margs), stream.cuda_stream))
            torch.cuda.synchronize()
            m0 = torch.cuda.Event(enable_timing=True)
            m1 = torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            for _ in range(args.steps):
                tod.zero_()
                _native.check(lib.todgpu_gather_accum(ctypes.byref(margs), stream.cuda_stream))
            m1.record(stream)
            m1.synchronize()
            mms = dist.max(m0.elapsed_time(m1) / args.steps)
            entry = {"value": B * dist.world / (mms / 1e3), "ms_per_step": mms,
                     "map": {"planar_f64": "planar float64 (C, N), the reference's mp_stacked",
                             "f32": "packed f32 records (16 B/pixel)", "bf16": "packed bf16 records (8 B/pixel)"}[kind]}
            # the gather view for this map layout: S x K stencil pixels of R bytes
            # (planar float64: three 8-byte reads per pixel) against the L2 bandwidth
            rec = {"planar_f64": 24, "f32": 16, "bf16": 8}[kind]
            gb = float(B) * S * (4 if args.mode == "bilinear" else 1) * rec / (mms / 1e3) / 1e9
            entry["gather"] = {"bytes_per_sample": S * (4 if args.mode == "bilinear" else 1) * rec,
                               "achieved": round(gb, 1), "peak": round(l2_peak, 1), "unit": "GB/s",
                               "frac": round(gb / l2_peak, 4)}
            if kind == "planar_f64":
                entry["bit_identical_to_value"] = bool(torch.equal(tod, tod_rec))
            elif dist.rank == 0 and not args.no_cpu_baseline:
                entry.update(mixed_error_uk(wl, args.mode, kind, tod, cargs, margs, lib, stream))
            mixed[kind] = entry
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
                         "api": "driver.DayRunner.run: host float32 (theta, phi, psi) -> host "
                                "float64 tod_day (3, n); rotation derived on the GPU in FP64"}
        drop_s, res = timed(lambda: tod_core.beam_tod_batch(nside, None, data, wl["rot"], wl["phi"],
                                                            wl["theta"], wl["psis"],
                                                            interp_mode=args.mode))
        assert res[0].shape == (B,)
        result["e2e_drop_in"] = {"value": B * dist.world * args.steps / drop_s, "unit": "samples/s",
                                 "h2d_bytes_per_step": int(B * (4 * 10 + 4)),
                                 "d2h_bytes_per_step": int(B * 3 * 4),
                                 "api": "tod_core.beam_tod_batch: host rot_vecs/angles in (host "
                                        "float32 parameter prep as the reference), float32 dict out"}

    if not args.no_cpu_baseline and dist.rank == 0:
        rate, n, threads = cpu_rate(wl, args.mode, args.cpu_seconds)
        result["cpu_baseline"] = {"value": rate, "unit": "samples/s", "cores": threads,
                                  "kind": "port",
                                  "sample": f"{n} consecutive samples of the same workload "
                                            f"(S={S}, nside {nside}), C/OpenMP oracle, best of 2"}
    return result, B, S


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
    return {"rms_uK": np.sqrt((d ** 2).mean(axis=1)).tolist(), "max_uK": np.abs(d).max(axis=1).tolist()}


def run_precision(args, dist, sky):
    """Precision form (config 3): nside 2048 synfast-like sky (seed 2) as
    packed float32 and bfloat16 records, 30' beam at nside 4096 with a 0.999
    cut, 8.64e6 scan samples with the rotation derived on the device in
    float64; one timed launch per form (each ~4 s) after one warm-up, errors
    on 4096 samples against the float64 path on the same inputs."""
    import torch

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
    vec = torch.from_numpy(beam.vec_orig.astype(np.float64)[order]).to(dev)
    bv = torch.from_numpy(beam.beam_vals[order]).to(dev)
    interp = _native.BILINEAR if args.mode == "bilinear" else _native.NEAREST
    idx = torch.from_numpy(np.linspace(0, B - 1, 4096).astype(np.int64)).to(dev)
    out, subs = {}, {}
    for kind in ("f64", "f32", "bf16"):
        mp = pack_map(sky, kind)
        tod = torch.zeros((3, B), dtype=torch.float64, device=dev)

        def launch():
            tod.zero_()
            gather_accum_angles(interp, vec, *ang, 0.0, 0.0, 2048, mp, bv, tod, c_q=1, c_u=2)

        launch()
        ms = dist.max(_evt_ms(launch, stream))
        subs[kind] = tod[:, idx].cpu().numpy()
        rec = {"f64": 32, "f32": 16, "bf16": 8}[kind]
        kk = 4 if args.mode == "bilinear" else 1
        gb = float(B) * beam.S * kk * rec / (ms / 1e3) / 1e9
        out[kind] = {"value": B * dist.world / (ms / 1e3), "ms_per_step": ms,
                     "map": {"f64": "packed f64 records (32 B/pixel; TOD bit-identical to the planar "
                                    "float64 map)", "f32": "packed f32 records (16 B/pixel)",
                             "bf16": "packed bf16 records (8 B/pixel)"}[kind],
                     "gather": {"bytes_per_sample": beam.S * kk * rec, "achieved": round(gb, 1),
                                "peak": round(l2_peak, 1), "unit": "GB/s", "frac": round(gb / l2_peak, 4)}}
        del tod, mp
    for kind in ("f32", "bf16"):
        out[kind].update(_err_uk(subs[kind], subs["f64"]))
    return {"workload": f"config3 precision form, {args.mode}: nside 2048 synfast-like sky (seed 2), 30' "
                        f"beam @ nside 4096, 0.999 cut (S={beam.S}), 100 Hz scan, angles (FP64 rotation "
                        "on the device)", "samples_per_gpu": B, "S": beam.S, "forms": out,
            "error_reference": "float64 map, same kernel and pointing (the FP64 path, within 1e-10 of "
                               "the FP64 CPU oracle in the tests); 4096 samples spread over the day"}


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
    n, evals = batch.n_samples, batch.n_evals

    def loop():
        for d, vec, bvt, angs, o in zip(dets, batch.vec, batch.beam, batch.angles, batch.out):
            o.zero_()
            gather_accum_angles(batch.interp, vec, *angs, 0.0, 0.0, 2048, pm, bvt, o, c_q=1, c_u=2)

    loop_ms = dist.max(_evt_ms(loop, stream))
    batch.release()
    return {"workload": f"config4 batched, {args.mode}: {len(dets)} detectors, own beams (S "
                        f"{min(v.shape[0] for v in batch.vec)}-{max(v.shape[0] for v in batch.vec)}), "
                        "scans log-uniform 1e5-9e6 samples, nside 2048 packed f32 sky",
            "value": n * dist.world / (ms / 1e3), "unit": "samples/s", "samples_per_gpu": n,
            "evals_per_s": evals * dist.world / (ms / 1e3), "ms_per_step": ms, "tile": batch.tile,
            "autotune_seconds": tune_s, "graph": True,
            "per_detector_launches_value": n * dist.world / (loop_ms / 1e3)}


def run_learned(args, dist, sky):
    """Learned-tail form (config 5): nside 2048 synfast-like sky (seed 2),
    30' Gaussian main lobe kept exact within 45' (packed float32 map, Kahan
    sums, float64 decisions) plus a 10-20 deg far-sidelobe annulus with 1% of
    the power replaced by the Fourier-feature network, trained here on
    plain-method tail targets at uniform pointings (seed 6).  Throughput over
    the config-2 scan (8.64e6 samples at 100 Hz) against the plain float64
    path on the whole beam; errors on 4096 held-out scan samples against the
    plain float64 path, with the tail dropped for comparison."""
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
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    lt.full_plain(*sub)
    p1.record(stream)
    p1.synchronize()
    plain_rate = 2048 / (dist.max(p0.elapsed_time(p1)) / 1e3)
    value = B * dist.world / (step_ms / 1e3)
    F, H, D, O = lt.net.dims
    flops = 2.0 * (7 * F + 2 * F * H + (D - 1) * H * H + O * H)
    peaks, peak_src = measured_peaks()
    net_tflops = B * flops / (net_ms_mean / 1e3) / 1e12
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    return {
        "workload": "config5 learned tail: nside 2048 f64 synfast-like sky (seed 2); beam = 30' Gaussian "
                    f"main lobe within 45' ({main.S} px, exact, packed f32 map + Kahan) + 10-20 deg annulus "
                    f"({tail.S} px, 1% power, r^-3 x (1 + sum_m<=8 a_m cos(m phi + phi_m)), seed 5) replaced "
                    "by the network; config-2 scan",
        "value": value, "unit": "samples/s", "samples_per_gpu": B, "ms_per_step": step_ms,
        "plain_fp64_value": plain_rate, "plain_fp64_sample": "2048 held-out scan samples, whole beam "
                                                            "(main + tail) by the float64 gather",
        "speedup_vs_plain_fp64": value / (plain_rate * dist.world),
        "error_vs_plain_fp64": judged["learned"], "error_tail_dropped": judged["dropped"],
        "tail_rms_uK": judged["tail_rms_uK"], "surrogate_error": judged["surrogate"],
        "budget_uK": judged["budget_uK"], "within_budget": bool(judged["use_surrogate"]),
        "judge_samples": judged["samples"],
        "main_lobe_ms": statistics.mean(main_ms), "network_ms": net_ms_mean,
        "network": {"dims": {"n_freq": F, "width": H, "depth": D, "n_out": O}, "flops_per_sample": flops,
                    "achieved": round(net_tflops, 2), "unit": "TFLOP/s", "peak": bf16_peak,
                    "frac": round(net_tflops / bf16_peak, 4),
                    "peak_source": f"bf16 dense GEMM burst ({peak_src}); hidden layers on mma.sync bf16"},
        "training": dict(info, sigma=list(lt.net.sigma)),
    }


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return None
    wl = make_workload(min(args.samples, 2_000_000), 0)
    rates = []
    per_step = max(2.0, 120.0 / max(1, args.steps + args.warmup))
    for i in range(args.warmup + args.steps):
        rate, n, threads = cpu_rate(wl, args.mode, min(args.cpu_seconds, per_step))
        if i >= args.warmup:
            rates.append((rate, n))
    value = statistics.mean(r for r, _ in rates)
    n = rates[-1][1]
    return {"impl": "reference", "value": value, "threads": threads, "n": n, "S": wl["beam"].S}


def main():
    args = parse_args()
    base = {"metric": METRIC, "unit": "samples/s", "higher_is_better": True, "steps": args.steps,
            "warmup": args.warmup, "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded 100 Hz spin scan, pole-centred Gaussian beam, seeded "
                    "synfast-like I/Q/U sky (GPU alm2map, C_l^TT ~ (l+10)^-2, 100 uK RMS)"}
    config = {"workload": f"config2 plain FP64, {args.mode}: nside 1024 f64 I/Q/U sky (float64 records), 30' FWHM "
                          f"beam @ nside 2048 0.99 cut, 100 Hz spin scan, one beam entry (I,Q,U; spin-2)",
              "samples_per_gpu": args.samples, "mode": args.mode,
              "l2": "inputs larger than L2 (params+map ~1 GB), no flush needed",
              "params": "float32 reference-typed rotation parameters"}
    if args.impl == "reference":
        r = run_reference(args)
        if r is None:
            return
        config["samples_per_gpu"] = r["n"]
        line = dict(base, impl="reference", value=r["value"], n_gpus=args.gpus,
                    ms_per_step=r["n"] / r["value"] * 1e3, scaling="weak", config=config,
                    cpu_baseline={"value": r["value"], "unit": "samples/s", "cores": r["threads"],
                                  "kind": "port",
                                  "sample": f"{r['n']} samples per step (S={r['S']}), C/OpenMP "
                                            "restatement of the reference Numba kernel"},
                    e2e={"value": r["value"], "unit": "samples/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0})
        print(json.dumps(line))
        return

    dist = Dist()
    res, B, S = run_ours(args, dist)
    if not (args.no_learned and args.no_precision and args.no_batched):
        import torch

        from tod_generation_mapbased_beam_b200 import sky as SKY

        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        sky2048 = SKY.synfast_iqu(2048, seed=2)  # configs 3-5
        torch.cuda.synchronize()
        res["sky2048_seconds"] = time.perf_counter() - t0
        if not args.no_precision:
            res["precision"] = run_precision(args, dist, sky2048)
        if not args.no_batched:
            res["batched"] = run_batched(args, dist, sky2048)
        if not args.no_learned:
            res["learned"] = run_learned(args, dist, sky2048)
        del sky2048
    if dist.rank == 0:
        line = dict(base, value=res["value"], n_gpus=dist.world, ms_per_step=res["ms_per_step"],
                    scaling="weak", config=dict(config, S=S, parallelism=f"samples x{dist.world}"),
                    roofline=res["roofline"], gpu_launches=res["gpu_launches"],
                    clocks=res["clocks"])
        for key in ("e2e", "e2e_drop_in", "mixed", "precision", "batched", "learned", "sky2048_seconds"):
            if key in res:
                line[key] = res[key]
        if "cpu_baseline" in res:
            line["cpu_baseline"] = res["cpu_baseline"]
        print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
