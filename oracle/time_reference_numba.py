"""Time the reference's own Numba path beside the C/OpenMP oracle port, on the
same inputs and the same host cores -- TEST INFRASTRUCTURE ONLY.

The reference is Python + Numba and cannot travel to the GPU machine, so the
benchmark's CPU arm times the oracle port there.  This script, run where the
reference checkout is (``--reference DIR`` or ``TOD_REFERENCE_DIR``, default
/root/reference), measures how the two compare: the reference's batch loop
of ``tod_calibrate._run_one`` (tod_calibrate.py:93-114:
``precompute_rotation_vector_batch`` then ``tod_core.beam_tod_batch`` per
batch of 32768 samples, Numba JIT warm-up excluded, best of 2) against the
oracle (``oracle.gather_accum_fused`` / ``gather_accum_nearest`` on the
float32 parameters of ``tod_rotations._rotation_params``) on the config-2
workload: nside 1024 float64 I/Q/U sky (seeded Gaussian, the cost does not
depend on its content), 30' beam at nside 2048 with a 0.99 cut (S = 1512),
a stretch of the 100 Hz spin scan.  Both use every core of the machine.  It
also checks that the two give the same TOD (float32 dict of the reference
against the float32 cast of the oracle's float64 result).

    python oracle/time_reference_numba.py [--samples N] [--mode bilinear|nearest]
"""

from __future__ import annotations

import argparse
import os
import shutil
import sys
import time
import types

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


def _import_reference(ref):
    copy = "/tmp/refcopy_timing"
    if not os.path.isdir(copy):
        shutil.copytree(ref, copy, ignore=shutil.ignore_patterns("__pycache__", "*.nbc", "*.nbi"))
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache_timing")
    sys.path.insert(0, copy)
    hp = types.ModuleType("healpy")  # tod_core imports healpy; its batch path never calls it
    hp.nside2npix = lambda nside: 12 * int(nside) ** 2
    sys.modules.setdefault("healpy", hp)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--reference", default=os.environ.get("TOD_REFERENCE_DIR", "/root/reference"))
    p.add_argument("--samples", type=int, default=131072)
    p.add_argument("--mode", choices=["bilinear", "nearest"], default="bilinear")
    p.add_argument("--batch", type=int, default=32768)
    args = p.parse_args()
    _import_reference(args.reference)

    import numba
    import numpy as np

    import oracle
    import tod_core as ref_core
    import tod_rotations as ref_rot
    from tod_generation_mapbased_beam_b200 import tod_rotations as R
    from tod_generation_mapbased_beam_b200 import workloads as W

    cores = len(os.sched_getaffinity(0))
    numba.set_num_threads(cores)
    beam = W.pole_gaussian_beam(30.0, 2048, 0.99, search_fwhm=1.5)
    th, ph, ps = W.spin_scan(args.samples, 100.0)
    sky = W.white_sky(1024, seed=1)
    data = dict(vec_orig=beam.vec_orig, beam_vals=beam.beam_vals, comp_indices=[0, 1, 2], mp_stacked=sky,
                n_sel=beam.S, ra=beam.ra, dec=beam.dec)
    ra0, dec0 = beam.ra, beam.dec

    def run_reference():
        out = []
        t0 = time.perf_counter()
        for s in range(0, args.samples, args.batch):
            e = min(s + args.batch, args.samples)
            rot, betas = ref_rot.precompute_rotation_vector_batch(ra0, dec0, ph[s:e], th[s:e])
            res = ref_core.beam_tod_batch(1024, list(sky), data, rot, ph[s:e], th[s:e], -betas + ps[s:e],
                                          interp_mode=args.mode)
            out.append(np.stack([res[c] for c in (0, 1, 2)]))
        return time.perf_counter() - t0, np.concatenate(out, axis=1)

    def run_port():
        out = np.zeros((3, args.samples))
        t0 = time.perf_counter()
        for s in range(0, args.samples, args.batch):
            e = min(s + args.batch, args.samples)
            rot, betas = R.precompute_rotation_vector_batch(ra0, dec0, ph[s:e], th[s:e])
            prm = R._rotation_params(rot, ph[s:e], th[s:e], -betas + ps[s:e])
            part = np.zeros((3, e - s))
            fn = oracle.gather_accum_fused if args.mode == "bilinear" else oracle.gather_accum_nearest
            fn(beam.vec_orig, *prm, 1024, sky, beam.beam_vals, e - s, beam.S, part, 1, 2, nthreads=cores)
            out[:, s:e] = part
        return time.perf_counter() - t0, out

    # JIT compilation and page-in outside the timing
    ref_core.beam_tod_batch(1024, list(sky), data, *ref_rot.precompute_rotation_vector_batch(ra0, dec0, ph[:64],
                                                                                               th[:64])[:1],
                            ph[:64], th[:64], ps[:64], interp_mode=args.mode)
    run_port()
    t_ref = min(run_reference()[0] for _ in range(2))
    t_port = min(run_port()[0] for _ in range(2))
    _, tod_ref = run_reference()
    _, tod_port = run_port()
    same = float(np.abs(tod_ref - tod_port.astype(np.float32)).max() / np.abs(tod_ref).max())
    import platform

    cpu = platform.processor() or platform.machine()
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    print(f"cpu: {cpu}; cores used: {cores}; numba {numba.__version__}; mode {args.mode}; "
          f"{args.samples} samples in batches of {args.batch}; S = {beam.S}")
    print(f"reference Numba path: {args.samples / t_ref:,.0f} samples/s ({t_ref:.2f} s, best of 2)")
    print(f"oracle port:          {args.samples / t_port:,.0f} samples/s ({t_port:.2f} s, best of 2)")
    print(f"port / reference: {t_ref / t_port:.3f}; max |float32 TOD difference| / max |TOD|: {same:.2e}")


if __name__ == "__main__":
    main()
