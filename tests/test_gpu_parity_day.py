"""Parity of the benchmarked configuration at scale, in both modes.

Config 2 as the benchmark times it: nside 1024 float64 I/Q/U sky (held on the
device as float64 records), 30' Gaussian beam pixelised at nside 2048 with a
0.99 power cut (S = 1512, uploaded in the library's gather order), one I/Q/U
entry with spin-2, reference float32 rotation parameters.  One million
samples spread evenly over the 8.64e6-sample 100 Hz day go through the
drop-in ``tod_core.beam_tod_batch`` (pipelined host preparation, as for a
full day) and through the CPU oracle (tod_bilinear.py:205-477,
tod_nearest.py:21-158):

* bilinear and nearest TOD within 1e-12 of the largest magnitude;
* nearest pixels identical: an index map (pixel number, and a hash of it)
  with unit beam weights makes every TOD value an exact integer sum of the
  chosen pixels, compared for equality.
"""

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

TOD_RTOL = 1e-12
N_DAY = 8_640_000
N_SUB = 1_000_000


@pytest.fixture(scope="module")
def day():
    from tod_generation_mapbased_beam_b200 import tod_rotations as R
    from tod_generation_mapbased_beam_b200 import workloads as W

    beam = W.pole_gaussian_beam(30.0, 2048, 0.99, search_fwhm=1.5)
    assert beam.S == 1512
    th, ph, ps = W.spin_scan(N_DAY, 100.0)
    idx = np.linspace(0, N_DAY - 1, N_SUB).astype(np.int64)
    th, ph, ps = th[idx].copy(), ph[idx].copy(), ps[idx].copy()
    rot, beta = R.precompute_rotation_vector_batch(beam.ra, beam.dec, ph, th)
    psis = -beta + ps
    sky = W.white_sky(1024, seed=1)
    data = dict(vec_orig=beam.vec_orig, beam_vals=beam.beam_vals, comp_indices=[0, 1, 2], mp_stacked=sky,
                ra=beam.ra, dec=beam.dec)
    params = R._rotation_params(rot, ph, th, psis)
    return dict(beam=beam, rot=rot, th=th, ph=ph, psis=psis, sky=sky, data=data, params=params)


@pytest.mark.parametrize("mode", ["bilinear", "nearest"])
def test_day_subset_matches_oracle(day, mode):
    from tod_generation_mapbased_beam_b200 import tod_core
    from tod_generation_mapbased_beam_b200.kernels import beam_order

    got = tod_core.beam_tod_batch(1024, None, day["data"], day["rot"], day["ph"], day["th"], day["psis"],
                                  interp_mode=mode, return_device=True).cpu().numpy()
    beam = day["beam"]
    order = beam_order(beam.vec_orig)
    ref = np.zeros((3, N_SUB))
    fn = oracle.gather_accum_fused if mode == "bilinear" else oracle.gather_accum_nearest
    fn(beam.vec_orig[order], *day["params"], 1024, day["sky"], beam.beam_vals[order], N_SUB, beam.S, ref, 1, 2)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(got - ref).max() <= TOD_RTOL * scale


def test_day_subset_nearest_pixels_identical(day):
    from tod_generation_mapbased_beam_b200 import _native
    from tod_generation_mapbased_beam_b200.kernels import gather_accum

    beam = day["beam"]
    npix = 12 * 1024 ** 2
    p = torch.arange(npix, dtype=torch.int64, device="cuda")
    imap = torch.stack([p.double(), ((p * 2654435761) % 1048573).double()]).contiguous()
    ones = np.ones(beam.S, np.float32)
    got = torch.zeros((2, N_SUB), dtype=torch.float64, device="cuda")
    gather_accum(_native.NEAREST, beam.vec_orig, *day["params"], 1024, imap, ones, N_SUB, beam.S, got)
    ref = np.zeros((2, N_SUB))
    oracle.gather_accum_nearest(beam.vec_orig, *day["params"], 1024, imap.cpu().numpy(), ones, N_SUB, beam.S, ref)
    got = got.cpu().numpy()
    # exact integers: the sums of the pixel numbers (and their hashes) agree
    assert np.array_equal(got[0], np.round(got[0]))
    assert np.array_equal(got, ref), int(np.count_nonzero(got != ref))
