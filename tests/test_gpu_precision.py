"""Precision form (packed float32 / bfloat16 maps, float32 spin-2 angles,
float32 Kahan accumulation, float64 decisions) against the FP64 oracle.

Error budgets are stated in microkelvin for a sky of 100 uK RMS in I and
31.6 uK in Q/U (white, so every pixel is independent: a harsher case for
map rounding than a smooth CMB sky)."""

import numpy as np
import pytest
import torch

import oracle
from tod_generation_mapbased_beam_b200 import _native
from tod_generation_mapbased_beam_b200 import tod_rotations as R
from tod_generation_mapbased_beam_b200 import workloads as W
from tod_generation_mapbased_beam_b200.kernels import gather_accum, pack_map

pytestmark = pytest.mark.gpu


def _case(nside, B, fwhm, beam_nside, cut, seed):
    beam = W.pole_gaussian_beam(fwhm, beam_nside, cut, search_fwhm=2.0)
    theta, phi, psi = W.spin_scan(B, 100.0, phi0=0.4)
    rot, beta = R.precompute_rotation_vector_batch(beam.ra, beam.dec, phi, theta)
    params = R._rotation_params(rot, phi, theta, -beta + psi)
    sky = W.white_sky(nside, seed)
    return beam, params, sky


@pytest.mark.parametrize("kind", ["f32", "bf16"])
def test_pack_map_records(kind):
    rng = np.random.default_rng(1)
    mp = rng.standard_normal((3, 5000))
    packed = pack_map(mp, kind)
    got = packed.data.float().cpu().numpy()
    want32 = mp.astype(np.float32)
    if kind == "f32":
        np.testing.assert_array_equal(got[:, :3], want32.T)
    else:
        ref = torch.from_numpy(want32.T.copy()).to(torch.bfloat16).float().numpy()
        np.testing.assert_array_equal(got[:, :3], ref)
    np.testing.assert_array_equal(got[:, 3], 0.0)


@pytest.mark.parametrize("mode", ["bilinear", "nearest"])
@pytest.mark.parametrize("kind, rms_uk, max_uk", [("f32", 1e-3, 1e-2), ("bf16", 0.1, 1.0)])
def test_precision_form_error_budget(mode, kind, rms_uk, max_uk):
    """Config-3 shapes scaled down: 30' beam at beam nside 1024 (0.999 cut), nside 512 sky."""
    nside, B = 512, 2000
    beam, params, sky = _case(nside, B, 30.0, 1024, 0.999, seed=2)
    interp = _native.BILINEAR if mode == "bilinear" else _native.NEAREST
    tod = torch.zeros((3, B), dtype=torch.float64, device="cuda")
    gather_accum(interp, beam.vec_orig, *params, nside, pack_map(sky, kind), beam.beam_vals, B, beam.S, tod, 1, 2)
    ref = np.zeros((3, B))
    fn = oracle.gather_accum_fused if mode == "bilinear" else oracle.gather_accum_nearest
    fn(beam.vec_orig, *params, nside, sky, beam.beam_vals, B, beam.S, ref, 1, 2)
    err_uk = (tod.cpu().numpy() - ref) * 1e6
    rms = float(np.sqrt(np.mean(err_uk ** 2)))
    assert rms <= rms_uk, f"{kind} {mode}: RMS {rms:.3e} uK"
    assert float(np.abs(err_uk).max()) <= max_uk


def test_precision_form_keeps_float64_decisions():
    """A packed float32 map of float32 values: the same pixels and weights as
    the float64 path, so the only difference is float32 mixing (< 1e-6
    relative)."""
    nside, B = 256, 800
    beam, params, sky = _case(nside, B, 60.0, 512, 0.99, seed=3)
    sky32 = sky.astype(np.float32)
    out = []
    for mp in (sky32, pack_map(sky32, "f32")):
        tod = torch.zeros((3, B), dtype=torch.float64, device="cuda")
        gather_accum(_native.BILINEAR, beam.vec_orig, *params, nside, mp, beam.beam_vals, B, beam.S, tod, 1, 2)
        out.append(tod.cpu().numpy())
    assert np.abs(out[0] - out[1]).max() <= 1e-6 * np.abs(out[0]).max()
