"""Spherical-harmonic synthesis (todgpu_alm2map) against scipy's spherical
harmonics evaluated at the RING pixel centres."""

import numpy as np
import pytest
from scipy.special import sph_harm_y

import oracle
from tod_generation_mapbased_beam_b200 import sky

pytestmark = pytest.mark.gpu


def _direct(alm, lmax, theta, phi):
    out = np.zeros_like(theta)
    for m in range(lmax + 1):
        i0 = m * (2 * lmax + 1 - m) // 2
        for ell in range(m, lmax + 1):
            a = alm[i0 + ell, 0] + 1j * alm[i0 + ell, 1]
            y = sph_harm_y(ell, m, theta, phi)
            out += (a * y).real if m == 0 else 2.0 * (a * y).real
    return out


@pytest.mark.parametrize("nside, lmax", [(4, 11), (16, 40)])
def test_alm2map_matches_scipy(nside, lmax):
    rng = np.random.default_rng(5)
    alm = sky.random_alm(np.ones(lmax + 1), rng)
    got = sky.alm2map(alm, nside, lmax)[0].cpu().numpy()
    theta, phi = oracle.pix2ang(nside, np.arange(12 * nside * nside))
    ref = _direct(alm, lmax, theta, phi)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * np.abs(ref).max())


def test_high_l_single_modes_stay_finite_and_normalised():
    """Single modes up to l = 3 nside - 1 near the poles (the scaled
    recurrence must not underflow to zero or overflow): the map's mean square
    equals 1/(4 pi) of the mode's power within pixelisation error."""
    nside, lmax = 256, 767
    for ell, m in ((767, 0), (767, 700), (500, 500), (767, 767)):
        alm = np.zeros(((lmax + 1) * (lmax + 2) // 2, 2))
        alm[m * (2 * lmax + 1 - m) // 2 + ell, 0] = 1.0
        mp = sky.alm2map(alm, nside, lmax)[0].cpu().numpy()
        assert np.isfinite(mp).all()
        power = (1.0 if m == 0 else 2.0) / (4 * np.pi)
        assert np.mean(mp ** 2) == pytest.approx(power, rel=0.05)


def test_synfast_rms():
    mp = sky.synfast_iqu(128, seed=0).cpu().numpy()
    assert np.std(mp[0]) == pytest.approx(100e-6, rel=0.2)
    assert np.std(mp[1]) == pytest.approx(100e-6 * np.sqrt(0.055), rel=0.2)
