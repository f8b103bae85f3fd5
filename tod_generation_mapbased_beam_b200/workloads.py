"""Seeded synthetic workloads with the shapes of the reference's benchmark
configurations (the reference itself ships no data).

* :func:`pole_gaussian_beam` -- a Gaussian beam pixelised at HEALPix pixel
  centres around the north pole of the beam frame, selected with the
  reference's power cut (dB threshold, strict ``>``; tod_utils.py:254-297 and
  sample_based_tod_generation_gridint.py:131-146) and normalised to sum 1.
* :func:`spin_scan` -- the spin scan theta = pi/2 + 0.87 sin(2 pi t / 60 s),
  phi drifting 360 deg per day, psi = phi + pi/2, cast to float32 as the
  reference driver does (gridint.py:277-279).
* :func:`white_sky` -- seeded Gaussian I/Q/U pixel values (100 uK RMS in I,
  ~31.6 uK in Q and U).  It stands in for a synfast sky: throughput and
  parity do not depend on the map content.

Beam-centre convention: (ra, dec) = (0, pi/2), i.e. the beam is centred on
the beam-frame +z axis, passed through a 3x3 grid whose centre entry is that
point (tod_rotations.py:251-263 picks the grid centre).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

ARCMIN = math.pi / (180.0 * 60.0)


def compute_db_threshold_from_power(beam_vals, power_cut):
    """dB level keeping ``power_cut`` of the summed beam (tod_utils.py:254-297):
    sort ascending in dB, suffix sums from the top, last index whose suffix
    sum still reaches the target."""
    prof = np.asarray(beam_vals).ravel()
    target = np.sum(prof) * power_cut
    with np.errstate(divide="ignore", invalid="ignore"):
        prof_db = 10 * np.log10(prof)
    order = np.argsort(prof_db)
    sorted_db = prof_db[order]
    suffix = np.cumsum(prof[order][::-1])[::-1]
    k = np.searchsorted(suffix[::-1], target, side="left")
    return sorted_db[max(0, len(suffix) - 1 - k)]


def select_beam_pixels(beam_vals, power_cut):
    """Boolean selection ``10 log10(|b| + 1e-30) > threshold``
    (gridint.py:131-133)."""
    db = compute_db_threshold_from_power(beam_vals, power_cut)
    with np.errstate(divide="ignore", invalid="ignore"):
        return 10 * np.log10(np.abs(beam_vals) + 1e-30) > db


def north_cap_pixel_centres(nside, n_rings):
    """(theta, phi) of every pixel in RING rings 1..n_rings (n_rings < nside)."""
    th, ph = [], []
    for i in range(1, n_rings + 1):
        z = 1.0 - i * i / (3.0 * nside * nside)
        j = np.arange(4 * i)
        th.append(np.full(4 * i, math.acos(z)))
        ph.append((j + 0.5) * (math.pi / (2 * i)))
    return np.concatenate(th), np.concatenate(ph)


@dataclass
class Beam:
    vec_orig: np.ndarray   # (S, 3) float32 beam-frame unit vectors
    beam_vals: np.ndarray  # (S,) float32, sum 1
    ra: np.ndarray         # (3, 3) beam grid around the centre (only the centre is used)
    dec: np.ndarray
    radius: float          # max angular distance of a selected pixel from the centre [rad]

    @property
    def S(self):
        return int(self.vec_orig.shape[0])


def pole_gaussian_beam(fwhm_arcmin, beam_nside, power_cut, fwhm2_arcmin=None, pol_angle=0.0,
                       search_fwhm=3.0):
    """Elliptical Gaussian beam (FWHM along the beam-frame x axis rotated by
    ``pol_angle``; ``fwhm2_arcmin`` across it) at nside ``beam_nside`` pixel
    centres within ``search_fwhm`` FWHMs of the pole, power-cut and normalised."""
    f1 = fwhm_arcmin * ARCMIN
    f2 = (fwhm2_arcmin if fwhm2_arcmin is not None else fwhm_arcmin) * ARCMIN
    rmax = search_fwhm * max(f1, f2)
    pix_size = math.sqrt(4 * math.pi / (12 * beam_nside * beam_nside))
    n_rings = int(rmax / (pix_size * 0.6)) + 2
    theta, phi = north_cap_pixel_centres(beam_nside, min(n_rings, beam_nside - 1))
    keep = theta <= rmax
    theta, phi = theta[keep], phi[keep]
    x = theta * np.cos(phi - pol_angle)
    y = theta * np.sin(phi - pol_angle)
    s1, s2 = f1 / math.sqrt(8 * math.log(2)), f2 / math.sqrt(8 * math.log(2))
    b = np.exp(-0.5 * ((x / s1) ** 2 + (y / s2) ** 2))
    sel = select_beam_pixels(b, power_cut)
    bv = b[sel].astype(np.float32)
    bv /= bv.sum()
    st = np.sin(theta[sel])
    vec = np.stack([st * np.cos(phi[sel]), st * np.sin(phi[sel]), np.cos(theta[sel])], -1)
    ra = np.zeros((3, 3))
    dec = np.full((3, 3), math.pi / 2)
    return Beam(vec.astype(np.float32), bv, ra, dec, float(theta[sel].max()))


def spin_scan(n_samples, rate_hz, t0=0.0, phi0=0.0):
    """Float32 (theta, phi, psi) of the spin scan."""
    t = t0 + np.arange(n_samples, dtype=np.float64) / rate_hz
    theta = math.pi / 2 + 0.87 * np.sin(2 * math.pi * t / 60.0)
    phi = np.mod(phi0 + 2 * math.pi * t / 86400.0, 2 * math.pi)
    psi = phi + math.pi / 2
    return theta.astype(np.float32), phi.astype(np.float32), psi.astype(np.float32)


def white_sky(nside, seed, dtype=np.float64):
    """(3, 12 nside^2) seeded Gaussian I/Q/U in K (I RMS 100 uK, Q/U ~31.6 uK)."""
    rng = np.random.default_rng(seed)
    npix = 12 * nside * nside
    out = np.empty((3, npix), dtype=dtype)
    for c, rms in enumerate((100e-6, 31.6e-6, 31.6e-6)):
        out[c] = rng.standard_normal(npix) * rms
    return out


def config1(n_samples=100_000, rate_hz=20.0):
    """Plain method, CPU-runnable (config 1): nside 128 sky; an elliptical
    Gaussian I beam (FWHM 1.8 deg along the beam-frame x axis, 1.5 deg across)
    at beam nside 256 with a 0.99 power cut; Q beam = I beam, so I and Q share
    one entry (C = 2, no spin-2); the U beam is 1% of the I beam times
    sin 2 phi_b on the I selection, normalised by the I beam's sum (signed,
    zero-mean weights; the reference's normalise-by-sum of such a beam would
    divide by ~0); a 20 Hz spin scan.  Returns the two beam entries (the
    reference's data dicts without maps) and the float32 scan."""
    beam = pole_gaussian_beam(108.0, 256, 0.99, fwhm2_arcmin=90.0, search_fwhm=3.0)
    v = beam.vec_orig.astype(np.float64)
    phi_b = np.arctan2(v[:, 1], v[:, 0])
    u_vals = (0.01 * beam.beam_vals.astype(np.float64) * np.sin(2 * phi_b)).astype(np.float32)
    iq = dict(vec_orig=beam.vec_orig, beam_vals=beam.beam_vals, comp_indices=[0, 1], ra=beam.ra, dec=beam.dec)
    u = dict(vec_orig=beam.vec_orig, beam_vals=u_vals, comp_indices=[2], ra=beam.ra, dec=beam.dec)
    theta, phi, psi = spin_scan(n_samples, rate_hz)
    return dict(nside=128, entries={"IQ": iq, "U": u}, theta=theta, phi=phi, psi=psi, beam=beam)


def config2(n_samples=8_640_000, seed=1):
    """Plain method on GPU (config 2): nside 1024 float64 sky, 30' FWHM
    circular beam at beam nside 2048 with a 0.99 power cut, 100 Hz spin scan."""
    beam = pole_gaussian_beam(30.0, 2048, 0.99, search_fwhm=1.5)  # S = 1512
    theta, phi, psi = spin_scan(n_samples, 100.0)
    sky = white_sky(1024, seed)
    return dict(nside=1024, beam=beam, theta=theta, phi=phi, psi=psi, sky=sky)


def rotate_beam(vec, pol_angle, offset_theta, offset_phi):
    """Beam vectors centred on the beam-frame pole, turned by ``pol_angle``
    about the pole and then moved so the pole lands at (offset_theta,
    offset_phi): a detector whose beam sits off the boresight."""
    v = np.asarray(vec, np.float64)
    c, s = math.cos(pol_angle), math.sin(pol_angle)
    v = np.stack([c * v[:, 0] - s * v[:, 1], s * v[:, 0] + c * v[:, 1], v[:, 2]], -1)
    if offset_theta == 0.0:
        return v
    t = np.array([math.sin(offset_theta) * math.cos(offset_phi),
                  math.sin(offset_theta) * math.sin(offset_phi), math.cos(offset_theta)])
    k = np.cross([0.0, 0.0, 1.0], t)
    k /= np.linalg.norm(k)
    ca, sa = math.cos(offset_theta), math.sin(offset_theta)
    return v * ca + np.cross(k, v) * sa + np.outer(v @ k, k) * (1 - ca)


def config4(n_det=64, seed=4, n_min=1e5, n_max=9e6, nside=2048, beam_nside=2048, rate_hz=100.0, make_sky=True):
    """Batched form (config 4): detectors with their own beam (FWHM ~ U(25', 35'),
    ellipticity ~ U(0, 0.1), polarisation angle ~ U(0, pi)), boresight offset
    uniform in a 1 deg disc and a scan length ~ log-uniform in [n_min, n_max];
    a float32 sky.  Returns (detectors, sky); each detector is a dict with
    ``vec_orig`` (float64, offset beam), ``beam_vals``, ``theta, phi, psi``
    (float32 scan of its own length and phase) and ``center`` (0, 0).  With
    ``make_sky=False`` the sky is None (the caller brings its own)."""
    rng = np.random.default_rng(seed)
    dets = []
    for d in range(n_det):
        fwhm = rng.uniform(25.0, 35.0)
        ell = rng.uniform(0.0, 0.1)
        pol = rng.uniform(0.0, math.pi)
        r_off = math.radians(1.0) * math.sqrt(rng.uniform())
        p_off = rng.uniform(0.0, 2 * math.pi)
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        beam = pole_gaussian_beam(fwhm, beam_nside, 0.99, fwhm2_arcmin=fwhm * (1.0 - ell),
                                  search_fwhm=1.5)
        th, ph, ps = spin_scan(n, rate_hz, t0=rng.uniform(0, 3600.0), phi0=rng.uniform(0, 2 * math.pi))
        dets.append(dict(vec_orig=rotate_beam(beam.vec_orig, pol, r_off, p_off),
                         beam_vals=beam.beam_vals, theta=th, phi=ph, psi=ps, center=(0.0, 0.0),
                         fwhm_arcmin=fwhm, ellipticity=ell, pol_angle=pol, offset=(r_off, p_off)))
    sky = white_sky(nside, seed, dtype=np.float32) if make_sky else None
    return dets, sky


def _weights_sum_to(w, total):
    w = np.asarray(w, np.float64)
    return (w * (total / w.sum())).astype(np.float32)


def config5_beams(beam_nside=2048, seed=5, fwhm_arcmin=30.0, main_fwhm=1.5, tail_deg=(10.0, 20.0), alpha=3.0,
                  m_max=8, tail_power=0.01):
    """Learned-tail form (config 5): a Gaussian main lobe (FWHM ``fwhm_arcmin``)
    kept within ``main_fwhm`` FWHMs of the pole, and a far-sidelobe annulus
    ``tail_deg`` carrying ``tail_power`` of the beam with a power-law radial
    falloff r^-alpha times a seeded azimuthal modulation
    1 + sum_{m <= m_max} a_m cos(m phi + phi_m), a_m ~ U(0, 0.1).  Pixel centres
    at ``beam_nside``.  Returns (main, tail) :class:`Beam` objects whose weights
    sum to 1 - tail_power and tail_power."""
    rng = np.random.default_rng(seed)
    f = fwhm_arcmin * ARCMIN
    r_main = main_fwhm * f
    r_in, r_out = (math.radians(d) for d in tail_deg)
    n_rings = int(beam_nside * math.sqrt(3.0 * (1.0 - math.cos(r_out)))) + 2
    if n_rings >= beam_nside:
        raise ValueError("tail radius reaches past the polar cap; use a smaller tail radius")
    theta, phi = north_cap_pixel_centres(beam_nside, n_rings)
    st, ct = np.sin(theta), np.cos(theta)
    vec = np.stack([st * np.cos(phi), st * np.sin(phi), ct], -1)
    ra = np.zeros((3, 3))
    dec = np.full((3, 3), math.pi / 2)
    m_sel = theta <= r_main
    sigma = f / math.sqrt(8 * math.log(2))
    main = Beam(vec[m_sel].astype(np.float32),
                _weights_sum_to(np.exp(-0.5 * (theta[m_sel] / sigma) ** 2), 1.0 - tail_power), ra, dec,
                float(theta[m_sel].max()))
    t_sel = (theta >= r_in) & (theta <= r_out)
    am = rng.uniform(0.0, 0.1, m_max)
    phm = rng.uniform(0.0, 2 * math.pi, m_max)
    mod = 1.0 + sum(am[m - 1] * np.cos(m * phi[t_sel] + phm[m - 1]) for m in range(1, m_max + 1))
    tail = Beam(vec[t_sel].astype(np.float32), _weights_sum_to(theta[t_sel] ** -alpha * mod, tail_power), ra, dec,
                float(theta[t_sel].max()))
    return main, tail
