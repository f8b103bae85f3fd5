"""Day driver (the GPU counterpart of tod_exact_gen_batched / _process_day):
scan-file IO on CPU; the reference- and device-pointing day loops on GPU."""

import numpy as np
import pytest

import oracle
from tod_generation_mapbased_beam_b200 import driver
from tod_generation_mapbased_beam_b200 import tod_rotations as R
from tod_generation_mapbased_beam_b200 import workloads as W


def _write_scan(folder, days, n, rate=5.0):
    for d in range(days):
        th, ph, ps = W.spin_scan(n, rate, t0=86400.0 * d / 50, phi0=0.3 * d)
        np.save(folder / f"theta_{d}.npy", th)
        np.save(folder / f"phi_{d}.npy", ph)
        np.save(folder / f"psi_{d}.npy", ps)


def test_scan_information_and_open(tmp_path):
    _write_scan(tmp_path, 3, 432)
    days, fsamp = driver.load_scan_information(str(tmp_path))
    assert days == 3 and fsamp == pytest.approx(432 / 86400)
    th, ph, ps = driver.open_scan_day(str(tmp_path), 2)
    assert th.shape == ph.shape == ps.shape == (432,) and th.dtype == np.float32


def test_scan_information_errors(tmp_path):
    with pytest.raises(FileNotFoundError):
        driver.load_scan_information(str(tmp_path))
    np.save(tmp_path / "psi_x.npy", np.zeros(3))
    with pytest.raises(ValueError):
        driver.load_scan_information(str(tmp_path))


def _beam_data(nside, seed, split):
    beam = W.pole_gaussian_beam(90.0, 256, 0.99, search_fwhm=1.5)
    rng = np.random.default_rng(seed)
    mp = rng.standard_normal((3, 12 * nside * nside)).astype(np.float32)
    mk = lambda comps: dict(vec_orig=beam.vec_orig, beam_vals=beam.beam_vals, comp_indices=comps,  # noqa: E731
                            mp_stacked=np.ascontiguousarray(mp[comps]), ra=beam.ra, dec=beam.dec)
    if split:
        return {"IQ": mk([0, 1]), "U": mk([2])}, mp, beam
    return {"IQU": mk([0, 1, 2])}, mp, beam


def _oracle_day(beam_data, theta, phi, psi, nside, batch, f64):
    """The reference day loop with the oracle as the kernel."""
    n = len(phi)
    first = next(iter(beam_data.values()))
    out = np.zeros((3, n))
    for s0 in range(0, n, batch):
        s1 = min(n, s0 + batch)
        th, ph, ps = (np.asarray(x[s0:s1], np.float32) for x in (theta, phi, psi))
        if f64:
            rot, beta = oracle.rotation_vectors_f64(0.0, 0.0, ph.astype(np.float64), th.astype(np.float64))
            params = oracle.rotation_params_f64(rot, ph, th, ps.astype(np.float64) - beta)
        else:
            rot, beta = R.precompute_rotation_vector_batch(first["ra"], first["dec"], ph, th)
            params = R._rotation_params(rot, ph, th, -beta + ps)
        for data in beam_data.values():
            comps = data["comp_indices"]
            c_q = comps.index(1) if 1 in comps else -1
            c_u = comps.index(2) if 2 in comps else -1
            tod = np.zeros((len(comps), s1 - s0))
            vec = data["vec_orig"].astype(np.float64) if f64 else data["vec_orig"]
            oracle.gather_accum_fused(vec, *params, nside, data["mp_stacked"], data["beam_vals"],
                                      s1 - s0, len(vec), tod, c_q, c_u, f64=f64)
            for i, c in enumerate(comps):
                out[c, s0:s1] += tod[i] if f64 else tod[i].astype(np.float32)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("split", [False, True])
def test_reference_pointing_day_matches_reference_loop(split):
    nside, n = 64, 1500
    beam_data, mp, beam = _beam_data(nside, 3, split)
    theta, phi, psi = W.spin_scan(n, 5.0, phi0=2.0)
    got = driver.DayRunner(beam_data, nside, chunk=400, pointing="reference").run(theta, phi, psi)
    ref = _oracle_day(beam_data, theta, phi, psi, nside, 400, f64=False)
    assert got.dtype == np.float64 and got.shape == (3, n)
    # each entry is cast to float32 like the reference; the kernels agree to 1e-12
    np.testing.assert_allclose(got, ref, rtol=0, atol=2 * np.finfo(np.float32).eps * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("split", [False, True])
def test_device_pointing_day_matches_fp64_ideal(split):
    nside, n = 64, 2500
    beam_data, mp, beam = _beam_data(nside, 4, split)
    theta, phi, psi = W.spin_scan(n, 5.0, phi0=1.0)
    got = driver.DayRunner(beam_data, nside, chunk=700).run(theta, phi, psi)
    ref = _oracle_day(beam_data, theta, phi, psi, nside, 10_000, f64=True)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    one_chunk = driver.DayRunner(beam_data, nside, chunk=10_000).run(theta, phi, psi)
    np.testing.assert_array_equal(got, one_chunk)


@pytest.mark.gpu
def test_process_day_writes_tod_day(tmp_path):
    scan = tmp_path / "scan"
    out = tmp_path / "out"
    scan.mkdir()
    out.mkdir()
    _write_scan(scan, 2, 900)
    beam_data, mp, beam = _beam_data(32, 5, False)
    day, ok, err = driver.process_day(1, beam_data, None, 256, str(scan), str(out), 32)
    assert ok and err is None and day == 1
    tod = np.load(out / "tod_day_1.npy")
    assert tod.shape == (3, 900) and tod.dtype == np.float64 and np.isfinite(tod).all()
    day, ok, err = driver.process_day(7, beam_data, None, 256, str(scan), str(out), 32)
    assert not ok and "theta_7" in err
