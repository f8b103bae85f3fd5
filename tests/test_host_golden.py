"""CPU tests of the host-side preparation on the path against golden vectors
made by the reference itself (tests/golden/make_golden.py):

* pointing: precompute_rotation_vector_batch (tod_rotations.py:219-303), the
  psi combination (gridint.py:281) and _rotation_params (tod_rotations.py:
  306-333) -- bit-exact;
* beam selection: the dB threshold of tod_utils.py:254-297 and the strict '>'
  mask of gridint.py:131-133 -- bit-exact."""

import numpy as np
import pytest

from conftest import load_flat
from tod_generation_mapbased_beam_b200 import tod_rotations as R
from tod_generation_mapbased_beam_b200 import workloads as W


def test_rotation_vectors_and_params_bit_exact():
    g = load_flat("rotations")
    rot, beta = R.precompute_rotation_vector_batch(g["ra"], g["dec"], g["phi"], g["theta"])
    assert rot.dtype == g["rot_vecs"].dtype and np.array_equal(rot, g["rot_vecs"])
    assert np.array_equal(beta, g["beta"])
    psis = -beta + g["psi"]
    assert np.array_equal(psis, g["psis"])
    got = R._rotation_params(rot, g["phi"], g["theta"], psis)
    for name, arr in zip(("axes", "cos_a", "sin_a", "ax_pts", "cos_p", "sin_p"), got):
        assert arr.dtype == np.float32, name
        assert np.array_equal(arr, g[name]), name


@pytest.mark.parametrize("cut", [0.9, 0.99, 0.999, 1.0])
def test_beam_selection_bit_exact(cut):
    g = load_flat("beam_prep")
    db = W.compute_db_threshold_from_power(g["beam"], cut)
    assert db == g[f"db_{cut}"]
    assert np.array_equal(W.select_beam_pixels(g["beam"], cut), g[f"sel_{cut}"])


def test_chunked_parameter_preparation_bit_exact():
    """The pipelined drop-in prepares the float32 parameters chunk by chunk on
    a thread pool; every chunk boundary (ragged ones included) gives the
    whole-batch values bit for bit."""
    from tod_generation_mapbased_beam_b200 import tod_core as TC
    from tod_generation_mapbased_beam_b200.kernels import boresight_phi_host

    beam = W.pole_gaussian_beam(30.0, 256, 0.99, search_fwhm=1.5)
    B = 50_021
    th, ph, ps = W.spin_scan(B, 100.0, phi0=0.3)
    rot, beta = R.precompute_rotation_vector_batch(beam.ra, beam.dec, ph, th)
    psis = -beta + ps
    whole = R._rotation_params(rot, ph, th, psis)
    bore = boresight_phi_host(whole[3])
    for step in (1 << 12, 7_777, B):
        parts = [TC._prep_chunk(rot, ph, th, psis, a, min(B, a + step), True) for a in range(0, B, step)]
        fields = [[] for _ in TC._PIPE_WIDTHS]
        for a, part in zip(range(0, B, step), parts):
            n = min(B, a + step) - a
            o = 0
            for i, w in enumerate(TC._PIPE_WIDTHS):
                fields[i].append(part[o:o + w * n])
                o += w * n
        got = [np.concatenate(f) for f in fields]
        for i, ref in enumerate(list(whole) + [bore]):
            assert np.array_equal(got[i], np.asarray(ref, np.float32).reshape(-1)), (step, i)


def test_beam_order_is_a_local_permutation():
    """The gather's beam-pixel order: a permutation whose consecutive pixels
    are neighbours on the sky (Morton order in the plane of the beam), for a
    pole-centred and for an offset beam."""
    from tod_generation_mapbased_beam_b200.kernels import beam_order

    beam = W.pole_gaussian_beam(30.0, 2048, 0.99, search_fwhm=1.5)
    rot = np.array([[1.0, 0.0, 0.0], [0.0, np.cos(0.3), -np.sin(0.3)], [0.0, np.sin(0.3), np.cos(0.3)]])
    for v in (beam.vec_orig.astype(np.float64), beam.vec_orig.astype(np.float64) @ rot.T):
        o = beam_order(v)
        assert np.array_equal(np.sort(o), np.arange(len(v)))

        def span(u):
            # median extent of a warp's 32 consecutive pixels, across the beam axis
            c = u.mean(axis=0)
            c /= np.linalg.norm(c)
            e1 = np.cross(c, [1.0, 0.0, 0.0])
            e1 /= np.linalg.norm(e1)
            e2 = np.cross(c, e1)
            xy = np.stack([u @ e1, u @ e2], -1)
            return np.median([np.ptp(xy[k:k + 32], axis=0).max() for k in range(0, len(u) - 32, 32)])

        # ring order strings a warp along an arc; the Morton order keeps it compact
        assert span(v[o]) < 0.5 * span(v)
        assert span(v[o]) < 12 * np.sqrt(4 * np.pi / (12 * 2048 ** 2))
    assert list(beam_order(np.zeros((1, 3)))) == [0]
