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
