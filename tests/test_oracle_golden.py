"""Pins the CPU oracle (oracle/tod_oracle.c) to golden vectors that the
reference's own Numba kernels produced (tests/golden/make_golden.py).

Everything here is bit-exact: the oracle restates the reference operation by
operation with the same operand types and the same libm."""

import numpy as np
import pytest

import oracle
from conftest import PARAM_KEYS, load_cases, load_flat


@pytest.mark.parametrize("mode", ["bilinear", "nearest"])
def test_fused_kernels_bit_exact(kernel_case, mode):
    name, g = kernel_case
    fn = oracle.gather_accum_fused if mode == "bilinear" else oracle.gather_accum_nearest
    tod = g["tod_init"].copy()
    errs = fn(*[g[k] for k in PARAM_KEYS], int(g["nside"]), g["mp_stacked"], g["beam_vals"],
              int(g["B"]), int(g["S"]), tod, int(g["c_q"]), int(g["c_u"]))
    assert errs == 0
    np.testing.assert_array_equal(tod, g["tod_" + mode])


def test_fused_stencils_bit_exact(kernel_case):
    name, g = kernel_case
    pix, wgt = oracle.bilinear_stencils(*[g[k] for k in PARAM_KEYS], int(g["nside"]),
                                        int(g["B"]), int(g["S"]))
    np.testing.assert_array_equal(pix, g["stencil_pix"])
    np.testing.assert_array_equal(wgt, g["stencil_wgt"])


@pytest.mark.parametrize("case", sorted(load_cases("healpix")))
def test_healpix_helpers_bit_exact(case):
    g = load_cases("healpix")[case]
    ns = int(g["nside"])
    pix, wgt = oracle.get_interp_weights(ns, g["theta"], g["phi"])
    np.testing.assert_array_equal(pix, g["pix"])
    np.testing.assert_array_equal(wgt, g["wgt"])
    np.testing.assert_array_equal(oracle.ang2pix(ns, g["theta"], g["phi"]), g["ang2pix"])
    th, ph = oracle.pix2ang(ns, g["pix2ang_pix"])
    np.testing.assert_array_equal(th, g["pix2ang_theta"])
    np.testing.assert_array_equal(ph, g["pix2ang_phi"])


def test_spin2_bit_exact():
    g = load_flat("spin2")
    c2, s2 = oracle.spin2(g["z_pix"], g["sth_pix"], g["phi_pix"], g["z_pts"], g["sth_pts"],
                          g["phi_pts"])
    np.testing.assert_array_equal(c2, g["c2d"])
    np.testing.assert_array_equal(s2, g["s2d"])


def test_ideal_mode_close_to_reference(kernel_case):
    """The all-float64 mode differs from the reference only by the float32
    rounding the reference applies inside its rotation (~1e-7 relative)."""
    name, g = kernel_case
    tod = g["tod_init"].copy()
    f64 = [np.asarray(g[k], np.float64) for k in PARAM_KEYS]
    oracle.gather_accum_fused(*f64, int(g["nside"]), g["mp_stacked"], g["beam_vals"], int(g["B"]),
                              int(g["S"]), tod, int(g["c_q"]), int(g["c_u"]), f64=True)
    ref = g["tod_bilinear"]
    scale = np.abs(ref - g["tod_init"]).max()
    assert np.abs(tod - ref).max() <= 1e-4 * scale + 1e-12
