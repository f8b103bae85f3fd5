"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, validates arguments before touching CUDA, and its host-side
helper reproduces the host C library's atan2f."""

import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from tod_generation_mapbased_beam_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    text = open(os.path.join(ROOT, "include", "todgpu.h")).read()
    return sorted(set(re.findall(r"\b(todgpu_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    lib = _native.lib()
    declared = _header_functions()
    assert declared, "no functions parsed from include/todgpu.h"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in todgpu.h but not exported"
    assert sorted(_native.exported_symbols()) == declared


def test_abi_version():
    assert _native.lib().todgpu_abi_version() == _native.ABI_VERSION


def _args(**kw):
    a = _native.GatherArgs()
    a.abi_version = _native.ABI_VERSION
    a.interp = _native.BILINEAR
    a.nside = 16
    a.B = 0
    a.S = 0
    a.C = 3
    a.c_q = 1
    a.c_u = 2
    a.params_dtype = _native.F32
    a.map_dtype = _native.F32
    a.map_stride = 12 * 16 * 16
    a.tod_stride = 0
    for k, v in kw.items():
        setattr(a, k, v)
    return a


@pytest.mark.parametrize("kw, code", [
    (dict(abi_version=99), _native.EABI),
    (dict(nside=0), _native.ENSIDE),
    (dict(nside=1 << 20), _native.ENSIDE),
    (dict(interp=7), _native.EINVAL),
    (dict(C=0), _native.ESHAPE),
    (dict(C=5), _native.ESHAPE),
    (dict(c_q=1, c_u=1), _native.ESHAPE),
    (dict(c_q=3), _native.ESHAPE),
    (dict(map_dtype=9), _native.EDTYPE),
    (dict(params_dtype=9), _native.EDTYPE),
    (dict(map_stride=10), _native.ESHAPE),
    (dict(B=-1), _native.ESHAPE),
    (dict(tab_slots=-1), _native.EINVAL),
    (dict(B=4, S=4, tod_stride=4), _native.EINVAL),  # NULL pointers with work to do
])
def test_argument_validation(kw, code):
    lib = _native.lib()
    a = _args(**kw)
    rc = lib.todgpu_gather_accum(ctypes.byref(a), None)
    assert rc == code
    assert lib.todgpu_last_error_string()


def test_null_args_rejected():
    assert _native.lib().todgpu_gather_accum(None, None) == _native.EINVAL


def test_empty_batch_is_a_noop():
    # B == 0 or S == 0 returns before any CUDA call.
    assert _native.lib().todgpu_gather_accum(ctypes.byref(_args(B=0, S=5)), None) == 0
    assert _native.lib().todgpu_gather_accum(ctypes.byref(_args(B=5, S=0, tod_stride=5)), None) == 0


def test_boresight_phi_host_matches_libm_atan2f():
    rng = np.random.default_rng(3)
    pts = rng.standard_normal((200_000, 3)).astype(np.float32)
    from tod_generation_mapbased_beam_b200.kernels import boresight_phi_host

    got = boresight_phi_host(pts)
    np.testing.assert_array_equal(got, oracle.atan2f(pts[:, 1], pts[:, 0]))


def test_table_slots_request():
    """Spin-2 table slots asked for per call: a footprint's worth for small
    reaches (grows with reach and nside), the default beyond 0.05 rad."""
    from tod_generation_mapbased_beam_b200 import kernels as K

    assert K.table_slots(1024, 0.0143) < K.table_slots(2048, 0.0143) < K.table_slots(2048, 0.02)
    # config 2: 1.05 x (1.02 x 3 r^2 n^2 + 3 per ring over 3 r n + 4 rings) + 32
    assert 800 < K.table_slots(1024, 0.0143) < 950
    assert K.table_slots(256, 0.05) == 0 and K.table_slots(256, 0.2) == 0
    assert K.table_slots_for(None, 1024) == 0


def test_pointing_params_validation():
    """todgpu_pointing_params checks its arguments before any CUDA call: a
    negative count, a bad angle type and NULL arrays are rejected; no samples
    is a no-op."""
    lib = _native.lib()
    p = ctypes.c_void_p(16)  # never dereferenced: every case fails (or returns) before use
    args = lambda B, dt, ptr: [ptr, p, p, dt, B, 0.0, 0.0] + [p] * 6 + [None]  # noqa: E731
    assert lib.todgpu_pointing_params(*args(-1, _native.F32, p)) == _native.ESHAPE
    assert lib.todgpu_pointing_params(*args(4, 7, p)) == _native.EDTYPE
    assert lib.todgpu_pointing_params(*args(4, _native.F64, None)) == _native.EINVAL
    assert lib.todgpu_pointing_params(*args(0, _native.F32, None)) == 0
    assert lib.todgpu_last_error_string()


def test_static_entry_rejects_nside_above_its_table():
    """todgpu_gather_accum_static holds a ring table for nside <= 4096 only and
    rejects larger maps before any CUDA call."""
    lib = _native.lib()
    a = _args(nside=8192, B=4, S=4, C=1, c_q=-1, c_u=-1, map_dtype=_native.F64, map_stride=12 * 8192 * 8192,
              tod_stride=4)
    for name in ("vec_orig", "axes", "cos_a", "sin_a", "ax_pts", "cos_p", "sin_p", "beam_vals", "map", "tod"):
        setattr(a, name, 16)  # never dereferenced: the size check comes first
    assert lib.todgpu_gather_accum_static(ctypes.byref(a), None) == _native.ENSIDE
    assert b"4096" in lib.todgpu_last_error_string()
