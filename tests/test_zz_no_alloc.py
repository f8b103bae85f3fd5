"""The allocation-free entry point, todgpu_gather_accum_static.

Some callers cannot allocate device memory -- for example a host application
whose device memory is owned by another framework's allocator, or a foreign-
language binding that can pass existing buffers but cannot create new ones.
For them the library offers an entry point whose only scratch memory (the
ring table) is a fixed-size array built into the library.  This test calls
it through the C ABI twice in a row and checks both results against the
regular entry point, which uses a caller-allocated ring table.  It is kept in
a file of its own that pytest collects last.
"""

import ctypes

import numpy as np
import pytest
import torch

from tod_generation_mapbased_beam_b200 import _native
from tod_generation_mapbased_beam_b200.kernels import (beam_reach, boresight_phi_host, make_args,
                                                       ring_table)

pytestmark = pytest.mark.gpu

TOD_RTOL = 1e-12  # the tolerance of the other parity tests


def _inputs(nside, B, S, seed):
    rng = np.random.default_rng(seed)
    r = np.radians(0.6) * np.sqrt(rng.uniform(0, 1, S))
    a = rng.uniform(0, 2 * np.pi, S)
    vec = np.stack([np.sin(r) * np.cos(a), np.sin(r) * np.sin(a), np.cos(r)], -1).astype(np.float32)
    ax = rng.standard_normal((B, 3))
    ax = (ax / np.linalg.norm(ax, axis=1, keepdims=True)).astype(np.float32)
    ang = rng.uniform(0, np.pi, B).astype(np.float32)
    th = rng.uniform(0.05, np.pi - 0.05, B)
    ph = rng.uniform(0, 2 * np.pi, B)
    pts = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1).astype(np.float32)
    psi = rng.uniform(0, 2 * np.pi, B).astype(np.float32)
    params = [vec, ax, np.cos(ang), np.sin(ang), pts, np.cos(psi), np.sin(psi)]
    mp = rng.standard_normal((3, 12 * nside * nside))
    bv = rng.uniform(0.1, 1.0, S).astype(np.float32)
    bv /= bv.sum()
    return params, mp, bv


def _run(entry, interp, nside, params, mp, bv, table=None):
    dev = torch.device("cuda")
    B, S = params[1].shape[0], params[0].shape[0]
    tp = [torch.from_numpy(np.ascontiguousarray(p)).to(dev) for p in params]
    bore = torch.from_numpy(boresight_phi_host(params[4])).to(dev)
    beam = torch.from_numpy(bv).to(dev)
    sky = torch.from_numpy(mp).to(dev)
    tod = torch.zeros((3, B), dtype=torch.float64, device=dev)
    args = make_args(interp, nside, B, S, 3, 1, 2, tp, np.float32, bore, beam, sky, tod, table=table)
    rc = entry(ctypes.byref(args), torch.cuda.current_stream().cuda_stream)
    _native.check(rc)
    torch.cuda.synchronize()
    return tod.cpu().numpy()


@pytest.mark.parametrize("interp", [_native.BILINEAR, _native.NEAREST])
def test_static_entry_matches_regular_entry(interp):
    lib = _native.lib()
    nside, B, S = 1024, 600, 800
    params, mp, bv = _inputs(nside, B, S, seed=91)
    table = ring_table(nside, beam_reach(params[0], nside))
    ref = _run(lib.todgpu_gather_accum, interp, nside, params, mp, bv, table=table)
    first = _run(lib.todgpu_gather_accum_static, interp, nside, params, mp, bv)
    second = _run(lib.todgpu_gather_accum_static, interp, nside, params, mp, bv)
    scale = np.abs(ref).max()
    assert np.abs(first - ref).max() <= TOD_RTOL * scale
    assert np.abs(second - ref).max() <= TOD_RTOL * scale


def test_static_entry_follows_a_different_nside():
    """The built-in table is rebuilt per call: a call at another nside and
    beam right after the first still matches the regular entry point."""
    lib = _native.lib()
    for nside, S, seed in ((256, 300, 5), (64, 120, 6)):
        params, mp, bv = _inputs(nside, 200, S, seed)
        table = ring_table(nside, beam_reach(params[0], nside))
        ref = _run(lib.todgpu_gather_accum, _native.BILINEAR, nside, params, mp, bv, table=table)
        got = _run(lib.todgpu_gather_accum_static, _native.BILINEAR, nside, params, mp, bv)
        assert np.abs(got - ref).max() <= TOD_RTOL * np.abs(ref).max()


def test_static_entry_rejects_nside_above_its_table():
    lib = _native.lib()
    a = _native.GatherArgs()
    a.abi_version = _native.ABI_VERSION
    a.interp = _native.BILINEAR
    a.nside = 8192
    a.B = 4
    a.S = 4
    a.C = 1
    a.c_q = -1
    a.c_u = -1
    a.map_stride = 12 * 8192 * 8192
    a.tod_stride = 4
    for name in ("vec_orig", "axes", "cos_a", "sin_a", "ax_pts", "cos_p", "sin_p", "beam_vals", "map", "tod"):
        setattr(a, name, 16)  # never dereferenced: the size check comes first
    assert lib.todgpu_gather_accum_static(ctypes.byref(a), None) == _native.ENSIDE
    assert b"4096" in lib.todgpu_last_error_string()
