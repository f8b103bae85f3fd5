"""The allocation-free entry point, todgpu_gather_accum_static.

Some callers cannot allocate device memory -- for example a host application
whose device memory is owned by another framework's allocator, or a foreign-
language binding that can pass existing buffers but cannot create new ones.
For them the library offers an entry point whose only scratch memory (the
ring table) is a fixed-size array built into the library.  These tests call
it through the C ABI twice in a row and check both results against the
regular entry point, which uses a caller-allocated ring table, for every
pointing mode (reference float32 parameters, float64 parameters, angles), a
packed map and an entry without Q and U.  They are kept in a file of their
own that pytest collects last.
"""

import ctypes

import numpy as np
import pytest
import torch

from tod_generation_mapbased_beam_b200 import _native
from tod_generation_mapbased_beam_b200.kernels import (beam_reach, boresight_phi_host, make_args, pack_map,
                                                       pointing_params, ring_table)

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
    angles = (th, ph, psi.astype(np.float64))
    return params, mp, bv, angles


def _args(pmode, interp, nside, params, angles, mp, bv, tod, comps, table):
    """todgpu_gather_args for one pointing mode ("f32", "f64" or "angles")."""
    dev = torch.device("cuda")
    B, S = params[1].shape[0], params[0].shape[0]
    C, c_q, c_u = (3, 1, 2) if comps == "IQU" else (1, -1, -1)
    beam = torch.from_numpy(bv).to(dev)
    if pmode == "f32":
        tp = [torch.from_numpy(np.ascontiguousarray(p)).to(dev) for p in params]
        bore = torch.from_numpy(boresight_phi_host(params[4])).to(dev)
        a = make_args(interp, nside, B, S, C, c_q, c_u, tp, np.float32, bore, beam, mp, tod, table=table)
        keep = tp + [bore]
    else:
        vec = torch.from_numpy(params[0].astype(np.float64)).to(dev)
        th, ph, ps = (torch.from_numpy(x).to(dev) for x in angles)
        if pmode == "f64":
            rot = list(pointing_params(th, ph, ps, 0.3, 0.02))
            a = make_args(interp, nside, B, S, C, c_q, c_u, [vec] + rot, np.float64, None, beam, mp, tod,
                          table=table)
            keep = [vec] + rot
        else:
            a = make_args(interp, nside, B, S, C, c_q, c_u, [vec] + [None] * 6, np.float64, None, beam, mp, tod,
                          table=table)
            a.params_dtype = _native.ANGLES
            a.theta, a.phi, a.psi = th.data_ptr(), ph.data_ptr(), ps.data_ptr()
            a.angles_dtype = _native.F64
            a.center_phi, a.center_theta = 0.3, 0.02
            keep = [vec, th, ph, ps]
    return a, keep + [beam]


def _run(entry, pmode, interp, nside, params, angles, mp, bv, comps="IQU", table=None):
    dev = torch.device("cuda")
    B = params[1].shape[0]
    C = 3 if comps == "IQU" else 1
    tod = torch.zeros((C, B), dtype=torch.float64, device=dev)
    args, _keep = _args(pmode, interp, nside, params, angles, mp, bv, tod, comps, table)
    rc = entry(ctypes.byref(args), torch.cuda.current_stream().cuda_stream)
    _native.check(rc)
    torch.cuda.synchronize()
    return tod.cpu().numpy()


def _map(mp, kind, comps):
    sky = torch.from_numpy(mp if comps == "IQU" else mp[:1].copy()).cuda()
    return sky if kind == "planar_f64" else pack_map(sky, kind)


@pytest.mark.parametrize("interp", [_native.BILINEAR, _native.NEAREST])
@pytest.mark.parametrize("pmode, kind, comps", [
    ("f32", "planar_f64", "IQU"),
    ("f64", "planar_f64", "IQU"),
    ("angles", "planar_f64", "IQU"),
    ("angles", "f32", "IQU"),
    ("f32", "planar_f64", "I"),
])
def test_static_entry_matches_regular_entry(interp, pmode, kind, comps):
    lib = _native.lib()
    nside, B, S = 1024, 600, 800
    params, mp, bv, angles = _inputs(nside, B, S, seed=91)
    dmap = _map(mp, kind, comps)
    table = ring_table(nside, beam_reach(params[0], nside))
    ref = _run(lib.todgpu_gather_accum, pmode, interp, nside, params, angles, dmap, bv, comps, table=table)
    first = _run(lib.todgpu_gather_accum_static, pmode, interp, nside, params, angles, dmap, bv, comps)
    second = _run(lib.todgpu_gather_accum_static, pmode, interp, nside, params, angles, dmap, bv, comps)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(first - ref).max() <= TOD_RTOL * scale
    assert np.abs(second - ref).max() <= TOD_RTOL * scale


def test_static_entry_follows_a_different_nside():
    """The built-in table is rebuilt per call: a call at another nside and
    beam right after the first still matches the regular entry point."""
    lib = _native.lib()
    for nside, S, seed in ((256, 300, 5), (64, 120, 6)):
        params, mp, bv, angles = _inputs(nside, 200, S, seed)
        dmap = _map(mp, "planar_f64", "IQU")
        table = ring_table(nside, beam_reach(params[0], nside))
        ref = _run(lib.todgpu_gather_accum, "f32", _native.BILINEAR, nside, params, angles, dmap, bv, table=table)
        got = _run(lib.todgpu_gather_accum_static, "f32", _native.BILINEAR, nside, params, angles, dmap, bv)
        assert np.abs(got - ref).max() <= TOD_RTOL * np.abs(ref).max()
