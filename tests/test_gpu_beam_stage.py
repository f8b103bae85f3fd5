"""The beam in shared memory.

When a launch leaves room beside the spin-2 table, every CTA copies its
beam (pixel vectors and weights) into shared memory with bulk copies and the
pixel loop reads it from there; the 16-byte aligned middle of each array goes
by cp.async.bulk, the unaligned ends by plain loads.  The TOD must be the same
bit for bit as with the beam read from global memory (TODGPU_FLAG_NO_BEAM_STAGE),
for every pointing mode, both interpolation modes (nearest launches never
stage: the comparison then covers the flag alone), beams whose arrays start at
any element offset, and beams too large to stage (read from global memory
either way).  No bounded wait of the copies may run out."""

import numpy as np
import pytest
import torch

from tod_generation_mapbased_beam_b200 import _native
from tod_generation_mapbased_beam_b200.kernels import gather_accum, gather_accum_angles, pack_map

pytestmark = pytest.mark.gpu


def _beam(S, seed, radius_deg=0.7):
    rng = np.random.default_rng(seed)
    r = np.radians(radius_deg) * np.sqrt(rng.uniform(0, 1, S))
    a = rng.uniform(0, 2 * np.pi, S)
    vec = np.stack([np.sin(r) * np.cos(a), np.sin(r) * np.sin(a), np.cos(r)], -1)
    bv = rng.uniform(0.1, 1.0, S).astype(np.float32)
    return vec, bv / bv.sum()


def _offset_view(arr, dtype, offset):
    """A CUDA tensor holding arr that starts `offset` elements into its buffer."""
    flat = torch.from_numpy(np.ascontiguousarray(arr, dtype=dtype).reshape(-1))
    buf = torch.zeros(flat.numel() + offset + 3, dtype=flat.dtype, device="cuda")
    buf[offset:offset + flat.numel()] = flat.cuda()
    return buf[offset:offset + flat.numel()].view(arr.shape)


def _ref_params(B, seed):
    rng = np.random.default_rng(seed)
    ax = rng.standard_normal((B, 3))
    ax = (ax / np.linalg.norm(ax, axis=1, keepdims=True)).astype(np.float32)
    ang = rng.uniform(0, np.pi, B).astype(np.float32)
    th = rng.uniform(0.05, np.pi - 0.05, B)
    ph = rng.uniform(0, 2 * np.pi, B)
    pts = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1).astype(np.float32)
    psi = rng.uniform(0, 2 * np.pi, B).astype(np.float32)
    return [ax, np.cos(ang), np.sin(ang), pts, np.cos(psi), np.sin(psi)], (th, ph, psi.astype(np.float64))


@pytest.mark.parametrize("interp", [_native.BILINEAR, _native.NEAREST])
@pytest.mark.parametrize("offset", [0, 1, 2, 3])
def test_reference_typed_beam_staged_equals_global(interp, offset):
    nside, B, S = 512, 700, 900
    vec, bv = _beam(S, 3)
    params, _ = _ref_params(B, 4)
    sky = torch.from_numpy(np.random.default_rng(5).standard_normal((3, 12 * nside * nside))).cuda()
    mp = pack_map(sky, "f64")
    v = _offset_view(vec, np.float32, offset)
    b = _offset_view(bv, np.float32, (offset * 3) % 4)
    outs = []
    for flags in (0, _native.FLAG_NO_BEAM_STAGE):
        tod = torch.zeros((3, B), dtype=torch.float64, device="cuda")
        gather_accum(interp, v, *params, nside, mp, b, B, S, tod, 1, 2, flags=flags)
        outs.append(tod.cpu().numpy())
    assert np.abs(outs[0]).max() > 0
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("interp", [_native.BILINEAR, _native.NEAREST])
@pytest.mark.parametrize("kind", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("precompute", [True, False])
def test_float64_beam_staged_equals_global(interp, kind, precompute):
    nside, B, S = 512, 500, 1300
    vec, bv = _beam(S, 6)
    _, (th, ph, ps) = _ref_params(B, 7)
    sky = torch.from_numpy(np.random.default_rng(8).standard_normal((3, 12 * nside * nside))).cuda()
    mp = pack_map(sky, kind)
    v = _offset_view(vec, np.float64, 1)
    b = _offset_view(bv, np.float32, 2)
    ang = [torch.from_numpy(a).cuda() for a in (th, ph, ps)]
    outs = []
    for flags in (0, _native.FLAG_NO_BEAM_STAGE):
        tod = torch.zeros((3, B), dtype=torch.float64, device="cuda")
        gather_accum_angles(interp, v, *ang, 0.2, 0.01, nside, mp, b, tod, c_q=1, c_u=2, flags=flags,
                            precompute=precompute)
        outs.append(tod.cpu().numpy())
    assert np.abs(outs[0]).max() > 0
    assert np.array_equal(outs[0], outs[1])


def test_large_beam_and_tiny_beam():
    """A beam too large for shared memory (read from global memory by both
    launches) and a beam of a few pixels (no aligned middle at all)."""
    nside = 256
    sky = torch.from_numpy(np.random.default_rng(9).standard_normal((3, 12 * nside * nside))).cuda()
    mp = pack_map(sky, "f64")
    _, (th, ph, ps) = _ref_params(64, 10)
    ang = [torch.from_numpy(a).cuda() for a in (th, ph, ps)]
    for S, offset in ((20000, 0), (1, 1), (3, 3)):
        vec, bv = _beam(S, 11, radius_deg=3.0)
        v = _offset_view(vec, np.float64, offset)
        b = _offset_view(bv, np.float32, offset)
        outs = []
        for flags in (0, _native.FLAG_NO_BEAM_STAGE):
            tod = torch.zeros((3, 64), dtype=torch.float64, device="cuda")
            gather_accum_angles(_native.BILINEAR, v, *ang, 0.0, 0.0, nside, mp, b, tod, c_q=1, c_u=2, flags=flags)
            outs.append(tod.cpu().numpy())
        assert np.array_equal(outs[0], outs[1]), S


def test_no_wait_ran_out():
    assert _native.lib().todgpu_gather_wait_timeouts() == 0
