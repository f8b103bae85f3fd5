"""The gather's two CTA shapes give the same TOD bit for bit.

A launch whose requested spin-2 table fits an eighth of an SM's shared memory
runs 128-thread CTAs, 8 per SM; TODGPU_FLAG_WIDE_CTAS (and any larger table)
runs 256-thread CTAs.  Either way the beam pixels of a sample are summed in the
same 256 strided partial sums, reduced in the same order, so the TOD must not
change: for both interpolation modes, every map type, the three pointing forms,
beams of a few pixels and beams too large to stage, and the batched launch."""

import math

import numpy as np
import pytest
import torch

from tod_generation_mapbased_beam_b200 import _native
from tod_generation_mapbased_beam_b200 import workloads as W
from tod_generation_mapbased_beam_b200.batched import DetectorBatch
from tod_generation_mapbased_beam_b200.kernels import (beam_reach, gather_accum, gather_accum_angles, pack_map,
                                                       table_slots)

pytestmark = pytest.mark.gpu

# spin-2 table slots of a 128-thread CTA at 8 per SM: (228 KiB / 8 - 3 KiB
# reserved - 1312 B table header of 80 window rings) / 16 B per float64 pair;
# the request must also need at most those 80 rings (3 sqrt(slots / 3.2) + 6)
NARROW_F64_SLOTS = (228 * 1024 // 8 - 1024 - 2048 - (32 + 16 * 80)) // 16
WIDE = _native.FLAG_WIDE_CTAS


def _narrow(slots):
    return 0 < slots <= NARROW_F64_SLOTS and math.ceil(3.0 * math.sqrt(slots / 3.2)) + 6 <= 80


def _beam(S, seed, radius_deg=0.7):
    rng = np.random.default_rng(seed)
    r = np.radians(radius_deg) * np.sqrt(rng.uniform(0, 1, S))
    a = rng.uniform(0, 2 * np.pi, S)
    vec = np.stack([np.sin(r) * np.cos(a), np.sin(r) * np.sin(a), np.cos(r)], -1)
    bv = rng.uniform(0.1, 1.0, S).astype(np.float32)
    return vec, bv / bv.sum()


def _ref_params(B, seed):
    rng = np.random.default_rng(seed)
    ax = rng.standard_normal((B, 3))
    ax = (ax / np.linalg.norm(ax, axis=1, keepdims=True)).astype(np.float32)
    ang = rng.uniform(0, np.pi, B).astype(np.float32)
    th = rng.uniform(0.02, np.pi - 0.02, B)
    ph = rng.uniform(0, 2 * np.pi, B)
    pts = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1).astype(np.float32)
    psi = rng.uniform(0, 2 * np.pi, B).astype(np.float32)
    return [ax, np.cos(ang), np.sin(ang), pts, np.cos(psi), np.sin(psi)], (th, ph, psi.astype(np.float64))


def _sky(nside, seed):
    return torch.from_numpy(np.random.default_rng(seed).standard_normal((3, 12 * nside * nside))).cuda()


def test_narrow_shape_is_taken():
    """The workloads below ask for tables the narrow shape holds (else both
    launches would be wide and the comparison empty)."""
    for nside, S in ((512, 900), (256, 1300)):
        vec, _ = _beam(S, 3)
        assert _narrow(table_slots(nside, beam_reach(vec.astype(np.float32), nside)))


@pytest.mark.parametrize("interp", [_native.BILINEAR, _native.NEAREST])
@pytest.mark.parametrize("kind", ["planar", "f64", "f32", "bf16"])
def test_reference_typed_params(interp, kind):
    nside, B, S = 512, 900, 900
    vec, bv = _beam(S, 3)
    params, _ = _ref_params(B, 4)
    sky = _sky(nside, 5)
    mp = sky if kind == "planar" else pack_map(sky, kind)
    outs = []
    for flags in (0, WIDE):
        tod = torch.zeros((3, B), dtype=torch.float64, device="cuda")
        gather_accum(interp, vec.astype(np.float32), *params, nside, mp, bv, B, S, tod, 1, 2, flags=flags)
        outs.append(tod.cpu().numpy())
    assert np.abs(outs[0]).max() > 0
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("interp", [_native.BILINEAR, _native.NEAREST])
@pytest.mark.parametrize("precompute", [True, False])
@pytest.mark.parametrize("S", [1, 5, 1300])
def test_angles(interp, precompute, S):
    nside, B = 256, 700
    vec, bv = _beam(S, 6)
    _, (th, ph, ps) = _ref_params(B, 7)
    sky = _sky(nside, 8)
    ang = [torch.from_numpy(a).cuda() for a in (th, ph, ps)]
    outs = []
    for flags in (0, WIDE):
        tod = torch.zeros((3, B), dtype=torch.float64, device="cuda")
        gather_accum_angles(interp, vec, *ang, 0.2, 0.01, nside, pack_map(sky, "f64"), bv, tod, c_q=1, c_u=2,
                            flags=flags, precompute=precompute)
        outs.append(tod.cpu().numpy())
    assert np.abs(outs[0]).max() > 0
    assert np.array_equal(outs[0], outs[1])


def test_intensity_only_and_generic_layout():
    """I alone, and I/Q/U in another component order."""
    nside, B, S = 256, 500, 700
    vec, bv = _beam(S, 9)
    params, _ = _ref_params(B, 10)
    sky = _sky(nside, 11)
    for mp, c_q, c_u in ((sky[:1].contiguous(), -1, -1), (sky[[2, 0, 1]].contiguous(), 2, 0)):
        outs = []
        for flags in (0, WIDE):
            tod = torch.zeros((mp.shape[0], B), dtype=torch.float64, device="cuda")
            gather_accum(_native.BILINEAR, vec.astype(np.float32), *params, nside, mp, bv, B, S, tod, c_q, c_u,
                         flags=flags)
            outs.append(tod.cpu().numpy())
        assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("mode", ["bilinear", "nearest"])
def test_batched(mode):
    dets, sky = W.config4(n_det=5, seed=45, n_min=300, n_max=2500, nside=128, beam_nside=512)
    outs = []
    for wide in (False, True):
        batch = DetectorBatch(128, sky, dets, interp_mode=mode, tile=4, graph=False, wide_ctas=wide)
        batch.run()
        torch.cuda.synchronize()
        outs.append([o.cpu().numpy() for o in batch.out])
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
