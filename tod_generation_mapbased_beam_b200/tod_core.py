"""Batch TOD dispatch (drop-in for ``tod_core.beam_tod_batch``,
tod_core.py:52-167).

``beam_tod_batch`` accumulates the TOD contribution of one beam entry for a
batch of samples on the GPU and returns ``{stokes_component: float32 (B,)}``
exactly like the reference: component -> (c_q, c_u) mapping (spin-2 only when
the entry carries both Q and U, tod_core.py:105-112), the ``interp_mode``
check with the same ValueError (tod_core.py:114-119), float32 rotation
parameters prepared on the host as in tod_core.py:121-125, a zeroed float64
accumulator (tod_core.py:128) and the float32 cast of the result
(tod_core.py:165-167).

Differences, all additive:
* map, beam vectors and weights may be torch CUDA tensors (zero copy); numpy
  inputs are uploaded once per array object and cached on the device;
* without ``data["mp_stacked"]`` the ``mp`` component list is stacked and
  uploaded (the reference falls back to a healpy path there, which needs
  healpy; the result is the same gather);
* a float64 map is kept on the device as float64 records {I, Q, U, 0} (one
  memory sector per pixel; the same TOD bit for bit);
* ``return_device=True`` returns the (C, B) float64 CUDA accumulator instead
  of the float32 host dict.
"""

from __future__ import annotations

import weakref

import numpy as np
import torch

from . import _native
from ._device import is_tensor, require_cuda
from .kernels import beam_center_angles, boresight_phi_host, gather_accum, gather_accum_angles, pack_map
from .tod_rotations import _rotation_params, precompute_rotation_vector_batch  # noqa: F401

_INTERP = {"bilinear": _native.BILINEAR, "nearest": _native.NEAREST}


class _UploadCache:
    """Device copies of read-only host arrays, keyed by array identity and
    dropped when the host array is garbage-collected."""

    def __init__(self):
        self._store = {}

    def get(self, arr, dtype):
        if is_tensor(arr):
            t = arr.to(device="cuda", dtype=dtype)
            return t.contiguous()
        key = (id(arr), np.dtype(dtype).str if not isinstance(dtype, torch.dtype) else str(dtype))
        hit = self._store.get(key)
        if hit is not None and hit[1]() is arr:
            return hit[0]
        np_dt = {torch.float32: np.float32, torch.float64: np.float64}[dtype]
        t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np_dt)).to("cuda")
        try:
            ref = weakref.ref(arr, lambda _r, k=key: self._store.pop(k, None))
        except TypeError:
            return t
        self._store[key] = (t, ref)
        return t


_cache = _UploadCache()


def _map_dtype(mp):
    if is_tensor(mp):
        return mp.dtype if mp.dtype in (torch.float32, torch.float64) else torch.float64
    return torch.float32 if np.asarray(mp).dtype == np.float32 else torch.float64


def stacked_map(data, mp):
    """Device (C, N) map of a beam entry: ``data['mp_stacked']`` if present,
    else the entry's components stacked from the ``mp`` list."""
    ms = data.get("mp_stacked")
    if ms is not None:
        return _cache.get(ms, _map_dtype(ms))
    comps = data["comp_indices"]
    key = "_todgpu_stacked"
    cached = data.get(key)
    if cached is not None:
        return cached
    parts = [mp[c] for c in comps]
    if all(is_tensor(p) for p in parts):
        t = torch.stack([p.to("cuda") for p in parts]).contiguous()
    else:
        arr = np.stack([np.asarray(p) for p in parts])
        t = torch.from_numpy(arr).to("cuda").contiguous()
    data[key] = t
    return t


_packed = {}  # id(planar device map) -> (PackedMap, weak reference to the planar map)


def device_map(data, mp):
    """The entry's device map in the layout the kernels read fastest: a
    float64 map of up to 4 components as float64 records {I, Q, U, 0}
    (packed once and cached; the TOD is the same bit for bit), a float32 map
    planar (its float32 products are part of the reference's result)."""
    t = stacked_map(data, mp)
    if t.dtype != torch.float64 or t.shape[0] > 4:
        return t
    key = id(t)
    hit = _packed.get(key)
    if hit is not None and hit[1]() is t:
        return hit[0]
    pm = pack_map(t, "f64")
    try:
        ref = weakref.ref(t, lambda _r, k=key: _packed.pop(k, None))
    except TypeError:
        return pm
    _packed[key] = (pm, ref)
    return pm


def component_slots(comp_indices):
    """(c_q, c_u): positions of Stokes Q (1) and U (2) in comp_indices, or -1."""
    c_q = c_u = -1
    for i, comp in enumerate(comp_indices):
        if comp == 1:
            c_q = i
        elif comp == 2:
            c_u = i
    return c_q, c_u


def beam_tod_batch(nside, mp, data, rot_vecs, phi_b, theta_b, psis_b, interp_mode="bilinear",
                   *, return_device=False):
    """GPU replacement of ``tod_core.beam_tod_batch`` (tod_core.py:52-167)."""
    B = int(phi_b.shape[0])
    vec_orig = data["vec_orig"]
    beam_vals = data["beam_vals"]
    S = int(vec_orig.shape[0])
    comp_indices = list(data["comp_indices"])
    C = len(comp_indices)
    c_q, c_u = component_slots(comp_indices)
    if interp_mode not in ("nearest", "bilinear"):
        raise ValueError(
            f"interp_mode {interp_mode!r} not available on main branch; "
            "switch to the 'gaussian' or 'bicubic' branch")
    require_cuda()
    params = _rotation_params(rot_vecs, phi_b, theta_b, psis_b)
    bore_phi = boresight_phi_host(params[3]) if (c_q >= 0 and c_u >= 0) else None
    vec = _cache.get(vec_orig, torch.float32)
    bv = _cache.get(beam_vals, torch.float32)
    mpd = device_map(data, mp)
    tod = torch.zeros((C, B), dtype=torch.float64, device=mpd.device)
    gather_accum(_INTERP[interp_mode], vec, *params, nside, mpd, bv, B, S, tod, c_q, c_u,
                 bore_phi=bore_phi if bore_phi is not None else np.zeros(B, np.float32))
    if return_device:
        return tod
    host = tod.to(torch.float32).cpu().numpy()
    return {comp: host[i] for i, comp in enumerate(comp_indices)}


def beam_tod_angles(nside, data, theta_b, phi_b, psi_b, interp_mode="bilinear", *,
                    center=None, mp=None, return_device=False):
    """Device-pointing variant of :func:`beam_tod_batch` for one beam entry.

    Takes the scan angles themselves -- ``theta_b, phi_b, psi_b`` (B,), float32
    as the reference driver reads them (gridint.py:277-279) or float64 -- and
    derives each sample's rotation on the GPU in float64 (the steps of
    ``precompute_rotation_vector_batch`` and ``_rotation_params`` with the roll
    psi_b - beta, gridint.py:280-281), without the reference's float32
    parameter rounding.  ``center`` is (phi_c, theta_c) of the beam centre;
    by default the centre of ``data['ra'], data['dec']``.
    Returns ``{comp: float32 (B,)}`` or the float64 (C, B) CUDA tensor."""
    B = int(np.asarray(theta_b).shape[0]) if not is_tensor(theta_b) else int(theta_b.shape[0])
    comp_indices = list(data["comp_indices"])
    C = len(comp_indices)
    c_q, c_u = component_slots(comp_indices)
    if interp_mode not in ("nearest", "bilinear"):
        raise ValueError(
            f"interp_mode {interp_mode!r} not available on main branch; "
            "switch to the 'gaussian' or 'bicubic' branch")
    require_cuda()
    if center is None:
        center = beam_center_angles(data["ra"], data["dec"])
    vec = _cache.get(data["vec_orig"], torch.float64)
    bv = _cache.get(data["beam_vals"], torch.float32)
    mpd = device_map(data, mp)
    tod = torch.zeros((C, B), dtype=torch.float64, device=mpd.device)
    gather_accum_angles(_INTERP[interp_mode], vec, theta_b, phi_b, psi_b, center[0], center[1], nside,
                        mpd, bv, tod, c_q, c_u)
    if return_device:
        return tod
    host = tod.to(torch.float32).cpu().numpy()
    return {comp: host[i] for i, comp in enumerate(comp_indices)}
