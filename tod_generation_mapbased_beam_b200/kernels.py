"""Kernel-level entry points with the reference's Numba kernel ABI.

``gather_accum`` runs one fused gather/accumulate launch through
``todgpu_gather_accum``.  Arguments follow ``_gather_accum_fused_jit``
(tod_bilinear.py:205-222) and ``_gather_accum_nearest_jit``
(tod_nearest.py:21-38): beam-frame vectors, the six per-sample rotation
arrays, nside, the planar (C, N) map, beam weights, B, S, the (C, B) float64
output accumulated in place, and the Q/U component positions.

Inputs may be numpy arrays or torch tensors (CPU or CUDA).  When ``tod`` is a
numpy array it is copied to the GPU, accumulated there and copied back in
place, exactly like the reference mutates its argument; CUDA tensors are
updated in place without a host round trip.

Precision follows the parameter dtype, as it does in the reference (Numba
specialises the kernel on it): float32 parameters are combined with the
reference's float32/float64 operand typing (bit-parity form), float64
parameters give an all-float64 computation.
"""

from __future__ import annotations

import ctypes
import math
import weakref

import numpy as np
import torch

from . import _native
from ._device import dtype_of, is_tensor, ptr, require_cuda, stream_handle, to_device

_PARAM_NAMES = ("vec_orig", "axes", "cos_a", "sin_a", "ax_pts", "cos_p", "sin_p")


def _param_dtype(arrs):
    dts = {dtype_of(a) for a in arrs}
    if dts == {np.dtype(np.float32)}:
        return np.float32
    if dts == {np.dtype(np.float64)}:
        return np.float64
    raise TypeError("vec_orig and the rotation parameter arrays must all be float32 "
                    f"(reference typing) or all float64; got {sorted(str(d) for d in dts)}")


def boresight_phi_host(ax_pts) -> np.ndarray:
    """atan2f(ax_pts[:,1], ax_pts[:,0]) with the host C library (float32),
    the boresight longitude the reference kernels compute
    (tod_bilinear.py:308, tod_nearest.py:87)."""
    if is_tensor(ax_pts):
        ax_pts = ax_pts.detach().to("cpu")
        a = np.ascontiguousarray(ax_pts.numpy(), dtype=np.float32)
    else:
        a = np.ascontiguousarray(np.asarray(ax_pts), dtype=np.float32)
    a = a.reshape(-1, 3)
    out = np.empty(a.shape[0], dtype=np.float32)
    _native.check(_native.lib().todgpu_boresight_phi_host(
        a.ctypes.data_as(ctypes.c_void_p), a.shape[0], out.ctypes.data_as(ctypes.c_void_p), 0))
    return out


_RING_TABLES = {}
_REACH_STEP = 1e-4  # ring tables are built for reaches rounded up to this step [rad]


_REACH = {}  # (tensor identity, version, nside) -> (reach, weak reference to the tensor)


def beam_reach(vec_orig, nside):
    """Angular radius [rad] that every stencil neighbour of the rotated beam
    stays within around the rotated beam centre: the beam's radius about its
    mean direction plus 3/nside (stencil reach) plus float32 slack.  The
    kernel derives the same bound from the beam on the device and uses the
    ring table's spin-2 slots only if the table covers it.  For a CUDA tensor
    the value is remembered (until the tensor changes or is freed), so repeated
    calls do not copy the beam back to the host."""
    key = None
    if is_tensor(vec_orig):
        key = (id(vec_orig), vec_orig.data_ptr(), vec_orig._version, tuple(vec_orig.shape), int(nside))
        hit = _REACH.get(key)
        if hit is not None and hit[1]() is vec_orig:
            return hit[0]
    r = _beam_reach(vec_orig, nside)
    if key is not None:
        try:
            _REACH[key] = (r, weakref.ref(vec_orig, lambda _r, k=key: _REACH.pop(k, None)))
        except TypeError:
            pass
    return r


def _beam_reach(vec_orig, nside):
    v = vec_orig.detach().cpu().numpy() if is_tensor(vec_orig) else np.asarray(vec_orig)
    v = np.asarray(v, np.float64).reshape(-1, 3)
    if v.shape[0] == 0:
        return 0.0
    c = v.sum(axis=0)
    nc = np.linalg.norm(c)
    c = c / nc if nc > 0 else np.array([0.0, 0.0, 1.0])
    vn = np.linalg.norm(v, axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        d = np.where(vn > 0, (v @ c) / vn, -1.0)
    r = float(np.arccos(np.clip(d.min(), -1.0, 1.0)))
    return r + 3.0 / float(nside) + 2e-5


def _spread16(a):
    """The low 16 bits of a with a zero bit inserted after each."""
    a = a & 0xFFFF
    a = (a | (a << 8)) & 0x00FF00FF
    a = (a | (a << 4)) & 0x0F0F0F0F
    a = (a | (a << 2)) & 0x33333333
    a = (a | (a << 1)) & 0x55555555
    return a


def beam_order(vec_orig):
    """Order of a beam's pixels that puts neighbours on the sky next to each
    other: the Morton (Z) order of their coordinates in the plane orthogonal to
    the beam's mean direction, 16 bits per axis.  Consecutive pixels go to
    neighbouring threads of a warp, whose stencils then share memory sectors
    of the map (a 30' beam pixelised at nside 4096 over an nside 2048 map made
    16 sectors per gather request in its ring order).  Only the order of the
    sum over beam pixels changes."""
    v = vec_orig.detach().cpu().numpy() if is_tensor(vec_orig) else np.asarray(vec_orig)
    v = np.asarray(v, np.float64).reshape(-1, 3)
    n = v.shape[0]
    if n < 2:
        return np.arange(n, dtype=np.int64)
    c = v.sum(axis=0)
    nc = np.linalg.norm(c)
    c = c / nc if nc > 0 else np.array([0.0, 0.0, 1.0])
    a = np.zeros(3)
    a[int(np.argmin(np.abs(c)))] = 1.0
    e1 = np.cross(c, a)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(c, e1)
    code = np.zeros(n, dtype=np.int64)
    for shift, e in ((0, e1), (1, e2)):
        x = v @ e
        lo, hi = x.min(), x.max()
        q = np.clip(((x - lo) / max(hi - lo, 1e-300) * 65535.0).astype(np.int64), 0, 65535)
        code |= _spread16(q) << shift
    return np.argsort(code, kind="stable")


_TABLE_REACH = {}  # data_ptr of a cached ring table -> the reach it was built for


def table_slots(nside, reach):
    """Spin-2 table slots a sample needs for a footprint of radius ``reach``
    [rad] away from the poles, an upper bound of what the kernel fills: per
    window ring the disc's stretch with 2% margin, rounded up to 2k + 1 slots
    -- at most 1.02 x 3 (reach nside)^2 for the disc plus 3 per ring over at
    most 3 reach nside + 4 rings -- with 5% more and 32 to spare.  The request
    also sizes the table header (256-thread CTAs reserve window rings for a
    disc of request / 3.2 pixels, 128-thread CTAs a fixed 80).  Shared memory beyond them is left to L1, and a
    request of up to about 1500 slots (float64 tables; 1900 float32) lets the
    launch run 128-thread CTAs, 8 per SM.  For a reach of 0.05 rad or more the
    kernel reserves whole ring stretches instead of the disc, and the
    library's default (0) is asked for."""
    r = float(reach)
    n = float(nside)
    if not r < 0.05:
        return 0
    x = r * n
    need = 1.02 * 3.0 * x * x + 3.0 * (3.0 * x + 4.0)
    return int(min(1 << 20, math.ceil(1.05 * need) + 32))


def table_slots_for(table, nside):
    """``table_slots`` for a table made by :func:`ring_table` (0, the
    library's default, for any other table or none)."""
    if table is None:
        return 0
    reach = _TABLE_REACH.get(table.data_ptr()) if is_tensor(table) else None
    return 0 if reach is None else table_slots(nside, reach)


def ring_table(nside, reach, device=None):
    """Device ring table for ``nside`` covering footprints up to ``reach``
    (built once and cached per device, nside and rounded reach)."""
    dev = device if device is not None else require_cuda()
    reach_q = min(np.pi, np.ceil(reach / _REACH_STEP) * _REACH_STEP)
    key = (dev.index if isinstance(dev, torch.device) else int(dev), int(nside), round(reach_q / _REACH_STEP))
    t = _RING_TABLES.get(key)
    if t is None:
        nbytes = int(_native.lib().todgpu_ring_table_bytes(int(nside)))
        if nbytes == 0:
            raise _native.TodGpuError(_native.ENSIDE, f"nside {nside} out of range")
        t = torch.empty(nbytes // 8, dtype=torch.float64, device=dev)
        _native.check(_native.lib().todgpu_ring_table_build(int(nside), float(reach_q), t.data_ptr(),
                                                            nbytes, stream_handle()))
        _RING_TABLES[key] = t
        _TABLE_REACH[t.data_ptr()] = float(reach_q)
    return t


def _row_stride(t):
    """Row stride of a (rows, n) tensor with unit column stride; a single
    row's stride is free in torch (a ``[None, :]`` view may carry 0), so it
    is taken as n."""
    return t.stride(0) if t.shape[0] > 1 else t.shape[1]


def _set_map(a, mp):
    if isinstance(mp, PackedMap):
        a.map_dtype = mp.map_dtype
        a.map = mp.data.data_ptr()
        a.map_stride = mp.npix
    else:
        a.map_dtype = _native.F32 if mp.dtype == torch.float32 else _native.F64
        a.map = mp.data_ptr()
        a.map_stride = _row_stride(mp)


def _ncomp(mp):
    return mp.C if isinstance(mp, PackedMap) else mp.shape[0]


def make_args(interp, nside, B, S, C, c_q, c_u, params, pdt, bore_phi, beam, mp, tod,
              err=None, flags=0, table=None):
    a = _native.GatherArgs()
    a.abi_version = _native.ABI_VERSION
    a.interp = interp
    a.nside = int(nside)
    a.B = int(B)
    a.S = int(S)
    a.C = int(C)
    a.c_q = int(c_q)
    a.c_u = int(c_u)
    a.params_dtype = _native.F32 if pdt == np.float32 else _native.F64
    _set_map(a, mp)
    (a.vec_orig, a.axes, a.cos_a, a.sin_a, a.ax_pts, a.cos_p, a.sin_p) = [ptr(t) for t in params]
    a.bore_phi = ptr(bore_phi)
    a.beam_vals = ptr(beam)
    a.tod = ptr(tod)
    a.tod_stride = _row_stride(tod)
    a.err_count = ptr(err)
    a.flags = int(flags)
    a.ring_table = ptr(table)
    a.tab_slots = table_slots_for(table, nside)
    return a


class PackedMap:
    """A map with one record of 4 components per pixel: float32 (16 B) or
    bfloat16 (8 B) for the precision form, float64 (32 B) for the float64
    path with a pixel's components side by side (same results as the planar
    float64 map).  Built by :func:`pack_map`."""

    def __init__(self, data: torch.Tensor, C: int, kind: str):
        self.data = data
        self.C = int(C)
        self.kind = kind  # "f32" or "bf16"

    @property
    def map_dtype(self):
        return {"f32": _native.PACKED_F32, "bf16": _native.PACKED_BF16, "f64": _native.PACKED_F64}[self.kind]

    @property
    def npix(self):
        return self.data.shape[0]

    @property
    def device(self):
        return self.data.device


def pack_map(mp_stacked, kind="f32"):
    """Pack a planar (C, N) map (numpy or torch, float32/float64, C <= 4) into
    per-pixel records on the GPU (todgpu_pack_map): "f32" or "bf16" for the
    precision form, "f64" for the float64 path."""
    if kind not in ("f32", "bf16", "f64"):
        raise ValueError("kind must be 'f32', 'bf16' or 'f64'")
    mp = _map_tensor(mp_stacked)
    C, N = mp.shape
    if C > 4:
        raise ValueError("at most 4 components per record")
    dt = {"f32": torch.float32, "bf16": torch.bfloat16, "f64": torch.float64}[kind]
    out = torch.empty((N, 4), dtype=dt, device=mp.device)
    _native.check(_native.lib().todgpu_pack_map(
        mp.data_ptr(), _native.F32 if mp.dtype == torch.float32 else _native.F64, C, N, _row_stride(mp),
        {"f32": _native.PACKED_F32, "bf16": _native.PACKED_BF16, "f64": _native.PACKED_F64}[kind], out.data_ptr(),
        stream_handle()))
    return PackedMap(out, C, kind)


def _map_tensor(mp_stacked):
    if isinstance(mp_stacked, PackedMap):
        return mp_stacked
    dt = dtype_of(mp_stacked)
    if dt not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise TypeError(f"mp_stacked must be float32 or float64, got {dt}")
    mp = to_device(mp_stacked, dt.type)
    if mp.dim() != 2:
        raise ValueError("mp_stacked must be a (C, N) array")
    return mp


def gather_accum(interp, vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, mp_stacked,
                 beam_vals, B, S, tod, c_q=-1, c_u=-1, bore_phi=None, err_count=None, flags=0):
    """One fused launch; see the module docstring.  Returns ``tod``.

    ``err_count``: optional int64 CUDA tensor of one element that receives the
    number of (sample, beam pixel) terms skipped because a stencil pixel fell
    outside the map (only possible for non-finite pointing).
    ``flags``: ``_native.FLAG_NO_TABLES`` evaluates every ring quantity and
    spin-2 angle directly instead of from the per-sample footprint tables
    (identical results; for testing)."""
    require_cuda()
    B = int(B)
    S = int(S)
    nside = int(nside)
    raw = (vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p)
    pdt = _param_dtype(raw)
    shapes = [(S, 3), (B, 3), (B,), (B,), (B, 3), (B,), (B,)]
    params = [to_device(x, pdt, sh) for x, sh in zip(raw, shapes)]
    if dtype_of(beam_vals) != np.dtype(np.float32):
        raise TypeError("beam_vals must be float32 (the reference casts beam weights to float32)")
    beam = to_device(beam_vals, np.float32, (S,))
    mp = _map_tensor(mp_stacked)
    C = _ncomp(mp)
    if pdt == np.float32 and bore_phi is None and B > 0:
        bore_phi = boresight_phi_host(ax_pts if not is_tensor(ax_pts) else params[4])
    bphi = to_device(bore_phi, np.float32, (B,)) if (bore_phi is not None and pdt == np.float32) else None

    host_tod = None
    if is_tensor(tod) and tod.is_cuda:
        if tod.dtype != torch.float64 or tod.dim() != 2 or tod.stride(1) != 1:
            raise ValueError("tod must be a float64 (C, B) tensor with unit stride along B")
        dtod = tod
    else:
        host_tod = tod
        arr = tod.numpy() if is_tensor(tod) else tod
        if arr.dtype != np.float64 or arr.ndim != 2:
            raise ValueError("tod must be a float64 (C, B) array")
        dtod = torch.from_numpy(np.ascontiguousarray(arr)).to(params[0].device)
    if tuple(dtod.shape) != (C, B):
        raise ValueError(f"tod has shape {tuple(dtod.shape)}, expected {(C, B)}")

    table = None
    if not flags & _native.FLAG_NO_TABLES and B > 0 and S > 0:
        table = ring_table(nside, beam_reach(vec_orig, nside), params[0].device)
    args = make_args(interp, nside, B, S, C, c_q, c_u, params, pdt, bphi, beam, mp, dtod,
                     err_count, flags, table)
    _native.check(_native.lib().todgpu_gather_accum(ctypes.byref(args), stream_handle()))
    if host_tod is not None:
        res = dtod.cpu().numpy()
        if is_tensor(host_tod):
            host_tod.copy_(torch.from_numpy(res))
        else:
            host_tod[...] = res
    return tod


def bilinear_stencils(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, B, S):
    """Per-(b, s) bilinear pixels (4, B*S) int64 and weights (4, B*S) float64 of
    the fused path, as CUDA tensors."""
    require_cuda()
    B = int(B)
    S = int(S)
    raw = (vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p)
    pdt = _param_dtype(raw)
    shapes = [(S, 3), (B, 3), (B,), (B,), (B, 3), (B,), (B,)]
    params = [to_device(x, pdt, sh) for x, sh in zip(raw, shapes)]
    dev = params[0].device
    pix = torch.empty((4, B * S), dtype=torch.int64, device=dev)
    wgt = torch.empty((4, B * S), dtype=torch.float64, device=dev)
    a = _native.GatherArgs()
    a.abi_version = _native.ABI_VERSION
    a.nside = int(nside)
    a.B = B
    a.S = S
    a.params_dtype = _native.F32 if pdt == np.float32 else _native.F64
    (a.vec_orig, a.axes, a.cos_a, a.sin_a, a.ax_pts, a.cos_p, a.sin_p) = [ptr(t) for t in params]
    _native.check(_native.lib().todgpu_bilinear_stencils(ctypes.byref(a), pix.data_ptr(),
                                                         wgt.data_ptr(), stream_handle()))
    return pix, wgt


def beam_center_angles(ra, dec, center_idx=None):
    """(phi_c, theta_c) of the beam centre: the grid centre by default, as
    tod_rotations.py:251-261 chooses it."""
    ra = np.asarray(ra)
    dec = np.asarray(dec)
    if center_idx is None:
        center_idx = (ra.shape[0] // 2, ra.shape[1] // 2)
    return float(ra[center_idx]), float(np.pi / 2 - dec[center_idx])


def _angles_on_device(theta, phi, psi):
    adt = dtype_of(theta)
    adt = np.float32 if adt == np.dtype(np.float32) else np.float64
    th = to_device(theta, adt).reshape(-1)
    ph = to_device(phi, adt).reshape(-1)
    ps = to_device(psi, adt).reshape(-1)
    if ph.shape[0] != th.shape[0] or ps.shape[0] != th.shape[0]:
        raise ValueError("theta, phi and psi must have the same length")
    return adt, th, ph, ps


def pointing_buffers(B, device):
    """Uninitialised float64 (axes (B, 3), cos_a, sin_a, ax_pts (B, 3), cos_p,
    sin_p) for :func:`pointing_params`."""
    axes = torch.empty((B, 3), dtype=torch.float64, device=device)
    pts = torch.empty((B, 3), dtype=torch.float64, device=device)
    cos_a, sin_a, cos_p, sin_p = (torch.empty(B, dtype=torch.float64, device=device) for _ in range(4))
    return axes, cos_a, sin_a, pts, cos_p, sin_p


def pointing_params(theta, phi, psi, center_phi, center_theta, out=None):
    """Float64 rotation parameters (axes (B, 3), cos_a, sin_a, ax_pts (B, 3),
    cos_p, sin_p) of every sample, derived on the device from the pointing
    angles and the beam centre -- the reference's
    precompute_rotation_vector_batch + _rotation_params
    (tod_rotations.py:219-333) in float64, one thread per sample.  A float64
    gather on them equals the angles-mode gather bit for bit.  ``out``: six
    contiguous float64 CUDA tensors of at least B samples to fill (e.g. from
    :func:`pointing_buffers`); returned as given."""
    require_cuda()
    adt, th, ph, ps = _angles_on_device(theta, phi, psi)
    B = th.shape[0]
    if out is None:
        out = pointing_buffers(B, th.device)
    elif len(out) != 6 or any(not (is_tensor(t) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
                                   and t.shape[0] >= B) for t in out):
        raise ValueError("out must be six contiguous float64 CUDA tensors of at least B samples")
    axes, cos_a, sin_a, pts, cos_p, sin_p = out
    _native.check(_native.lib().todgpu_pointing_params(
        th.data_ptr(), ph.data_ptr(), ps.data_ptr(), _native.F32 if adt == np.float32 else _native.F64, B,
        float(center_phi), float(center_theta), axes.data_ptr(), cos_a.data_ptr(), sin_a.data_ptr(),
        pts.data_ptr(), cos_p.data_ptr(), sin_p.data_ptr(), stream_handle()))
    return out


def gather_accum_angles(interp, vec_orig, theta, phi, psi, center_phi, center_theta, nside,
                        mp_stacked, beam_vals, tod, c_q=-1, c_u=-1, err_count=None, flags=0,
                        static_table=False, precompute=True):
    """One fused launch with the pointing given as angles: every CTA derives
    the sample's rotation on the device in float64 from (theta, phi, psi) and
    the beam centre (no float32 parameter rounding).  ``tod`` must be a float64
    (C, B) CUDA tensor; it is accumulated in place.  ``theta, phi, psi`` may be
    float32 or float64 (a float32 scan is widened exactly on the device).

    ``precompute`` (default) derives the rotations first with
    :func:`pointing_params` (one thread per sample, 80 bytes of scratch per
    sample) and runs the gather in its float64-parameter mode: the same TOD bit
    for bit, with the per-sample rotation taken off the gather's critical path.
    ``precompute=False`` (and ``static_table=True``, which allocates nothing)
    derive the rotation inside the gather."""
    require_cuda()
    vec = to_device(vec_orig, np.float64).reshape(-1, 3)
    S = vec.shape[0]
    adt, th, ph, ps = _angles_on_device(theta, phi, psi)
    B = th.shape[0]
    rot = pointing_params(th, ph, ps, center_phi, center_theta) if precompute and not static_table else None
    beam = to_device(beam_vals, np.float32, (S,))
    mp = _map_tensor(mp_stacked)
    C = _ncomp(mp)
    if not (is_tensor(tod) and tod.is_cuda and tod.dtype == torch.float64 and tod.dim() == 2
            and tod.stride(1) == 1 and tuple(tod.shape) == (C, B)):
        raise ValueError(f"tod must be a float64 CUDA tensor of shape {(C, B)} with unit stride")
    a = _native.GatherArgs()
    a.abi_version = _native.ABI_VERSION
    a.interp = interp
    a.nside = int(nside)
    a.B = B
    a.S = S
    a.C = C
    a.c_q = int(c_q)
    a.c_u = int(c_u)
    _set_map(a, mp)
    a.vec_orig = vec.data_ptr()
    if rot is not None:
        a.params_dtype = _native.F64
        (a.axes, a.cos_a, a.sin_a, a.ax_pts, a.cos_p, a.sin_p) = [t.data_ptr() for t in rot]
    else:
        a.params_dtype = _native.ANGLES
        a.theta, a.phi, a.psi = th.data_ptr(), ph.data_ptr(), ps.data_ptr()
        a.angles_dtype = _native.F32 if adt == np.float32 else _native.F64
        a.center_phi = float(center_phi)
        a.center_theta = float(center_theta)
    a.beam_vals = beam.data_ptr()
    a.tod = tod.data_ptr()
    a.tod_stride = _row_stride(tod)
    a.err_count = ptr(err_count)
    a.flags = int(flags)
    lib = _native.lib()
    if static_table:
        _native.check(lib.todgpu_gather_accum_static(ctypes.byref(a), stream_handle()))
        return tod
    if not flags & _native.FLAG_NO_TABLES and B > 0 and S > 0:
        table = ring_table(nside, beam_reach(vec, nside), vec.device)
        a.ring_table = table.data_ptr()
        a.tab_slots = table_slots_for(table, nside)
    _native.check(lib.todgpu_gather_accum(ctypes.byref(a), stream_handle()))
    return tod
