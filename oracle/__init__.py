"""CPU oracle for the beam-convolution TOD path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product package never does.

``tod_oracle.c`` restates the reference's Numba kernels operation by operation
(see the file header for the file:line map); this module loads the compiled
library and exposes numpy-level wrappers with the reference's kernel ABI:

* :func:`gather_accum_fused`   -- ``tod_bilinear._gather_accum_fused_jit``
* :func:`gather_accum_nearest` -- ``tod_nearest._gather_accum_nearest_jit``
* :func:`bilinear_stencils`    -- per-(b, s) pixels/weights of the fused path
* :func:`get_interp_weights`, :func:`pix2ang`, :func:`ang2pix`, :func:`spin2`

The ``*_f64`` variants take unrounded float64 rotation parameters: together
with :func:`rotation_params_f64` they form the FP64 "ideal" oracle used for
the µK error budget of the reduced-precision forms.

Pinning: ``tests/test_oracle_golden.py`` checks every wrapper against golden
vectors produced by the reference's own Numba kernels (``tests/golden/``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtodoracle.so")
_lib = None

_i64 = ctypes.c_int64
_int = ctypes.c_int
_p = ctypes.c_void_p


def build(force: bool = False) -> str:
    """Compile ``tod_oracle.c`` with the committed Makefile; return the .so path."""
    src = os.path.join(_HERE, "tod_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = ctypes.CDLL(_LIB_PATH)
    kern_args = [_p] * 7 + [_int, _i64, _p, _int, _i64, _i64, _p, _i64, _i64, _p, _i64, _i64, _int]
    for name in ("oracle_gather_accum_bilinear", "oracle_gather_accum_nearest"):
        fn = getattr(lib, name)
        fn.argtypes = kern_args
        fn.restype = _i64
    lib.oracle_bilinear_stencils.argtypes = [_p] * 7 + [_int, _i64, _i64, _i64, _p, _p, _int]
    lib.oracle_atan2f.argtypes = [_p, _p, _i64, _p]
    lib.oracle_atan2f.restype = None
    lib.oracle_bilinear_stencils.restype = None
    lib.oracle_get_interp_weights.argtypes = [_i64, _p, _p, _i64, _p, _p]
    lib.oracle_get_interp_weights.restype = None
    lib.oracle_pix2ang.argtypes = [_i64, _p, _i64, _p, _p]
    lib.oracle_pix2ang.restype = None
    lib.oracle_ang2pix.argtypes = [_i64, _p, _p, _i64, _p]
    lib.oracle_ang2pix.restype = None
    lib.oracle_spin2.argtypes = [_p] * 6 + [_i64, _p, _p]
    lib.oracle_spin2.restype = None
    lib.oracle_max_threads.argtypes = []
    lib.oracle_max_threads.restype = _int
    _lib = lib
    return lib


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def _f64(a, shape=None):
    out = np.ascontiguousarray(np.asarray(a), dtype=np.float64)
    if shape is not None:
        out = out.reshape(shape)
    return out


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _params(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, B, S, f64):
    dt = np.float64 if f64 else np.float32
    shapes = [(S, 3), (B, 3), (B,), (B,), (B, 3), (B,), (B,)]
    out = []
    for a, sh in zip((vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p), shapes):
        a = np.asarray(a)
        if not f64 and a.dtype != np.float32:
            raise TypeError("reference-typed parameters must be float32 arrays")
        out.append(np.ascontiguousarray(a, dtype=dt).reshape(sh))
    return out


def _kernel(name, vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, mp_stacked,
            beam_vals, B, S, tod, c_q, c_u, nthreads, f64):
    lib = _load()
    B = int(B)
    S = int(S)
    prm = _params(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, B, S, f64)
    bv = _f64(beam_vals, (S,))
    mp = np.asarray(mp_stacked)
    if mp.ndim != 2:
        raise ValueError("mp_stacked must be (C, N)")
    if mp.dtype not in (np.float32, np.float64):
        mp = mp.astype(np.float64)
    mp = np.ascontiguousarray(mp)
    if tod.dtype != np.float64 or not tod.flags.c_contiguous or tod.shape != (mp.shape[0], B):
        raise ValueError("tod must be a C-contiguous float64 (C, B) array")
    errs = getattr(lib, name)(
        *[_ptr(a) for a in prm], int(bool(f64)), int(nside), _ptr(mp),
        int(mp.dtype == np.float64), int(mp.shape[0]), int(mp.shape[1]), _ptr(bv), B, S,
        _ptr(tod), int(c_q), int(c_u), int(nthreads))
    return int(errs)


def gather_accum_fused(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, mp_stacked,
                       beam_vals, B, S, tod, c_q=-1, c_u=-1, nthreads=0, f64=False):
    """Oracle of ``_gather_accum_fused_jit`` (tod_bilinear.py:205-477).

    With ``f64=False`` the parameters must be float32 and are used with the
    reference's operand typing; with ``f64=True`` they are float64 and every
    step is float64 (the ideal oracle).  Accumulates into ``tod`` in place;
    returns the count of skipped out-of-range map reads (0 for finite pointing)."""
    return _kernel("oracle_gather_accum_bilinear", vec_orig, axes, cos_a, sin_a, ax_pts, cos_p,
                   sin_p, nside, mp_stacked, beam_vals, B, S, tod, c_q, c_u, nthreads, f64)


def gather_accum_nearest(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, mp_stacked,
                         beam_vals, B, S, tod, c_q=-1, c_u=-1, nthreads=0, f64=False):
    """Oracle of ``_gather_accum_nearest_jit`` (tod_nearest.py:21-158)."""
    return _kernel("oracle_gather_accum_nearest", vec_orig, axes, cos_a, sin_a, ax_pts, cos_p,
                   sin_p, nside, mp_stacked, beam_vals, B, S, tod, c_q, c_u, nthreads, f64)


def atan2f(y, x):
    """The host C library's float32 atan2 (what the reference's float32
    ``math.atan2`` calls)."""
    lib = _load()
    y = np.ascontiguousarray(y, dtype=np.float32).ravel()
    x = np.ascontiguousarray(x, dtype=np.float32).ravel()
    out = np.empty(y.shape[0], np.float32)
    lib.oracle_atan2f(_ptr(y), _ptr(x), y.shape[0], _ptr(out))
    return out


def bilinear_stencils(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, B, S,
                      nthreads=0, f64=False):
    """Per-(b, s) pixels (4, B*S) int64 and weights (4, B*S) float64 of the fused
    bilinear path (rotation -> clamp/atan2 -> numba_healpy.py:358-499)."""
    lib = _load()
    B = int(B)
    S = int(S)
    pix = np.empty((4, B * S), dtype=np.int64)
    wgt = np.empty((4, B * S), dtype=np.float64)
    prm = _params(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, B, S, f64)
    lib.oracle_bilinear_stencils(*[_ptr(a) for a in prm], int(bool(f64)), int(nside), B, S,
                                 _ptr(pix), _ptr(wgt), int(nthreads))
    return pix, wgt


def get_interp_weights(nside, theta, phi):
    """Oracle of ``get_interp_weights_numba`` (numba_healpy.py:120-253)."""
    lib = _load()
    th = _f64(theta).ravel()
    ph = _f64(phi).ravel()
    n = th.shape[0]
    pix = np.empty((4, n), dtype=np.int64)
    wgt = np.empty((4, n), dtype=np.float64)
    lib.oracle_get_interp_weights(int(nside), _ptr(th), _ptr(ph), n, _ptr(pix), _ptr(wgt))
    return pix, wgt


def pix2ang(nside, pix):
    """Oracle of ``pix2ang_numba`` (numba_healpy.py:505-635)."""
    lib = _load()
    p = np.ascontiguousarray(np.asarray(pix, dtype=np.int64).ravel())
    th = np.empty(p.shape[0])
    ph = np.empty(p.shape[0])
    lib.oracle_pix2ang(int(nside), _ptr(p), p.shape[0], _ptr(th), _ptr(ph))
    return th, ph


def ang2pix(nside, theta, phi):
    """Oracle of ``_ang2pix_ring_jit`` (numba_healpy.py:642-693), vectorised."""
    lib = _load()
    th = _f64(theta).ravel()
    ph = _f64(phi).ravel()
    out = np.empty(th.shape[0], dtype=np.int64)
    lib.oracle_ang2pix(int(nside), _ptr(th), _ptr(ph), th.shape[0], _ptr(out))
    return out


def spin2(z_pix, sth_pix, phi_pix, z_pts, sth_pts, phi_pts):
    """Oracle of ``_spin2_cos2d_sin2d_jit`` (tod_bilinear.py:84-145), vectorised."""
    lib = _load()
    arrs = [_f64(a).ravel() for a in (z_pix, sth_pix, phi_pix, z_pts, sth_pts, phi_pts)]
    n = arrs[0].shape[0]
    arrs = [np.broadcast_to(a, (n,)).copy() if a.shape[0] != n else a for a in arrs]
    c2 = np.empty(n)
    s2 = np.empty(n)
    lib.oracle_spin2(*[_ptr(a) for a in arrs], n, _ptr(c2), _ptr(s2))
    return c2, s2


# ---------------------------------------------------------------------------
# FP64 "ideal" pointing: the reference's host prep without float32 rounding.
# tod_rotations.py:219-303 (rotation vectors, beta) and :306-333 (params).
# ---------------------------------------------------------------------------


def rotation_vectors_f64(center_phi, center_theta, phi, theta):
    """Rodrigues vectors and beta (tod_rotations.py:219-303) in float64 for a
    beam centre (center_phi, center_theta) and boresights (phi, theta)."""
    phi = np.asarray(phi, dtype=np.float64)
    theta = np.asarray(theta, dtype=np.float64)
    st0, ct0 = np.sin(center_theta), np.cos(center_theta)
    sp0, cp0 = np.sin(center_phi), np.cos(center_phi)
    vc = np.array([st0 * cp0, st0 * sp0, ct0])
    nc = np.array([cp0 * ct0, sp0 * ct0, -st0])
    st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
    vt = np.stack([st * cp, st * sp, ct], axis=-1)
    nt = np.stack([cp * ct, sp * ct, -st], axis=-1)
    et = np.stack([-sp, cp, np.zeros_like(phi)], axis=-1)
    axis = np.cross(vc[None, :], vt)
    an = np.linalg.norm(axis, axis=-1, keepdims=True)
    axis = np.where(an > 1e-10, axis / np.where(an > 0, an, 1.0), 0.0)
    angle = np.arccos(np.clip(np.sum(vc[None, :] * vt, axis=-1), -1, 1))
    ca = np.cos(angle)
    dkv = np.sum(axis * nc[None, :], axis=-1, keepdims=True)
    w = (nc[None, :] * ca[:, None] + np.cross(axis, nc[None, :]) * np.sin(angle)[:, None]
         + axis * dkv * (1 - ca)[:, None])
    beta = np.arctan2(np.sum(w * et, axis=-1), np.sum(w * nt, axis=-1))
    beta = np.where(beta < 0, beta + 2 * np.pi, beta)
    return axis * angle[:, None], beta


def rotation_params_f64(rot_vecs, phi, theta, psis):
    """The six per-sample parameter arrays of tod_rotations.py:306-333 kept in
    float64 (no float32 rounding anywhere)."""
    rot_vecs = np.asarray(rot_vecs, dtype=np.float64)
    ang = np.linalg.norm(rot_vecs, axis=-1)
    safe = ang > 1e-10
    axes = np.where(safe[:, None], rot_vecs / np.where(safe, ang, 1.0)[:, None], 0.0)
    phi = np.asarray(phi, dtype=np.float64)
    theta = np.asarray(theta, dtype=np.float64)
    psis = np.asarray(psis, dtype=np.float64)
    st, ct = np.sin(theta), np.cos(theta)
    pts = np.stack([st * np.cos(phi), st * np.sin(phi), ct], axis=-1)
    return axes, np.cos(ang), np.sin(ang), pts, np.cos(psis), np.sin(psis)
