"""Per-sample pointing -> rotation parameters (drop-in for the reference
module ``tod_rotations``, tod_rotations.py).

The reference prepares pointing on the host with numpy and hands float32
parameters to its kernels; to be a bit-level drop-in the same host-side
preparation is kept here, with the same numpy primitives in the same order so
the float32 parameters come out identical:

* :func:`precompute_rotation_vector_batch` (tod_rotations.py:219-303):
  Rodrigues vector (axis * angle) taking the beam centre to each boresight,
  and the polarisation offset beta in [0, 2pi).
* :func:`_rotation_params` (tod_rotations.py:306-333): the six float32
  per-sample arrays the fused kernels consume.

Both are O(B) host work (~1% of the reference's batch time); the O(B*S) work
is on the GPU.
"""

from __future__ import annotations

import numpy as np

__all__ = ("precompute_rotation_vector_batch", "_rotation_params", "rotation_params")


def _components(phi, theta):
    st, ct = np.sin(theta), np.cos(theta)
    sp, cp = np.sin(phi), np.cos(phi)
    return st, ct, sp, cp


def _dot3(a0, a1, a2, b0, b1, b2):
    return a0 * b0 + a1 * b1 + a2 * b2


def precompute_rotation_vector_batch(ra, dec, phi_batch, theta_batch, center_idx=None):
    """Rodrigues vectors ``(B, 3)`` and beta ``(B,)`` for boresights
    ``(phi_batch, theta_batch)`` relative to the beam centre
    ``(ra, dec)[center_idx]`` (default: the grid centre)."""
    ra = np.asarray(ra)
    dec = np.asarray(dec)
    if center_idx is None:
        center_idx = (ra.shape[0] // 2, ra.shape[1] // 2)
    phi_c = ra[center_idx]
    theta_c = np.pi / 2 - dec[center_idx]
    phi = np.asarray(phi_batch)
    theta = np.asarray(theta_batch)

    st0, ct0, sp0, cp0 = _components(phi_c, theta_c)
    c0, c1, c2 = st0 * cp0, st0 * sp0, ct0                    # beam-centre unit vector
    n0, n1, n2 = cp0 * ct0, sp0 * ct0, -st0                    # its local north
    st, ct, sp, cp = _components(phi, theta)
    t0, t1, t2 = st * cp, st * sp, ct                          # boresight unit vectors
    nt0, nt1, nt2 = cp * ct, sp * ct, -st                      # boresight north
    et0, et1 = -sp, cp                                         # boresight east (z = 0)

    # axis = centre x boresight, normalised (zero when parallel)
    k0 = c1 * t2 - c2 * t1
    k1 = c2 * t0 - c0 * t2
    k2 = c0 * t1 - c1 * t0
    knorm = np.sqrt((k0 * k0 + k1 * k1) + k2 * k2)
    ok = knorm > 1e-10
    with np.errstate(invalid="ignore", divide="ignore"):
        k0 = np.where(ok, k0 / knorm, 0)
        k1 = np.where(ok, k1 / knorm, 0)
        k2 = np.where(ok, k2 / knorm, 0)
    angle = np.arccos(np.clip(_dot3(c0, c1, c2, t0, t1, t2), -1, 1))
    rot = np.stack([k0 * angle, k1 * angle, k2 * angle], axis=-1)

    # beam-centre north carried along by the recentring rotation
    ca = np.cos(angle)
    sa = np.sin(angle)
    dkn = _dot3(k0, k1, k2, n0, n1, n2)
    oma = 1 - ca
    w0 = n0 * ca + (k1 * n2 - k2 * n1) * sa + k0 * dkn * oma
    w1 = n1 * ca + (k2 * n0 - k0 * n2) * sa + k1 * dkn * oma
    w2 = n2 * ca + (k0 * n1 - k1 * n0) * sa + k2 * dkn * oma
    beta = np.arctan2(w0 * et0 + w1 * et1 + w2 * 0.0, _dot3(w0, w1, w2, nt0, nt1, nt2))
    beta = np.where(beta < 0, beta + 2 * np.pi, beta)
    return rot, beta


def _rotation_params(rot_vecs, phi_b, theta_b, psis_b):
    """``axes (B,3), cos_a, sin_a, ax_pts (B,3), cos_p, sin_p`` -- all float32."""
    rot_vecs = np.asarray(rot_vecs)
    r0, r1, r2 = rot_vecs[:, 0], rot_vecs[:, 1], rot_vecs[:, 2]
    angles = np.sqrt((r0 * r0 + r1 * r1) + r2 * r2).astype(np.float32)
    safe = angles > np.float32(1e-10)
    denom = np.where(safe, angles, np.float32(1.0))[:, None]
    axes = (rot_vecs / denom).astype(np.float32)
    axes = np.where(safe[:, None], axes, np.float32(0.0))
    cos_a = np.cos(angles)
    sin_a = np.sin(angles)
    phi_f = np.asarray(phi_b, dtype=np.float32)
    theta_f = np.asarray(theta_b, dtype=np.float32)
    psis_f = np.asarray(psis_b, dtype=np.float32)
    st = np.sin(theta_f)
    ax_pts = np.stack([st * np.cos(phi_f), st * np.sin(phi_f), np.cos(theta_f)], axis=-1)
    return axes, cos_a, sin_a, ax_pts, np.cos(psis_f), np.sin(psis_f)


rotation_params = _rotation_params
