"""Nearest-pixel-mode TOD kernel on the GPU (drop-in for the reference module
``tod_nearest``, tod_nearest.py).

:func:`gather_accum_nearest` / ``_gather_accum_nearest_jit`` replaces
``_gather_accum_nearest_jit`` (tod_nearest.py:21-158): rotate each beam pixel,
pick the nearest RING pixel by the reference's 4-candidate rule (two rings
bracketing z, two phi slots each, unnormalised z and sin theta, ties keep the
first), apply the spin-2 rotation at that pixel when the entry carries both Q
and U, and accumulate into ``tod`` in place.
"""

from __future__ import annotations

from . import _native
from .kernels import gather_accum

__all__ = ("gather_accum_nearest", "_gather_accum_nearest_jit")


def gather_accum_nearest(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, mp_stacked,
                         beam_vals, B, S, tod, c_q=-1, c_u=-1, bore_phi=None):
    """GPU replacement of ``_gather_accum_nearest_jit`` (tod_nearest.py:21-158)."""
    return gather_accum(_native.NEAREST, vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p,
                        nside, mp_stacked, beam_vals, B, S, tod, c_q, c_u, bore_phi=bore_phi)


_gather_accum_nearest_jit = gather_accum_nearest
