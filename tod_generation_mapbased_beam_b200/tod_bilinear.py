"""Bilinear-mode TOD kernels on the GPU (drop-in for the reference module
``tod_bilinear``, tod_bilinear.py).

* :func:`gather_accum_fused` / ``_gather_accum_fused_jit`` -- the fused
  rotate -> 4-neighbour RING stencil -> spin-2 -> gather -> accumulate kernel
  (tod_bilinear.py:205-477), same arguments, ``tod`` accumulated in place.
* :func:`spin2_cos2d_sin2d` / ``_spin2_cos2d_sin2d_jit`` -- the spin-2 frame
  rotation (tod_bilinear.py:84-145), vectorised on the device.
* :func:`get_interp_weights_numba` -- re-exported, as the reference module does.

The reference's per-sample spin-2 cache (tod_bilinear.py:151-199) is an
optimisation that returns the same values as direct evaluation; the GPU
kernel evaluates the spin-2 angle per stencil neighbour instead.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native
from ._device import require_cuda, stream_handle, to_device
from .kernels import gather_accum
from .numba_healpy import get_interp_weights_numba  # noqa: F401  (re-export)

__all__ = ("gather_accum_fused", "_gather_accum_fused_jit", "spin2_cos2d_sin2d",
           "_spin2_cos2d_sin2d_jit", "get_interp_weights_numba")


def gather_accum_fused(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, mp_stacked,
                       beam_vals, B, S, tod, c_q=-1, c_u=-1, bore_phi=None):
    """GPU replacement of ``_gather_accum_fused_jit`` (tod_bilinear.py:205-477)."""
    return gather_accum(_native.BILINEAR, vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p,
                        nside, mp_stacked, beam_vals, B, S, tod, c_q, c_u, bore_phi=bore_phi)


_gather_accum_fused_jit = gather_accum_fused


def spin2_cos2d_sin2d(z_pix, sth_pix, phi_pix, z_pts, sth_pts, phi_pts):
    """cos 2d, sin 2d (tod_bilinear.py:84-145) for arrays (or scalars) on the
    GPU; returns float64 CUDA tensors (numpy arrays for numpy/scalar input)."""
    require_cuda()
    host = not any(isinstance(x, torch.Tensor) for x in (z_pix, sth_pix, phi_pix, z_pts, sth_pts, phi_pts))
    arrs = [np.atleast_1d(np.asarray(x.cpu() if isinstance(x, torch.Tensor) else x, np.float64))
            for x in (z_pix, sth_pix, phi_pix, z_pts, sth_pts, phi_pts)]
    n = max(a.shape[0] for a in arrs)
    ts = [to_device(np.broadcast_to(a, (n,)), np.float64) for a in arrs]
    c2 = torch.empty(n, dtype=torch.float64, device=ts[0].device)
    s2 = torch.empty_like(c2)
    _native.check(_native.lib().todgpu_spin2(*[t.data_ptr() for t in ts], n, c2.data_ptr(),
                                             s2.data_ptr(), stream_handle()))
    if host:
        return c2.cpu().numpy(), s2.cpu().numpy()
    return c2, s2


_spin2_cos2d_sin2d_jit = spin2_cos2d_sin2d
