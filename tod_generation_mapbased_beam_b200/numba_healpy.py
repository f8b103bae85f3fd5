"""HEALPix RING helpers on the GPU (drop-in names of the reference module
``numba_healpy``).

* :func:`get_interp_weights_numba` -- hp.get_interp_weights in RING order
  (numba_healpy.py:239-253): pixels (4, N) int64 and weights (4, N) float64.
* :func:`pix2ang_numba` -- RING pixel centres (numba_healpy.py:622-635).
* :func:`ang2pix_ring` -- nearest pixel by the 4-candidate rule
  (numba_healpy.py:642-693), vectorised.

Inputs may be numpy arrays or torch tensors; numpy in -> numpy out, tensors
in -> CUDA tensors out.  All arithmetic runs in the sm_100a kernels of
libtodgpu.so.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native
from ._device import require_cuda, stream_handle, to_device


def _host(*xs):
    return not any(isinstance(x, torch.Tensor) for x in xs)


def _flat(x, dt):
    t = to_device(x if isinstance(x, torch.Tensor) else np.asarray(x, dt), dt)
    return t.reshape(-1)


def get_interp_weights_numba(nside, theta, phi):
    require_cuda()
    host = _host(theta, phi)
    th = _flat(theta, np.float64)
    ph = _flat(phi, np.float64)
    if th.shape != ph.shape:
        th, ph = torch.broadcast_tensors(th, ph)
        th, ph = th.contiguous(), ph.contiguous()
    n = th.shape[0]
    pix = torch.empty((4, n), dtype=torch.int64, device=th.device)
    wgt = torch.empty((4, n), dtype=torch.float64, device=th.device)
    _native.check(_native.lib().todgpu_get_interp_weights(int(nside), th.data_ptr(), ph.data_ptr(), n,
                                                          pix.data_ptr(), wgt.data_ptr(), stream_handle()))
    if host:
        return pix.cpu().numpy(), wgt.cpu().numpy()
    return pix, wgt


def pix2ang_numba(nside, pix, nest=False):
    if nest:
        raise ValueError("pix2ang_numba only supports nest=False (RING scheme)")
    require_cuda()
    host = _host(pix)
    p = _flat(pix, np.int64)
    n = p.shape[0]
    th = torch.empty(n, dtype=torch.float64, device=p.device)
    ph = torch.empty(n, dtype=torch.float64, device=p.device)
    _native.check(_native.lib().todgpu_pix2ang(int(nside), p.data_ptr(), n, th.data_ptr(), ph.data_ptr(),
                                               stream_handle()))
    if host:
        return th.cpu().numpy(), ph.cpu().numpy()
    return th, ph


def ang2pix_ring(nside, theta, phi):
    require_cuda()
    host = _host(theta, phi)
    th = _flat(theta, np.float64)
    ph = _flat(phi, np.float64)
    n = th.shape[0]
    out = torch.empty(n, dtype=torch.int64, device=th.device)
    _native.check(_native.lib().todgpu_ang2pix(int(nside), th.data_ptr(), ph.data_ptr(), n, out.data_ptr(),
                                               stream_handle()))
    if host:
        return out.cpu().numpy()
    return out


def nside2npix(nside):
    return 12 * int(nside) * int(nside)
