"""Seeded synthetic skies by spherical-harmonic synthesis on the GPU.

The reference's benchmark skies come from ``healpy.synfast`` with
C_l^TT proportional to (l + 10)^-2 scaled to 100 uK RMS in I, and EE / BB at
10% / 1% of TT; healpy is not available here, so this module draws the
harmonic coefficients itself (numpy, seeded) and synthesises the map with the
library's ``todgpu_alm2map``.  Q and U are drawn as independent scalar fields
with spectrum (EE + BB) / 2 (the spin-2 E/B synthesis is not reproduced; this
changes the statistics of Q/U, not their amplitude or smoothness).  The
monopole and dipole are left out.  Realisations do not match healpy's random
stream.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native
from ._device import require_cuda, stream_handle


def cl_tt(lmax, rms_k=100e-6):
    """(l + 10)^-2 for l >= 2 (0 below), scaled so the map RMS is ``rms_k``."""
    ell = np.arange(lmax + 1, dtype=np.float64)
    cl = (ell + 10.0) ** -2
    cl[:2] = 0.0
    var = np.sum((2 * ell + 1) / (4 * np.pi) * cl)
    return cl * (rms_k ** 2 / var)


def random_alm(cl, seed_or_rng):
    """Complex a_lm (m-major, as todgpu_alm2map expects) of a Gaussian field."""
    rng = np.random.default_rng(seed_or_rng) if not isinstance(seed_or_rng, np.random.Generator) else seed_or_rng
    lmax = len(cl) - 1
    n = (lmax + 1) * (lmax + 2) // 2
    out = np.empty((n, 2))
    for m in range(lmax + 1):
        i0 = m * (2 * lmax + 1 - m) // 2
        ls = np.arange(m, lmax + 1)
        sd = np.sqrt(cl[ls] * (1.0 if m == 0 else 0.5))
        out[i0 + ls, 0] = rng.standard_normal(len(ls)) * sd
        out[i0 + ls, 1] = 0.0 if m == 0 else rng.standard_normal(len(ls)) * sd
    return out


def alm2map(alm, nside, lmax, out=None, comp=0):
    """Synthesise one component into ``out[comp]`` (a (C, 12 nside^2) float64
    CUDA tensor, allocated when None); returns ``out``."""
    require_cuda()
    dev = torch.device("cuda", torch.cuda.current_device())
    npix = 12 * int(nside) ** 2
    if out is None:
        out = torch.empty((comp + 1, npix), dtype=torch.float64, device=dev)
    a = torch.from_numpy(np.ascontiguousarray(alm, dtype=np.float64)).to(dev)
    lib = _native.lib()
    ws_bytes = int(lib.todgpu_alm2map_workspace_bytes(int(nside), int(lmax)))
    ws = torch.empty(ws_bytes // 8 + 1, dtype=torch.float64, device=dev)
    _native.check(lib.todgpu_alm2map(int(nside), int(lmax), a.data_ptr(), ws.data_ptr(), ws_bytes,
                                     out.data_ptr(), out.stride(0), int(comp), stream_handle()))
    return out


def synfast_iqu(nside, seed, lmax=None, rms_k=100e-6, ee_frac=0.1, bb_frac=0.01, dtype=torch.float64):
    """(3, 12 nside^2) I/Q/U sky on the GPU: C_l^TT ~ (l+10)^-2 at ``rms_k``
    RMS, Q and U with (EE + BB) / 2 = (ee_frac + bb_frac) / 2 C_l^TT."""
    lmax = 3 * int(nside) - 1 if lmax is None else int(lmax)
    rng = np.random.default_rng(seed)
    tt = cl_tt(lmax, rms_k)
    dev = torch.device("cuda", torch.cuda.current_device())
    out = torch.empty((3, 12 * int(nside) ** 2), dtype=torch.float64, device=dev)
    alm2map(random_alm(tt, rng), nside, lmax, out, 0)
    qu = tt * 0.5 * (ee_frac + bb_frac)
    alm2map(random_alm(qu, rng), nside, lmax, out, 1)
    alm2map(random_alm(qu, rng), nside, lmax, out, 2)
    return out.to(dtype)
