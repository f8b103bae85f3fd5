"""B200-native beam-convolution TOD generation.

GPU drop-in for the per-sample beam-convolution path of
ArtemBasyrov/tod_generation_mapbased_beam:

    tod[c, t] = sum_s b_s * interp(map_c, R(theta_t, phi_t, psi_t) v_s)
                (+ spin-2 rotation of Q/U)

Entry points mirror the reference modules (tod_core, tod_bilinear,
tod_nearest, tod_rotations, numba_healpy); the arithmetic runs in the sm_100a
kernels of ``_lib/libtodgpu.so`` behind the C ABI in ``include/todgpu.h``.
"""

from .tod_core import beam_tod_batch  # noqa: F401
from .tod_rotations import _rotation_params, precompute_rotation_vector_batch  # noqa: F401

__all__ = ["beam_tod_batch", "precompute_rotation_vector_batch", "_rotation_params"]
