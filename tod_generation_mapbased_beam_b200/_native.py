"""ctypes binding of libtodgpu.so (the C ABI in include/todgpu.h).

The library is built in-tree by ``tod_generation_mapbased_beam_b200.build``.
There is no CPU fallback: if the library is missing or CUDA is unavailable,
every call raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libtodgpu.so")

ABI_VERSION = 1
OK = 0
EINVAL, ENSIDE, ESHAPE, EDTYPE, ECUDA, EABI = -1, -2, -3, -4, -5, -6
BILINEAR, NEAREST = 0, 1
F32, F64, ANGLES = 0, 1, 2
PACKED_F32, PACKED_BF16, PACKED_F64 = 2, 3, 4
FLAG_NO_TABLES = 1
FLAG_NO_BEAM_STAGE = 2
FLAG_WIDE_CTAS = 4

_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_p = ctypes.c_void_p


class GatherArgs(ctypes.Structure):
    """Mirror of ``todgpu_gather_args``."""

    _fields_ = [
        ("abi_version", _i32),
        ("interp", _i32),
        ("nside", _i64),
        ("B", _i64),
        ("S", _i64),
        ("C", _i64),
        ("c_q", _i32),
        ("c_u", _i32),
        ("params_dtype", _i32),
        ("map_dtype", _i32),
        ("vec_orig", _p),
        ("axes", _p),
        ("cos_a", _p),
        ("sin_a", _p),
        ("ax_pts", _p),
        ("cos_p", _p),
        ("sin_p", _p),
        ("bore_phi", _p),
        ("beam_vals", _p),
        ("map", _p),
        ("map_stride", _i64),
        ("tod", _p),
        ("tod_stride", _i64),
        ("err_count", _p),
        ("flags", _i32),
        ("tab_slots", _i32),
        ("ring_table", _p),
        ("theta", _p),
        ("phi", _p),
        ("psi", _p),
        ("angles_dtype", _i32),
        ("reserved2", _i32),
        ("center_phi", ctypes.c_double),
        ("center_theta", ctypes.c_double),
    ]


class MlpDesc(ctypes.Structure):
    """Mirror of ``todgpu_mlp`` (include/todgpu.h)."""

    _fields_ = [
        ("n_freq", _i32),
        ("width", _i32),
        ("depth", _i32),
        ("n_out", _i32),
        ("freq", _p),
        ("params", _p),
        ("params_bf16", _p),
        ("grad", _p),
        ("adam_m", _p),
        ("adam_v", _p),
    ]


MLP_TCGEN05, MLP_MMA_SYNC = 0, 1  # forward paths of todgpu_mlp_set_forward_path

# workspace regions of todgpu_mlp_workspace_offsets, in order
MLP_WS_REGIONS = ("x", "feat", "z", "a", "y", "dz", "part", "loss")


class TodGpuError(RuntimeError):
    """A libtodgpu call returned an error status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"libtodgpu error {code}: {message}")
        self.code = code


_lock = threading.Lock()
_lib = None


def _declare(lib):
    lib.todgpu_gather_accum.argtypes = [ctypes.POINTER(GatherArgs), _p]
    lib.todgpu_gather_accum.restype = ctypes.c_int
    lib.todgpu_gather_accum_batched.argtypes = [ctypes.POINTER(GatherArgs), _i32, _i64, _p]
    lib.todgpu_gather_accum_batched.restype = ctypes.c_int
    lib.todgpu_gather_accum_static.argtypes = [ctypes.POINTER(GatherArgs), _p]
    lib.todgpu_gather_accum_static.restype = ctypes.c_int
    lib.todgpu_gather_wait_timeouts.argtypes = []
    lib.todgpu_gather_wait_timeouts.restype = _i64
    lib.todgpu_bilinear_stencils.argtypes = [ctypes.POINTER(GatherArgs), _p, _p, _p]
    lib.todgpu_bilinear_stencils.restype = ctypes.c_int
    lib.todgpu_get_interp_weights.argtypes = [_i64, _p, _p, _i64, _p, _p, _p]
    lib.todgpu_get_interp_weights.restype = ctypes.c_int
    lib.todgpu_ang2pix.argtypes = [_i64, _p, _p, _i64, _p, _p]
    lib.todgpu_ang2pix.restype = ctypes.c_int
    lib.todgpu_pix2ang.argtypes = [_i64, _p, _i64, _p, _p, _p]
    lib.todgpu_pix2ang.restype = ctypes.c_int
    lib.todgpu_spin2.argtypes = [_p] * 6 + [_i64, _p, _p, _p]
    lib.todgpu_spin2.restype = ctypes.c_int
    lib.todgpu_boresight_phi_host.argtypes = [_p, _i64, _p, _i32]
    lib.todgpu_boresight_phi_host.restype = ctypes.c_int
    lib.todgpu_ring_table_bytes.argtypes = [_i64]
    lib.todgpu_ring_table_bytes.restype = ctypes.c_size_t
    lib.todgpu_ring_table_build.argtypes = [_i64, ctypes.c_double, _p, ctypes.c_size_t, _p]
    lib.todgpu_ring_table_build.restype = ctypes.c_int
    lib.todgpu_pack_map.argtypes = [_p, _i32, _i64, _i64, _i64, _i32, _p, _p]
    lib.todgpu_pack_map.restype = ctypes.c_int
    lib.todgpu_alm2map_workspace_bytes.argtypes = [_i64, _i32]
    lib.todgpu_alm2map_workspace_bytes.restype = ctypes.c_size_t
    lib.todgpu_alm2map.argtypes = [_i64, _i32, _p, _p, ctypes.c_size_t, _p, _i64, _i32, _p]
    lib.todgpu_alm2map.restype = ctypes.c_int
    lib.todgpu_fp64_probe.argtypes = [_i64, _i32, _p, ctypes.POINTER(ctypes.c_double), _p]
    lib.todgpu_fp64_probe.restype = ctypes.c_int
    lib.todgpu_pointing_params.argtypes = [_p, _p, _p, _i32, _i64, ctypes.c_double, ctypes.c_double] + [_p] * 6 + [_p]
    lib.todgpu_pointing_params.restype = ctypes.c_int
    lib.todgpu_l2_probe.argtypes = [_p, ctypes.c_size_t, _i32, _p, _i64, ctypes.POINTER(ctypes.c_double), _p]
    lib.todgpu_l2_probe.restype = ctypes.c_int
    mp = ctypes.POINTER(MlpDesc)
    lib.todgpu_mlp_param_count.argtypes = [mp]
    lib.todgpu_mlp_param_count.restype = _i64
    lib.todgpu_mlp_param_offsets.argtypes = [mp, _p, _p]
    lib.todgpu_mlp_param_offsets.restype = ctypes.c_int
    lib.todgpu_mlp_workspace_bytes.argtypes = [mp, _i64]
    lib.todgpu_mlp_workspace_bytes.restype = ctypes.c_size_t
    lib.todgpu_mlp_workspace_offsets.argtypes = [mp, _i64, _p]
    lib.todgpu_mlp_workspace_offsets.restype = ctypes.c_int
    lib.todgpu_mlp_sync_bf16.argtypes = [mp, _p]
    lib.todgpu_mlp_sync_bf16.restype = ctypes.c_int
    lib.todgpu_mlp_inputs.argtypes = [_p, _p, _p, _i32, _i64, _i64, _p, _p]
    lib.todgpu_mlp_inputs.restype = ctypes.c_int
    lib.todgpu_mlp_forward.argtypes = [mp, _p, _i64, _p, ctypes.c_size_t, _p, _p]
    lib.todgpu_mlp_forward.restype = ctypes.c_int
    lib.todgpu_mlp_loss_grad.argtypes = [mp, _p, _p, _i64, _p, ctypes.c_size_t, _p, _p]
    lib.todgpu_mlp_loss_grad.restype = ctypes.c_int
    lib.todgpu_mlp_adam.argtypes = [mp, _i64, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _p]
    lib.todgpu_mlp_adam.restype = ctypes.c_int
    lib.todgpu_mlp_train.argtypes = [mp, _p, _p, _i64, _i64, _i64, _i64, _i64, ctypes.c_float, ctypes.c_float,
                                     _p, ctypes.c_size_t, _p, _p]
    lib.todgpu_mlp_train.restype = ctypes.c_int
    lib.todgpu_tail_accumulate.argtypes = [mp, _p, _p, _p, _i32, _i64, _p, _p, _p, _p, _i64, _i64, _p,
                                           ctypes.c_size_t, _p]
    lib.todgpu_tail_accumulate.restype = ctypes.c_int
    lib.todgpu_mlp_set_forward_path.argtypes = [_i32]
    lib.todgpu_mlp_set_forward_path.restype = ctypes.c_int
    lib.todgpu_mlp_wait_timeouts.argtypes = []
    lib.todgpu_mlp_wait_timeouts.restype = _i64
    lib.todgpu_mlp_tcgen05_launches.argtypes = []
    lib.todgpu_mlp_tcgen05_launches.restype = _i64
    lib.todgpu_kmeans_workspace_bytes.argtypes = [_i64, _i32]
    lib.todgpu_kmeans_workspace_bytes.restype = ctypes.c_size_t
    lib.todgpu_kmeans_seed.argtypes = [_p, _p, _i64, _i32, _p, _p, _p, _p, ctypes.c_size_t, _p]
    lib.todgpu_kmeans_seed.restype = ctypes.c_int
    lib.todgpu_kmeans_assign.argtypes = [_p, _i64, _p, _i32, _p, _p, _p]
    lib.todgpu_kmeans_assign.restype = ctypes.c_int
    lib.todgpu_kmeans_sums.argtypes = [_p, _p, _p, _i64, _i32, _p, _p, ctypes.c_size_t, _p]
    lib.todgpu_kmeans_sums.restype = ctypes.c_int
    lib.todgpu_kmeans_argmin.argtypes = [_p, _i64, _p, _p]
    lib.todgpu_kmeans_argmin.restype = ctypes.c_int
    lib.todgpu_abi_version.argtypes = []
    lib.todgpu_abi_version.restype = ctypes.c_int
    lib.todgpu_last_error_string.argtypes = []
    lib.todgpu_last_error_string.restype = ctypes.c_char_p


def lib():
    """Load libtodgpu.so once (building it first if it is absent and nvcc is
    available); raise if that is impossible."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build as _build

            _build.build()
        handle = ctypes.CDLL(os.environ.get("TODGPU_LIBRARY", LIB_PATH))
        _declare(handle)
        if handle.todgpu_abi_version() != ABI_VERSION:
            raise TodGpuError(EABI, "libtodgpu ABI version mismatch; rebuild the library")
        _lib = handle
    return _lib


def check(rc: int):
    if rc != OK:
        msg = lib().todgpu_last_error_string()
        raise TodGpuError(rc, msg.decode() if msg else "")


def exported_symbols():
    """Names of the C entry points declared in include/todgpu.h."""
    return [
        "todgpu_gather_accum",
        "todgpu_gather_accum_batched",
        "todgpu_gather_accum_static",
        "todgpu_gather_wait_timeouts",
        "todgpu_bilinear_stencils",
        "todgpu_get_interp_weights",
        "todgpu_ang2pix",
        "todgpu_pix2ang",
        "todgpu_spin2",
        "todgpu_boresight_phi_host",
        "todgpu_ring_table_bytes",
        "todgpu_ring_table_build",
        "todgpu_pack_map",
        "todgpu_alm2map_workspace_bytes",
        "todgpu_alm2map",
        "todgpu_fp64_probe",
        "todgpu_l2_probe",
        "todgpu_pointing_params",
        "todgpu_mlp_set_forward_path",
        "todgpu_mlp_wait_timeouts",
        "todgpu_mlp_tcgen05_launches",
        "todgpu_mlp_param_count",
        "todgpu_mlp_param_offsets",
        "todgpu_mlp_workspace_bytes",
        "todgpu_mlp_workspace_offsets",
        "todgpu_mlp_sync_bf16",
        "todgpu_mlp_inputs",
        "todgpu_mlp_forward",
        "todgpu_mlp_loss_grad",
        "todgpu_mlp_adam",
        "todgpu_mlp_train",
        "todgpu_tail_accumulate",
        "todgpu_kmeans_workspace_bytes",
        "todgpu_kmeans_seed",
        "todgpu_kmeans_assign",
        "todgpu_kmeans_sums",
        "todgpu_kmeans_argmin",
        "todgpu_abi_version",
        "todgpu_last_error_string",
    ]
