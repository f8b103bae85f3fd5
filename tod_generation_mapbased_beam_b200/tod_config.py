"""config.yaml reader: drop-in for the reference module ``tod_config``
(tod_config.py:1-63).

The reference reads ``config_local.yaml`` (else ``config.yaml``) next to its
sources at import time and exposes every setting as a module constant.  This
module reads the same keys with the same defaults and checks and exposes them
the same way -- ``from tod_generation_mapbased_beam_b200 import tod_config as
cfg; cfg.FOLDER_SCAN`` -- loading lazily on first attribute access from
``$TODGPU_CONFIG``, else ``config_local.yaml`` / ``config.yaml`` in the current
directory.  :func:`load_config` reads an explicit file into a :class:`TodConfig`.

GPU-only settings live in an optional ``gpu:`` block that the reference
ignores::

    gpu:
      device: 0              # CUDA device index
      pointing: device       # device (FP64 rotation on the GPU) | reference (host float32 prep)
      map_precision: f64     # f64 | f32 | bf16 (packed records, Kahan sums)
      chunk: 1048576         # samples per streamed chunk
      tables: true           # per-sample spin-2 tables (false: direct evaluation)
      learned_tail:          # optional: far-sidelobe tail by the network
        enabled: false
        budget_uK: 0.1       # held-out RMS error above which the plain tail is used
        n_train: 262144      # training pointings (plain-method targets)
        steps: 4000
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field

import yaml

__all__ = ["TodConfig", "GpuConfig", "load_config", "default_config_path"]

_VALID_INTERP = {"nearest", "bilinear"}

# reference key -> attribute name (tod_config.py:16-28)
_REQUIRED = {
    "FOLDER_BEAM": "FOLDER_BEAM",
    "FOLDER_SCAN": "FOLDER_SCAN",
    "FOLDER_TOD_OUTPUT": "FOLDER_TOD_OUTPUT",
    "path_to_map": "path_to_map",
    "beam_file_I": "beam_file_I",
    "beam_file_Q": "beam_file_Q",
    "beam_file_U": "beam_file_U",
    "power_fraction_threshold_I": "power_threshold_I",
    "power_fraction_threshold_Q": "power_threshold_Q",
    "power_fraction_threshold_U": "power_threshold_U",
    "start_day": "start_day",
    "end_day": "end_day",
    "n_processes": "n_processes",
}
# optional keys and their defaults (tod_config.py:32-63)
_OPTIONAL = {
    "calibration_enabled": True,
    "calibration_n_processes": None,
    "calibration_numba_threads": None,
    "calibration_batch_size": None,
    "beam_interp_method": "bilinear",
    "n_beam_clusters": None,
    "beam_cluster_tail_fraction": None,
    "clustering_calibration_enabled": False,
    "clustering_error_threshold": 1e-3,
    "mp_start_method": "spawn",
}


@dataclass
class LearnedTailConfig:
    enabled: bool = False
    budget_uK: float = 0.1
    n_train: int = 1 << 18
    steps: int = 4000


@dataclass
class GpuConfig:
    device: int = 0
    pointing: str = "device"
    map_precision: str = "f64"
    chunk: int = 1 << 20
    tables: bool = True
    learned_tail: LearnedTailConfig = field(default_factory=LearnedTailConfig)

    @classmethod
    def from_dict(cls, d):
        d = dict(d or {})
        lt = LearnedTailConfig(**(d.pop("learned_tail", None) or {}))
        unknown = set(d) - {"device", "pointing", "map_precision", "chunk", "tables"}
        if unknown:
            raise ValueError(f"unknown gpu settings: {sorted(unknown)}")
        g = cls(learned_tail=lt, **d)
        if g.pointing not in ("device", "reference"):
            raise ValueError(f"gpu.pointing must be 'device' or 'reference', got {g.pointing!r}")
        if g.map_precision not in ("f64", "f32", "bf16"):
            raise ValueError(f"gpu.map_precision must be f64, f32 or bf16, got {g.map_precision!r}")
        if int(g.chunk) < 1 or int(g.device) < 0:
            raise ValueError("gpu.chunk must be >= 1 and gpu.device >= 0")
        if g.learned_tail.budget_uK <= 0 or g.learned_tail.n_train < 1 or g.learned_tail.steps < 1:
            raise ValueError("gpu.learned_tail: budget_uK, n_train and steps must be positive")
        return g


@dataclass
class TodConfig:
    FOLDER_BEAM: str
    FOLDER_SCAN: str
    FOLDER_TOD_OUTPUT: str
    path_to_map: str
    beam_file_I: str
    beam_file_Q: str
    beam_file_U: str
    power_threshold_I: float
    power_threshold_Q: float
    power_threshold_U: float
    start_day: int
    end_day: int
    n_processes: int
    calibration_enabled: bool = True
    calibration_n_processes: int | None = None
    calibration_numba_threads: int | None = None
    calibration_batch_size: int | None = None
    beam_interp_method: str = "bilinear"
    n_beam_clusters: int | None = None
    beam_cluster_tail_fraction: float | None = None
    clustering_calibration_enabled: bool = False
    clustering_error_threshold: float = 1e-3
    mp_start_method: str = "spawn"
    gpu: GpuConfig = field(default_factory=GpuConfig)
    CONFIG_FILE: str = ""

    def driver_kwargs(self):
        """Keyword arguments of driver.tod_exact_gen_batched / process_day."""
        return dict(interp_mode=self.beam_interp_method, pointing=self.gpu.pointing)


def default_config_path():
    env = os.environ.get("TODGPU_CONFIG")
    if env:
        return env
    local = os.path.abspath("config_local.yaml")
    return local if os.path.exists(local) else os.path.abspath("config.yaml")


def load_config(path=None):
    """Read a reference-format config file (plus the optional ``gpu`` block)."""
    path = path or default_config_path()
    with open(path) as f:
        raw = yaml.safe_load(f) or {}
    missing = [k for k in _REQUIRED if k not in raw]
    if missing:
        raise KeyError(f"{path}: missing required settings {missing}")
    kw = {attr: raw[key] for key, attr in _REQUIRED.items()}
    for key, default in _OPTIONAL.items():
        kw[key] = raw.get(key, default)
    if kw["beam_interp_method"] not in _VALID_INTERP:
        raise ValueError(f"beam_interp_method must be one of {sorted(_VALID_INTERP)!r}, "
                         f"got {kw['beam_interp_method']!r}")
    return TodConfig(gpu=GpuConfig.from_dict(raw.get("gpu")), CONFIG_FILE=os.path.abspath(path), **kw)


_loaded = None


def __getattr__(name):
    """Module constants like the reference's (loaded on first access)."""
    global _loaded
    if name.startswith("__"):
        raise AttributeError(name)
    if _loaded is None:
        _loaded = load_config()
    try:
        return getattr(_loaded, name)
    except AttributeError:
        raise AttributeError(f"module 'tod_config' has no setting {name!r}") from None
