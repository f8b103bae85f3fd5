"""CPU tests of the config.yaml reader (reference keys, defaults and checks of
tod_config.py:1-63, plus the gpu block)."""

import importlib

import pytest

from tod_generation_mapbased_beam_b200 import tod_config as TC

BASE = """
FOLDER_SCAN: "/data/scan/"
FOLDER_TOD_OUTPUT: "/data/tod/"
path_to_map: "/data/sky.fits"
FOLDER_BEAM: "/data/beam/"
beam_file_I: "bI.fits"
beam_file_Q: "bQ.fits"
beam_file_U: "bU.fits"
power_fraction_threshold_I: 0.99
power_fraction_threshold_Q: 0.99
power_fraction_threshold_U: 0.98
start_day: 3
end_day: 10
n_processes: 4
"""


def _write(tmp_path, text, name="config.yaml"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_reference_keys_and_defaults(tmp_path):
    c = TC.load_config(_write(tmp_path, BASE))
    assert c.FOLDER_SCAN == "/data/scan/" and c.FOLDER_BEAM == "/data/beam/"
    assert (c.power_threshold_I, c.power_threshold_Q, c.power_threshold_U) == (0.99, 0.99, 0.98)
    assert (c.start_day, c.end_day, c.n_processes) == (3, 10, 4)
    assert c.beam_interp_method == "bilinear" and c.calibration_enabled is True
    assert c.n_beam_clusters is None and c.beam_cluster_tail_fraction is None
    assert c.clustering_error_threshold == 1e-3 and c.mp_start_method == "spawn"
    assert c.gpu.pointing == "device" and c.gpu.map_precision == "f64" and not c.gpu.learned_tail.enabled
    assert c.driver_kwargs() == {"interp_mode": "bilinear", "pointing": "device"}


def test_optional_and_gpu_block(tmp_path):
    text = BASE + """
beam_interp_method: 'nearest'
n_beam_clusters: 100
beam_cluster_tail_fraction: 0.03
gpu:
  pointing: reference
  map_precision: bf16
  chunk: 4096
  learned_tail: {enabled: true, budget_uK: 0.05}
"""
    c = TC.load_config(_write(tmp_path, text))
    assert c.beam_interp_method == "nearest"
    assert (c.n_beam_clusters, c.beam_cluster_tail_fraction) == (100, 0.03)
    assert c.gpu.pointing == "reference" and c.gpu.map_precision == "bf16" and c.gpu.chunk == 4096
    assert c.gpu.learned_tail.enabled and c.gpu.learned_tail.budget_uK == 0.05


@pytest.mark.parametrize("extra", ["beam_interp_method: 'gaussian'\n", "gpu: {map_precision: f16}\n",
                                   "gpu: {pointing: host}\n", "gpu: {colour: red}\n",
                                   "gpu: {learned_tail: {budget_uK: -1}}\n"])
def test_invalid_settings_rejected(tmp_path, extra):
    with pytest.raises(ValueError):
        TC.load_config(_write(tmp_path, BASE + extra))


def test_missing_required_key(tmp_path):
    with pytest.raises(KeyError):
        TC.load_config(_write(tmp_path, BASE.replace('FOLDER_SCAN: "/data/scan/"\n', "")))


def test_module_constants_like_the_reference(tmp_path, monkeypatch):
    monkeypatch.setenv("TODGPU_CONFIG", _write(tmp_path, BASE))
    mod = importlib.reload(TC)
    assert mod.FOLDER_TOD_OUTPUT == "/data/tod/"
    assert mod.power_threshold_U == 0.98
    assert mod.CONFIG_FILE.endswith("config.yaml")
    with pytest.raises(AttributeError):
        mod.not_a_setting
    importlib.reload(TC)
