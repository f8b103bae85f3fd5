"""CPU tests of the beam_cluster drop-in: the main/tail split rule and the
cases that need no clustering, against golden outputs of the reference's
cluster_beam_pixels (beam_cluster.py:215-397), and the k-means ABI's argument
checks (no GPU needed)."""

import numpy as np
import pytest

from conftest import load_flat
from tod_generation_mapbased_beam_b200 import _native
from tod_generation_mapbased_beam_b200 import beam_cluster as BC


@pytest.mark.parametrize("case", ["0.05_20", "0.2_10000", "0.5_7"])
def test_split_main_tail_matches_reference_labels(case):
    g = load_flat("beam_prep")
    tf = float(case.split("_")[0])
    main_idx, tail_idx = BC.split_main_tail(g["cl_bv_in"], tf)
    lab = g[f"cl_{case}_labels"]
    n_main = len(main_idx)
    assert np.array_equal(lab[main_idx], np.arange(n_main))
    assert np.all(lab[tail_idx] >= n_main)
    assert np.array_equal(np.sort(np.concatenate([main_idx, tail_idx])), np.arange(len(lab)))


def test_unclustered_tail_is_bit_exact():
    g = load_flat("beam_prep")
    vo, bo, lab = BC.cluster_beam_pixels(g["cl_vec_in"], g["cl_bv_in"], 10000, tail_fraction=0.2, verbose=False)
    assert np.array_equal(vo, g["cl_0.2_10000_vec"])
    assert np.array_equal(bo, g["cl_0.2_10000_bv"])
    assert np.array_equal(lab, g["cl_0.2_10000_labels"])


def test_full_mode_without_reduction_passes_through():
    g = load_flat("beam_prep")
    vec, bv = g["cl_vec_in"], g["cl_bv_in"]
    vo, bo, lab = BC.cluster_beam_pixels(vec, bv, len(bv) + 5, verbose=False)
    assert np.array_equal(vo, vec) and np.array_equal(bo, bv) and np.array_equal(lab, np.arange(len(bv)))


def test_bad_tail_fraction_rejected():
    g = load_flat("beam_prep")
    for tf in (0.0, 1.0, -0.1):
        with pytest.raises(ValueError):
            BC.cluster_beam_pixels(g["cl_vec_in"], g["cl_bv_in"], 5, tail_fraction=tf, verbose=False)


def test_kmeans_abi_validation():
    lib = _native.lib()
    assert lib.todgpu_kmeans_workspace_bytes(0, 4) == 0
    assert lib.todgpu_kmeans_workspace_bytes(100, 9000) == 0
    assert lib.todgpu_kmeans_workspace_bytes(100, 4) > 0
    assert lib.todgpu_kmeans_assign(None, 0, None, 4, None, None, None) == _native.ESHAPE
    assert lib.todgpu_kmeans_assign(None, 10, None, 9000, None, None, None) == _native.ESHAPE
    assert lib.todgpu_kmeans_assign(None, 10, None, 4, None, None, None) == _native.EINVAL
    assert lib.todgpu_kmeans_seed(None, None, 10, 4, None, None, None, None, 0, None) == _native.EINVAL
    assert lib.todgpu_kmeans_sums(None, None, None, 10, 4, None, None, 0, None) == _native.EINVAL
    assert lib.todgpu_kmeans_argmin(None, 0, None, None) == _native.ESHAPE
