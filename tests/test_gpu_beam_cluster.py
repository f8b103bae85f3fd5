"""GPU k-means of cluster_beam_pixels against golden outputs of the
reference (beam_cluster.py:215-397): full and hybrid modes, Gaussian beams
and a far-sidelobe annulus, 3 to 200 clusters.  Labels must be identical and
the float32 centroids and weights bit-identical (the per-cluster sums are
taken in the same order as the reference's numpy.bincount)."""

import numpy as np
import pytest

from conftest import load_cases, load_flat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def BC():
    from tod_generation_mapbased_beam_b200 import beam_cluster

    return beam_cluster


@pytest.mark.parametrize("case", ["0.05_20", "0.5_7"])
def test_hybrid_small_matches_reference(BC, case):
    g = load_flat("beam_prep")
    tf, k = case.split("_")
    vo, bo, lab = BC.cluster_beam_pixels(g["cl_vec_in"], g["cl_bv_in"], int(k), tail_fraction=float(tf),
                                         verbose=False)
    assert np.array_equal(lab, g[f"cl_{case}_labels"])
    assert np.array_equal(vo, g[f"cl_{case}_vec"])
    assert np.array_equal(bo, g[f"cl_{case}_bv"])


@pytest.mark.parametrize("case", sorted(load_cases("clusters")))
def test_larger_cases_match_reference(BC, case):
    g = load_cases("clusters")[case]
    tf = float(g["tail_fraction"])
    vo, bo, lab = BC.cluster_beam_pixels(g["vec_in"], g["bv_in"], int(g["k"]),
                                         tail_fraction=None if tf < 0 else tf, verbose=True)
    assert np.array_equal(lab, g["labels"])
    assert np.array_equal(vo, g["vec"])
    assert np.array_equal(bo, g["bv"])


def test_empty_cluster_reseeding_and_determinism(BC):
    # duplicated points force empty clusters: K larger than the distinct points
    rng = np.random.default_rng(3)
    base = rng.standard_normal((5, 3))
    base /= np.linalg.norm(base, axis=1, keepdims=True)
    vec = np.repeat(base, 40, axis=0).astype(np.float32)
    bv = np.full(len(vec), 1.0 / len(vec), np.float32)
    a = BC.cluster_beam_pixels(vec, bv, 8, verbose=False)
    b = BC.cluster_beam_pixels(vec, bv, 8, verbose=False)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert np.isclose(a[1].sum(), 1.0, atol=1e-6)
