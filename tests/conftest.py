"""Shared pytest set-up: the ``gpu`` marker, repo root on sys.path and golden
fixture loaders."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_cases(name):
    """Load tests/golden/<name>.npz into {case: {field: array}}."""
    raw = np.load(os.path.join(GOLDEN, name + ".npz"))
    out = {}
    for key in raw.files:
        case, field = key.split("__", 1)
        out.setdefault(case, {})[field] = raw[key]
    return out


def load_flat(name):
    raw = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: raw[k] for k in raw.files}


KERNEL_CASES = load_cases("kernels")
PARAM_KEYS = ("vec_orig", "axes", "cos_a", "sin_a", "ax_pts", "cos_p", "sin_p")


@pytest.fixture(params=sorted(KERNEL_CASES))
def kernel_case(request):
    return request.param, KERNEL_CASES[request.param]
