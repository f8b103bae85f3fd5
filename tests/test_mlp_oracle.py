"""CPU checks of the learned-tail network oracle and of the network ABI's
host-side helpers (no GPU needed)."""

import ctypes

import numpy as np
import torch

from oracle import mlp_oracle as MO
from tod_generation_mapbased_beam_b200 import _native


def test_bf16_round_matches_torch():
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.standard_normal(20000) * 10.0 ** rng.integers(-30, 30, 20000),
                        [0.0, -0.0, 1.0, -1.0, 1.00390625, 1.01171875, 3.4e38, 1e-40, np.inf, -np.inf]])
    f32 = v.astype(np.float32)
    # exact ties: low halves equal to 0x8000 (round half to even)
    ties = ((np.arange(1000, dtype=np.uint32) + 0x3F80) << 16 | 0x8000).view(np.float32)
    f32 = np.concatenate([f32, ties, -ties])
    ref = torch.from_numpy(f32).to(torch.bfloat16).to(torch.float64).numpy()
    got = MO.bf16_round(f32)
    assert np.array_equal(got, ref)
    assert np.isnan(MO.bf16_round(np.array([np.nan]))).all()


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    dims = (3, 5, 3, 2)  # F, H, D, O (the oracle has no shape restrictions)
    _, _, n = MO.param_offsets(*dims)
    p = rng.standard_normal(n) * 0.5
    x = MO.inputs(rng.uniform(0, np.pi, 16), rng.uniform(0, 2 * np.pi, 16), rng.uniform(0, 2 * np.pi, 16))
    freq = rng.standard_normal((dims[0], 7))
    feat = MO.features(x, freq, bf16=False)
    t = rng.standard_normal((16, dims[3]))
    loss, g = MO.loss_grad(p, dims, feat, t, bf16=False)
    h = 1e-6
    for i in rng.choice(n, 60, replace=False).tolist() + [n - 1, n - 2]:
        e = np.zeros(n)
        e[i] = h
        lp, _ = MO.loss_grad(p + e, dims, feat, t, bf16=False)
        lm, _ = MO.loss_grad(p - e, dims, feat, t, bf16=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_adam_step_oracle_first_step_is_sign_step():
    g = np.array([1e-3, -2.0, 0.0])
    p, m, v = MO.adam_step(np.zeros(3), np.zeros(3), np.zeros(3), g, 1, 0.01)
    assert np.allclose(p[:2], [-0.01, 0.01], rtol=1e-4) and p[2] == 0.0


def _desc(F, H, D, O):
    d = _native.MlpDesc()
    d.n_freq, d.width, d.depth, d.n_out = F, H, D, O
    return d


def test_param_layout_matches_library():
    lib = _native.lib()
    for dims in [(64, 128, 1, 1), (256, 256, 4, 3), (128, 384, 8, 4)]:
        d = _desc(*dims)
        w = (ctypes.c_int64 * (dims[2] + 1))()
        b = (ctypes.c_int64 * (dims[2] + 1))()
        assert lib.todgpu_mlp_param_offsets(ctypes.byref(d), w, b) == 0
        ow, ob, total = MO.param_offsets(*dims)
        assert list(w) == ow and list(b) == ob
        assert lib.todgpu_mlp_param_count(ctypes.byref(d)) == total


def test_network_shape_validation():
    lib = _native.lib()
    for bad in [(32, 128, 2, 3), (64, 100, 2, 3), (64, 128, 0, 3), (64, 128, 9, 3), (64, 128, 2, 5)]:
        d = _desc(*bad)
        assert lib.todgpu_mlp_param_count(ctypes.byref(d)) == -1
        assert lib.todgpu_mlp_workspace_bytes(ctypes.byref(d), 256) == 0
    d = _desc(64, 128, 2, 3)
    assert lib.todgpu_mlp_workspace_bytes(ctypes.byref(d), 100) == 0
    off = (ctypes.c_int64 * 9)()
    assert lib.todgpu_mlp_workspace_offsets(ctypes.byref(d), 256, off) == 0
    assert list(off) == sorted(off) and off[8] == lib.todgpu_mlp_workspace_bytes(ctypes.byref(d), 256)
    # calls that would launch work are rejected before any CUDA call
    assert lib.todgpu_mlp_forward(ctypes.byref(d), None, 256, None, 0, None, None) == _native.EINVAL
    assert lib.todgpu_mlp_loss_grad(None, None, None, 256, None, 0, None, None) == _native.EINVAL
    assert lib.todgpu_mlp_adam(ctypes.byref(d), 1, 1e-3, 0.9, 0.999, 1e-8, None) == _native.EINVAL
    assert lib.todgpu_mlp_inputs(None, None, None, 7, 0, 128, None, None) == _native.EINVAL
