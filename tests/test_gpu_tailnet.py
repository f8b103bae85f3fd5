"""GPU tests of the learned-tail network kernels against the CPU oracle
(oracle/mlp_oracle.py): inputs, Fourier features, every hidden layer, the
loss and the full gradient, the Adam step, training, and the TOD
accumulation entry point."""

import numpy as np
import pytest
import torch

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def TN():
    from tod_generation_mapbased_beam_b200 import tailnet

    return tailnet


def _pointings(n, seed):
    rng = np.random.default_rng(seed)
    return (np.arccos(rng.uniform(-1, 1, n)), rng.uniform(0, 2 * np.pi, n), rng.uniform(0, 2 * np.pi, n))


def _smooth_target(theta, phi, psi):
    x = MO.inputs(theta, phi, psi).astype(np.float64)
    return np.stack([np.sin(2 * x[:, 2]) + 0.3 * x[:, 0] * x[:, 1],
                     x[:, 5] * (1 - x[:, 2] ** 2) + 0.2 * x[:, 0],
                     x[:, 6] * x[:, 0] - 0.1 * np.cos(3 * x[:, 1])], -1)


def _bf16_region(net, rows, name, shape):
    raw = net.ws_region(rows, name)
    n = int(np.prod(shape))
    return raw.view(torch.bfloat16)[:n].view(*shape).double().cpu().numpy()


def _f32_region(net, rows, name, shape):
    raw = net.ws_region(rows, name)
    n = int(np.prod(shape))
    return raw.view(torch.float32)[:n].view(*shape).double().cpu().numpy()


def test_inputs_match_oracle(TN):
    net = TN.TailNet(64, 128, 2, 3)
    th, ph, ps = _pointings(1000, 1)
    x = net.inputs(th, ph, ps).cpu().numpy()
    assert x.shape == (1024, 7)
    assert np.allclose(x[:1000], MO.inputs(th, ph, ps), atol=2e-7, rtol=0)
    assert not x[1000:].any()
    x32 = net.inputs(th.astype(np.float32), ph.astype(np.float32), ps.astype(np.float32)).cpu().numpy()
    ref = MO.inputs(th.astype(np.float32), ph.astype(np.float32), ps.astype(np.float32))
    assert np.allclose(x32[:1000], ref, atol=2e-7, rtol=0)


def test_features_and_layers_match_oracle(TN):
    net = TN.TailNet(64, 128, 3, 3, sigma=(3.0, 1.0), seed=2)
    F, H, D, O = net.dims
    rows = 512
    th, ph, ps = _pointings(rows, 3)
    x = net.inputs(th, ph, ps)
    t = torch.from_numpy(_smooth_target(th, ph, ps).astype(np.float32)).cuda()
    net.loss_grad(x, t)
    torch.cuda.synchronize()
    feat = _bf16_region(net, rows, "feat", (rows, 2 * F))
    ref = MO.features(x.cpu().numpy(), net.freq.cpu().numpy(), bf16=False)
    assert np.abs(feat - ref).max() <= 2.0 ** -8 + 1e-5
    # each hidden layer from the GPU's own input to it (teacher forcing)
    z = _f32_region(net, rows, "z", (D, rows, H))
    a = _bf16_region(net, rows, "a", (D, rows, H))
    p = net.params.double().cpu().numpy()
    layers = MO.unpack(p, F, H, D, O)
    for l in range(D):
        a_in = feat if l == 0 else a[l - 1]
        W, b = layers[l]
        zo = a_in @ MO.bf16_round(W).T + b
        bound = np.abs(a_in) @ np.abs(MO.bf16_round(W)).T + np.abs(b)
        assert np.all(np.abs(z[l] - zo) <= 1e-5 * bound + 1e-7), l
        ao = MO.bf16_round(z[l] / (1 + np.exp(-z[l])))
        diff = a[l] != ao
        assert diff.mean() < 1e-3, l
        assert np.all(np.abs(a[l] - ao)[diff] <= 2.0 ** -7 * np.abs(ao)[diff] + 1e-30), l
    # head: the plain forward on the same inputs
    y = net.forward(x).double().cpu().numpy()
    a_last = _bf16_region(net, rows, "a", (D, rows, H))[D - 1]
    Wo, bo = layers[D]
    yo = a_last @ MO.bf16_round(Wo).T + bo
    assert np.abs(y - yo).max() <= 1e-5 * np.abs(yo).max() + 1e-6


def test_loss_and_gradient_match_oracle(TN):
    net = TN.TailNet(128, 256, 4, 3, sigma=(4.0, 1.0), seed=4)
    F, H, D, O = net.dims
    rows = 1024
    th, ph, ps = _pointings(rows, 5)
    x = net.inputs(th, ph, ps)
    tgt = _smooth_target(th, ph, ps)
    # move the weights off their initialisation so every layer carries gradient
    t32 = torch.from_numpy(tgt.astype(np.float32)).cuda()
    for _ in range(20):
        net.loss_grad(x, t32)
        net.adam(3e-3)
    loss, g = net.loss_grad(x, t32)
    torch.cuda.synchronize()
    feat = _bf16_region(net, rows, "feat", (rows, 2 * F))
    p = net.params.double().cpu().numpy()
    lo, go = MO.loss_grad(p, net.dims, feat, tgt.astype(np.float32).astype(np.float64))
    assert abs(loss - lo) <= 1e-4 * lo
    g = g.double().cpu().numpy()
    w_off, b_off, total = MO.param_offsets(*net.dims)
    for l in range(D + 1):
        n_out = H if l < D else O
        n_in = (2 * F if l == 0 else H) if l < D else H
        for lo_, hi_ in [(w_off[l], w_off[l] + n_out * n_in), (b_off[l], b_off[l] + n_out)]:
            err = np.linalg.norm(g[lo_:hi_] - go[lo_:hi_])
            assert err <= 5e-3 * np.linalg.norm(go[lo_:hi_]) + 1e-9, (l, err, np.linalg.norm(go[lo_:hi_]))


def test_gradient_is_deterministic(TN):
    net = TN.TailNet(64, 128, 2, 3, seed=6)
    th, ph, ps = _pointings(2048, 7)
    x = net.inputs(th, ph, ps)
    t = torch.from_numpy(_smooth_target(th, ph, ps).astype(np.float32)).cuda()
    _, g1 = net.loss_grad(x, t)
    g1 = g1.clone()
    _, g2 = net.loss_grad(x, t)
    assert torch.equal(g1, g2)


def test_adam_step_matches_oracle(TN):
    net = TN.TailNet(64, 128, 2, 3, seed=8)
    th, ph, ps = _pointings(512, 9)
    x = net.inputs(th, ph, ps)
    t = torch.from_numpy(_smooth_target(th, ph, ps).astype(np.float32)).cuda()
    p = net.params.double().cpu().numpy()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for step in (1, 2, 3):
        _, g = net.loss_grad(x, t)
        gh = g.double().cpu().numpy()
        net.adam(1e-3)
        p, m, v = MO.adam_step(p, m, v, gh, step, 1e-3)
        pg = net.params.double().cpu().numpy()
        assert np.abs(pg - p).max() <= 5e-8 + 1e-7 * np.abs(p).max()
        p = pg  # continue from the GPU's float32 parameters
    assert np.array_equal(net.params_bf16.double().cpu().numpy(), MO.bf16_round(net.params.cpu().numpy()))


def test_training_learns_a_smooth_function(TN):
    # frequencies low enough for 32K samples of a 3-dimensional pointing manifold
    # (at sigma 2 the same network memorises the set and does not generalise)
    net = TN.TailNet(128, 256, 4, 3, sigma=(0.5, 0.5), seed=10)
    th, ph, ps = _pointings(1 << 15, 11)
    x = net.inputs(th, ph, ps)
    tgt = _smooth_target(th, ph, ps)
    losses = net.fit(x, tgt, steps=1500, batch=2048, lr_max=2e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-50:].mean() < 0.01 * losses[:10].mean()
    th2, ph2, ps2 = _pointings(4096, 12)
    ref = _smooth_target(th2, ph2, ps2)
    err = net.predict(th2, ph2, ps2) - ref
    assert np.all(np.sqrt((err ** 2).mean(0)) < 0.05 * ref.std(0))


def test_accumulate_matches_predict_and_chunking(TN):
    net = TN.TailNet(64, 128, 2, 3, seed=13)
    net.shift = np.array([1e-6, -2e-6, 0.5e-6])
    net.scale = np.array([3e-6, 1e-6, 2e-6])
    B = 1000
    th, ph, ps = _pointings(B, 14)
    pred = net.predict(th, ph, ps)
    d = [torch.from_numpy(a).cuda() for a in (th, ph, ps)]
    outs = []
    for chunk in (128, 384, 1 << 20):
        tod = torch.zeros((4, B), dtype=torch.float64, device="cuda")
        tod[2] = 7.0
        net.accumulate(*d, tod, rows=(3, 0, 1), chunk=chunk)
        outs.append(tod.cpu().numpy())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    o = outs[0]
    assert np.array_equal(o[2], np.full(B, 7.0))
    assert np.allclose(o[3], pred[:, 0], rtol=1e-12, atol=0)
    assert np.allclose(o[0], pred[:, 1], rtol=1e-12, atol=0)
    assert np.allclose(o[1], pred[:, 2], rtol=1e-12, atol=0)


def test_state_round_trip(TN):
    net = TN.TailNet(64, 128, 2, 3, seed=15)
    net.shift = np.array([1.0, 2.0, 3.0])
    th, ph, ps = _pointings(300, 16)
    a = net.predict(th, ph, ps)
    net2 = TN.TailNet.from_state(net.state())
    assert np.array_equal(net2.predict(th, ph, ps), a)


def test_bad_rows_rejected(TN):
    from tod_generation_mapbased_beam_b200 import _native

    net = TN.TailNet(64, 128, 2, 3)
    x = torch.zeros((100, 7), dtype=torch.float32, device="cuda")
    with pytest.raises((_native.TodGpuError, ValueError)):
        net.forward(x)


@pytest.mark.parametrize("width", [128, 256])
def test_tcgen05_forward_matches_mma_sync_forward(TN, width):
    from tod_generation_mapbased_beam_b200 import _native

    lib = _native.lib()
    net = TN.TailNet(128, width, 3, 3, sigma=(2.0, 1.0), seed=17)
    th, ph, ps = _pointings(4096, 18)
    x = net.inputs(th, ph, ps)
    prev = lib.todgpu_mlp_set_forward_path(_native.MLP_MMA_SYNC)
    try:
        y_ref = net.forward(x).double().cpu().numpy()
        a_ref = _bf16_region(net, 4096, "a", (3, 4096, width))
        lib.todgpu_mlp_set_forward_path(_native.MLP_TCGEN05)
        n0 = lib.todgpu_mlp_tcgen05_launches()
        y_tc = net.forward(x).double().cpu().numpy()
        assert lib.todgpu_mlp_tcgen05_launches() == n0 + 3  # every hidden layer ran on tcgen05
        a_tc = _bf16_region(net, 4096, "a", (3, 4096, width))
    finally:
        lib.todgpu_mlp_set_forward_path(prev)
    assert lib.todgpu_mlp_wait_timeouts() == 0
    # same bf16 operands, float32 sums in a different order: activations agree
    # to a bf16 rounding step, the outputs to float32 sums
    diff = a_tc != a_ref
    assert diff.mean() < 0.02
    assert np.all(np.abs(a_tc - a_ref) <= 2.0 ** -6 * np.abs(a_ref) + 1e-6)
    assert np.abs(y_tc - y_ref).max() <= 1e-3 * np.abs(y_ref).max()


def test_forward_path_switch_rejects_unknown():
    from tod_generation_mapbased_beam_b200 import _native

    assert _native.lib().todgpu_mlp_set_forward_path(7) == _native.EINVAL


def test_data_parallel_trainer_on_one_rank_equals_fused_training():
    """The data-parallel step sequence (per-step gradient, the all-reduce
    that is the identity on one rank, Adam) trains the network exactly as the
    fused todgpu_mlp_train loop does: same batches, learning rates and Adam
    steps, same parameters bit for bit."""
    from tod_generation_mapbased_beam_b200.dp_train import DataParallelTrainer
    from tod_generation_mapbased_beam_b200.tailnet import TailNet

    rng = np.random.default_rng(21)
    n = 2048
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    ps = rng.uniform(0, 2 * np.pi, n)
    target = np.stack([np.sin(2 * th) * np.cos(ph), np.cos(ps) * th, np.sin(ph + ps)], -1) * 1e-7
    nets = [TailNet(n_freq=64, width=128, depth=2, n_out=3, seed=4) for _ in range(2)]
    x = nets[0].inputs(th, ph, ps)
    fused = nets[0].fit(x, target, steps=40, batch=512)
    dp = DataParallelTrainer(nets[1]).fit(x, target, 40, 512)
    assert torch.equal(nets[0].params, nets[1].params)
    np.testing.assert_allclose(dp, fused, rtol=1e-6)
