"""GPU tests of the learned-tail form on a reduced configuration (nside 128
sky, beam pixelised at nside 256: 4 deg main lobe, 10-20 deg tail annulus of
17,604 pixels carrying 1% of the power).

* the plain float64 form (main lobe + plain tail) against the CPU FP64 oracle
  of the whole beam;
* what the trained network gains: its TOD error against the plain float64
  form is well below that of the same form with the tail dropped;
* the fallback: tail="plain" is exactly the plain tail, "auto" follows the
  judged error against the budget."""

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from tod_generation_mapbased_beam_b200 import learned as L
    from tod_generation_mapbased_beam_b200 import sky as SKY
    from tod_generation_mapbased_beam_b200 import workloads as W

    nside = 128
    sky = SKY.synfast_iqu(nside, seed=2)
    main, tail = W.config5_beams(beam_nside=256, fwhm_arcmin=240.0)
    lt = L.LearnedTailTOD(nside, sky, main, tail)
    return L, W, lt, main, tail, sky.cpu().numpy(), nside


def _scan(W, n, step):
    th, ph, ps = W.spin_scan(n * step, 100.0)
    return th[::step].copy(), ph[::step].copy(), ps[::step].copy()


def test_plain_form_matches_fp64_oracle(setup):
    L, W, lt, main, tail, sky, nside = setup
    th, ph, ps = _scan(W, 48, 20011)
    got = lt.full_plain(torch.from_numpy(th).cuda(), torch.from_numpy(ph).cuda(),
                        torch.from_numpy(ps).cuda()).cpu().numpy()
    vec = np.concatenate([main.vec_orig, tail.vec_orig]).astype(np.float64)
    bv = np.concatenate([main.beam_vals, tail.beam_vals])
    B = th.size
    rot, beta = oracle.rotation_vectors_f64(0.0, 0.0, ph.astype(np.float64), th.astype(np.float64))
    params = oracle.rotation_params_f64(rot, ph, th, ps.astype(np.float64) - beta)
    ref = np.zeros((3, B))
    oracle.gather_accum_fused(vec, *params, nside, sky, bv, B, vec.shape[0], ref, 1, 2, f64=True)
    # float64 everywhere; only summation order and device pointing ulps differ
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_trained_network_beats_dropping_the_tail(setup):
    L, W, lt, main, tail, sky, nside = setup
    info = lt.fit(n_train=1 << 17, steps=3000, batch=4096, n_freq=128, width=256, depth=4)
    assert info["loss_last"] < 0.05 * info["loss_first"]
    th, ph, ps = _scan(W, 2048, 4001)
    j = lt.judge(torch.from_numpy(th).cuda(), torch.from_numpy(ph).cuda(), torch.from_numpy(ps).cuda(),
                 budget_uK=1e9)
    learned, dropped = j["learned"]["rms_uK"], j["dropped"]["rms_uK"]
    # the tail is worth keeping, and the network keeps most of it
    assert dropped[0] > 0.01
    for c in range(3):
        assert learned[c] < 0.3 * dropped[c], (c, learned, dropped)
    assert j["use_surrogate"]


def test_fallback_and_auto_choice(setup):
    L, W, lt, main, tail, sky, nside = setup
    if lt.net is None:
        lt.fit(n_train=1 << 13, steps=100, batch=2048, sigma=(1.0, 0.5), n_freq=64, width=128, depth=2)
    th, ph, ps = (torch.from_numpy(a).cuda() for a in _scan(W, 256, 977))
    plain = lt.tod(th, ph, ps, tail="plain")
    ref = lt.plain_tail(th, ph, ps, lt.main_lobe(th, ph, ps))
    assert torch.equal(plain, ref)
    none = lt.tod(th, ph, ps, tail="none")
    assert torch.equal(none, lt.main_lobe(th, ph, ps))
    lt.judge(th, ph, ps, budget_uK=0.0)
    assert not lt.judged["use_surrogate"]
    assert torch.equal(lt.tod(th, ph, ps, tail="auto"), plain)
    lt.judge(th, ph, ps, budget_uK=1e9)
    assert torch.equal(lt.tod(th, ph, ps, tail="auto"), lt.tod(th, ph, ps, tail="learned"))
    with pytest.raises(ValueError):
        lt.tod(th, ph, ps, tail="bogus")
