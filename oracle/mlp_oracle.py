"""CPU oracle of the learned-tail network -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` (and the CPU legs of ``bench.py``) may import this module.
It restates, in float64 numpy, the network that ``todgpu_mlp_*`` trains and
evaluates on the GPU (declared in ``include/todgpu.h``): the pointing inputs,
random Fourier features, SiLU hidden layers, the linear head, the mean squared
error and its gradient by reverse-mode differentiation, and one Adam step.

The GPU keeps weights and activations in bfloat16 and sums in float32.  With
``bf16=True`` this oracle rounds to bfloat16 at the same points (weights in the
contractions, stored features, activations and back-propagated pre-activation
gradients), so that GPU and oracle differ only by float32 summation order and
by the rare bfloat16 rounding flip that order causes.  With ``bf16=False`` it
is the exact float64 network, used to check the gradient by finite
differences.

The reference has no learned tail (its tail reduction is the k-means
clustering of beam_cluster.py:215-397); there is nothing of the reference to
pin this oracle to.  It is pinned instead by (i) a finite-difference check of
its own gradient and (ii) torch's CPU bfloat16 conversion for the rounding.
"""

from __future__ import annotations

import numpy as np

N_IN = 7


def bf16_round(a):
    """Round to the nearest bfloat16 (ties to even) via float32; returns float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    nan = np.isnan(f)
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)
    out[nan] = np.nan
    return out


def param_offsets(F, H, D, O):
    """Element offsets (w[l], b[l]) for l = 0..D (D = head) and the total count:
    per layer the weight matrix (row-major, out x in) then the bias."""
    w, b = [], []
    p = 0
    for l in range(D):
        k = 2 * F if l == 0 else H
        w.append(p)
        p += H * k
        b.append(p)
        p += H
    w.append(p)
    p += O * H
    b.append(p)
    p += O
    return w, b, p


def unpack(params, F, H, D, O):
    """[(W_l, b_l)] views of the flat parameter vector."""
    w, b, _ = param_offsets(F, H, D, O)
    out = []
    for l in range(D + 1):
        n_out = H if l < D else O
        n_in = (2 * F if l == 0 else H) if l < D else H
        out.append((params[w[l]:w[l] + n_out * n_in].reshape(n_out, n_in), params[b[l]:b[l] + n_out]))
    return out


def inputs(theta, phi, psi):
    """(n, 7) float32 inputs (sin t cos p, sin t sin p, cos t, cos psi, sin psi,
    cos 2 psi, sin 2 psi), computed in float64."""
    t = np.asarray(theta, np.float64)
    p = np.asarray(phi, np.float64)
    s = np.asarray(psi, np.float64)
    st, ct, sp, cp, ss, cs = np.sin(t), np.cos(t), np.sin(p), np.cos(p), np.sin(s), np.cos(s)
    x = np.stack([st * cp, st * sp, ct, cs, ss, cs * cs - ss * ss, 2 * ss * cs], -1)
    return x.astype(np.float32)


def features(x, freq, bf16=True):
    """(n, 2F) [cos(2 pi z), sin(2 pi z)] with z = x freq^T."""
    z = np.asarray(x, np.float64) @ np.asarray(freq, np.float64).T
    f = np.concatenate([np.cos(2 * np.pi * z), np.sin(2 * np.pi * z)], axis=1)
    return bf16_round(f) if bf16 else f


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, dims, feat, bf16=True):
    """Hidden pre-activations z_l, activations a_l and the head output y for
    features ``feat`` (n, 2F)."""
    F, H, D, O = dims
    layers = unpack(np.asarray(params, np.float64), F, H, D, O)
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    a = np.asarray(feat, np.float64)
    zs, acts = [], []
    for l in range(D):
        W, b = layers[l]
        z = a @ rnd(W).T + b
        a = rnd(_silu(z))
        zs.append(z)
        acts.append(a)
    Wo, bo = layers[D]
    y = a @ rnd(Wo).T + bo
    return zs, acts, y


def loss_grad(params, dims, feat, target, bf16=True):
    """(mean squared error, flat float64 gradient) of one batch."""
    F, H, D, O = dims
    params = np.asarray(params, np.float64)
    layers = unpack(params, F, H, D, O)
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    feat = np.asarray(feat, np.float64)
    zs, acts, y = forward(params, dims, feat, bf16)
    M = feat.shape[0]
    r = y - np.asarray(target, np.float64)
    loss = float(np.sum(r * r) / (M * O))
    dy = r * (2.0 / (M * O))
    w_off, b_off, total = param_offsets(F, H, D, O)
    g = np.zeros(total)
    Wo, _ = layers[D]
    g[w_off[D]:w_off[D] + O * H] = (dy.T @ acts[-1]).ravel()
    g[b_off[D]:b_off[D] + O] = dy.sum(0)
    dz = rnd((dy @ rnd(Wo)) * _dsilu(zs[-1]))
    for l in range(D - 1, -1, -1):
        a_in = feat if l == 0 else acts[l - 1]
        W, _ = layers[l]
        g[w_off[l]:w_off[l] + W.size] = (dz.T @ a_in).ravel()
        g[b_off[l]:b_off[l] + W.shape[0]] = dz.sum(0)
        if l > 0:
            dz = rnd((dz @ rnd(W)) * _dsilu(zs[l - 1]))
    return loss, g


def adam_step(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (step counts from 1); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
