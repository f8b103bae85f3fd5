"""Learned-tail TOD: the main lobe exact, the far-sidelobe tail from a network.

A beam is split into a main lobe, which keeps going through the gather kernel
(``todgpu_gather_accum``, pointing as angles, here with the packed float32
map and Kahan sums of the precision form), and a far-sidelobe tail of many
low-weight pixels, whose TOD contribution is a smooth function of the
pointing.  :class:`LearnedTailTOD` computes tail targets with the plain
method -- the same gather kernel on the tail pixels with the float64 map --
at pointings uniform on the sphere (theta, phi) and in roll psi, trains a
:class:`~tod_generation_mapbased_beam_b200.tailnet.TailNet` on them, judges it
on held-out pointings of a scan against the plain tail sum, and then adds its
prediction in place of the tail.  The plain tail sum stays available as the
fallback (``tail="plain"``; ``tail="auto"`` chooses it when the held-out error
measured by :meth:`LearnedTailTOD.judge` exceeds the budget).

The reference reduces a tail by k-means clustering instead
(beam_cluster.py:215-397, hybrid mode); the main/tail split rule of that mode
is ``beam_cluster.split_main_tail``.
"""

from __future__ import annotations

import time

import numpy as np
import torch

from . import _native
from ._device import require_cuda
from .kernels import beam_order, gather_accum_angles, pack_map
from .tailnet import TailNet

_INTERP = {"bilinear": _native.BILINEAR, "nearest": _native.NEAREST}


def uniform_pointings(n, seed):
    """(theta, phi, psi) float64, uniform on the sphere and in roll."""
    rng = np.random.default_rng(seed)
    return (np.arccos(rng.uniform(-1.0, 1.0, n)), rng.uniform(0.0, 2 * np.pi, n), rng.uniform(0.0, 2 * np.pi, n))


class LearnedTailTOD:
    """I/Q/U TOD of one beam entry (components [I, Q, U], spin-2 on) with the
    tail learned.

    ``sky``: (3, 12 nside^2) float64 map (numpy or CUDA tensor).  ``main`` and
    ``tail``: beams with ``vec_orig`` (S, 3) and ``beam_vals`` (S,) in the
    beam frame centred on the pole.  ``center``: beam centre (phi, theta) of the
    angle-mode pointing.  ``main_map``: "f32" or "bf16" (packed precision form)
    or "f64" for the main lobe."""

    def __init__(self, nside, sky, main, tail, center=(0.0, 0.0), main_map="f32", interp="bilinear",
                 tail_chunk=16384):
        self.device = require_cuda()
        self.nside = int(nside)
        sky = torch.as_tensor(sky, dtype=torch.float64, device=self.device).contiguous()
        if sky.shape != (3, 12 * self.nside ** 2):
            raise ValueError("sky must be a (3, 12 nside^2) I/Q/U map")
        self.sky = sky
        self.sky_main = sky if main_map == "f64" else pack_map(sky, main_map)
        self.main_map = main_map
        self.interp = _INTERP[interp]
        self.center = (float(center[0]), float(center[1]))
        # beam pixels in the gather's preferred order (neighbours on the sky next
        # to each other; only the order of the pixel sums changes)
        mo, to_ = beam_order(main.vec_orig), beam_order(tail.vec_orig)
        self.main_vec = torch.as_tensor(np.asarray(main.vec_orig, np.float64)[mo], device=self.device)
        self.main_bv = torch.as_tensor(np.asarray(main.beam_vals, np.float32)[mo], device=self.device)
        self.tail_vec = torch.as_tensor(np.asarray(tail.vec_orig, np.float64)[to_], device=self.device)
        self.tail_bv = torch.as_tensor(np.asarray(tail.beam_vals, np.float32)[to_], device=self.device)
        self.tail_chunk = int(tail_chunk)
        self.net = None
        self.judged = None

    # -- plain method --------------------------------------------------------
    def _gather(self, vec, bv, mp, theta, phi, psi, tod):
        gather_accum_angles(self.interp, vec, theta, phi, psi, self.center[0], self.center[1], self.nside, mp, bv,
                            tod, c_q=1, c_u=2)

    @staticmethod
    def _dev(a, dev):
        t = torch.as_tensor(a, device=dev)
        return t if t.dtype in (torch.float32, torch.float64) else t.double()

    def plain_tail(self, theta, phi, psi, tod=None):
        """Tail contribution by the plain method (float64 map), (3, B) float64;
        accumulated into ``tod`` when given.  Launches cover ``tail_chunk``
        samples each."""
        th, ph, ps = (self._dev(a, self.device) for a in (theta, phi, psi))
        B = th.numel()
        if tod is None:
            tod = torch.zeros((3, B), dtype=torch.float64, device=self.device)
        for b0 in range(0, B, self.tail_chunk):
            b1 = min(B, b0 + self.tail_chunk)
            part = torch.zeros((3, b1 - b0), dtype=torch.float64, device=self.device)
            self._gather(self.tail_vec, self.tail_bv, self.sky, th[b0:b1], ph[b0:b1], ps[b0:b1], part)
            tod[:, b0:b1] += part
        return tod

    def main_lobe(self, theta, phi, psi, tod=None, exact=False):
        """Main-lobe contribution, (3, B) float64: the packed map form, or the
        float64 map with ``exact``."""
        th, ph, ps = (self._dev(a, self.device) for a in (theta, phi, psi))
        if tod is None:
            tod = torch.zeros((3, th.numel()), dtype=torch.float64, device=self.device)
        self._gather(self.main_vec, self.main_bv, self.sky if exact else self.sky_main, th, ph, ps, tod)
        return tod

    def full_plain(self, theta, phi, psi):
        """The whole beam by the plain float64 method: main lobe (float64 map)
        plus plain tail -- the reference answer the learned form is judged by."""
        tod = self.main_lobe(theta, phi, psi, exact=True)
        return self.plain_tail(theta, phi, psi, tod)

    # -- the network -----------------------------------------------------------
    def fit(self, n_train=1 << 18, steps=4000, batch=8192, seed=6, net=None, lr_max=2e-3, lr_min=2e-5,
            group=None, **net_kwargs):
        """Tail targets at ``n_train`` uniform pointings (plain method), then
        training.  Returns timing and loss information.

        ``group``: a torch.distributed process group (one process per GPU, all
        calling fit with the same arguments).  Each rank then computes the
        targets of its share of the pointings and the ranks train together
        (``dp_train.DataParallelTrainer``: gradients all-reduced every step,
        ``batch`` rows per step over all ranks); every rank ends with the same
        network."""
        import torch.distributed as dist

        world = dist.get_world_size(group) if group is not None else 1
        rank = dist.get_rank(group) if world > 1 else 0
        t0 = time.perf_counter()
        th, ph, ps = uniform_pointings(int(n_train), seed)
        if world > 1:
            from .sharding import sample_shard

            a, b = sample_shard(int(n_train), rank, world)
            th, ph, ps = th[a:b], ph[a:b], ps[a:b]
        th_d, ph_d, ps_d = (torch.from_numpy(a).to(self.device) for a in (th, ph, ps))
        target = self.plain_tail(th_d, ph_d, ps_d)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        self.net = net if net is not None else TailNet(n_out=3, **net_kwargs)
        x = self.net.inputs(th_d, ph_d, ps_d)
        if world > 1:
            from .dp_train import DataParallelTrainer

            trainer = DataParallelTrainer(self.net, group)
            trainer.sync_parameters()
            losses = trainer.fit(x[:th.size], target.T.contiguous(), steps, batch // world, lr_max=lr_max,
                                 lr_min=lr_min)
        else:
            losses = self.net.fit(x[:th.size], target.T.contiguous(), steps=steps, batch=batch, lr_max=lr_max,
                                  lr_min=lr_min)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        self.judged = None
        return dict(n_train=int(n_train), steps=int(steps), batch=int(batch), target_seconds=t1 - t0,
                    train_seconds=t2 - t1, loss_first=float(losses[:10].mean()),
                    loss_last=float(losses[-100:].mean()), target_rms_K=target.std(dim=1).cpu().numpy().tolist(),
                    ranks=world)

    def learned_tail(self, theta, phi, psi, tod=None):
        """Tail contribution from the network, (3, B) float64."""
        if self.net is None:
            raise RuntimeError("no tail network: call fit() first")
        th, ph, ps = (self._dev(a, self.device) for a in (theta, phi, psi))
        if tod is None:
            tod = torch.zeros((3, th.numel()), dtype=torch.float64, device=self.device)
        self.net.accumulate(th, ph, ps, tod, rows=(0, 1, 2))
        return tod

    # -- judge and TOD ---------------------------------------------------------
    def judge(self, theta, phi, psi, budget_uK=0.1):
        """Errors in uK of the learned form against the plain float64 method on
        the given (held-out) samples, and of the same form with the tail
        dropped.  Sets the fallback decision for ``tod(tail="auto")``: the
        network is used only if the RMS error of every Stokes component is
        within ``budget_uK``."""
        ref = self.full_plain(theta, phi, psi)
        main = self.main_lobe(theta, phi, psi)
        learned = self.learned_tail(theta, phi, psi, main.clone())
        tail = self.plain_tail(theta, phi, psi)

        def stats(d):
            d = d.cpu().numpy() * 1e6
            return dict(rms_uK=np.sqrt((d ** 2).mean(axis=1)).tolist(), max_uK=np.abs(d).max(axis=1).tolist(),
                        rms_all_uK=float(np.sqrt((d ** 2).mean())))

        out = dict(samples=int(ref.shape[1]), learned=stats(learned - ref), dropped=stats(main - ref),
                   tail_rms_uK=(tail.std(dim=1).cpu().numpy() * 1e6).tolist(),
                   surrogate=stats(learned - main - tail), budget_uK=float(budget_uK))
        out["use_surrogate"] = max(out["learned"]["rms_uK"]) <= budget_uK
        self.judged = out
        return out

    def tod(self, theta, phi, psi, tail="auto"):
        """(3, B) float64 I/Q/U TOD: main lobe plus the tail from the network
        ("learned"), the plain method ("plain"), the choice made by judge() ("auto"),
        or none ("none")."""
        if tail == "auto":
            if self.judged is None:
                raise RuntimeError("tail='auto' needs judge() first")
            tail = "learned" if self.judged["use_surrogate"] else "plain"
        tod = self.main_lobe(theta, phi, psi)
        if tail == "learned":
            return self.learned_tail(theta, phi, psi, tod)
        if tail == "plain":
            return self.plain_tail(theta, phi, psi, tod)
        if tail == "none":
            return tod
        raise ValueError("tail must be 'auto', 'learned', 'plain' or 'none'")
