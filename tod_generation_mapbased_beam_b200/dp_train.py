"""Data-parallel training of the tail network: one process per GPU.

Training targets of the learned tail are independent per pointing, so each
rank computes the plain-method targets of its own share of the training
pointings (``sharding.sample_shard``) and keeps them.  A training step is
then: every rank takes its next local batch, computes the mean-squared-error
gradient on it with the library's kernels, the ranks sum their gradients
(weighted by their rows) with one all-reduce of the float32 gradient vector
(NCCL on GPUs, gloo on the CPU), and every rank applies the same Adam step --
so the parameters stay identical on all ranks and equal those of one process
training on the concatenated batches.  The target normalisation (per-output
mean and standard deviation) is reduced over all ranks' targets the same way.

The learning-rate schedule and the batch order are those of
``todgpu_mlp_train``: cosine from ``lr_max`` to ``lr_min`` over
``total_steps``; step k takes local rows [(k mod n_batches) b, ... + b).

``net`` is a :class:`~tod_generation_mapbased_beam_b200.tailnet.TailNet` (or
anything with ``params``, ``grad``, ``step``, ``shift``, ``scale``,
``loss_grad(x, t)`` and ``adam(lr)`` of the same meaning).  Every rank must
make the same calls in the same order.

The reference has no learned tail and no multi-process training; this is
the data-parallel MLP step of the path's multi-GPU plan.
"""

from __future__ import annotations

import math

import numpy as np
import torch

__all__ = ["DataParallelTrainer", "cosine_lr"]


def cosine_lr(step, total_steps, lr_max, lr_min):
    """Learning rate of step ``step`` (0-based), as todgpu_mlp_train sets it:
    float32 lr_max and lr_min and their float32 difference, the cosine factor
    in float64, the result rounded to float32."""
    hi, lo = np.float32(lr_max), np.float32(lr_min)
    span = float(np.float32(hi - lo))
    c = 0.5 * (1.0 + math.cos(math.pi * float(step) / float(max(1, total_steps))))
    return float(np.float32(float(lo) + span * c))


class DataParallelTrainer:
    def __init__(self, net, group=None):
        import torch.distributed as dist

        self.net = net
        self.group = group
        self.dist = dist
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0

    # -- collectives ------------------------------------------------------------
    def _sum(self, t):
        if self.world > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t

    def sync_parameters(self, src=0):
        """Every rank takes rank ``src``'s Fourier frequencies and parameters
        (and refreshes its bfloat16 copy)."""
        if self.world > 1:
            self.dist.broadcast(self.net.freq, src=src, group=self.group)
            self.dist.broadcast(self.net.params, src=src, group=self.group)
        if hasattr(self.net, "sync_bf16"):
            self.net.sync_bf16()

    def set_normalisation(self, local_target):
        """Per-output mean and (population) standard deviation over all ranks'
        targets (n_r, n_out), set on the network; the same values as
        ``TailNet.set_normalisation`` on the concatenated targets, up to the
        order of the sums."""
        t = np.asarray(local_target, np.float64)
        O = t.shape[1]
        acc = torch.zeros(1 + O, dtype=torch.float64, device=self._device())
        acc[0] = t.shape[0]
        acc[1:1 + O] = torch.from_numpy(t.sum(0))
        self._sum(acc)
        n = float(acc[0])
        mean = (acc[1:1 + O] / n).cpu().numpy()
        dev = torch.zeros(O, dtype=torch.float64, device=self._device())
        dev[:] = torch.from_numpy(((t - mean) ** 2).sum(0))
        self._sum(dev)
        sd = np.sqrt(dev.cpu().numpy() / n)
        self.net.shift = mean
        self.net.scale = np.where(sd > 0, sd, 1.0)
        return int(n)

    def _device(self):
        return self.net.params.device

    # -- steps ------------------------------------------------------------------
    def step(self, x, target, step, total_steps, lr_max=2e-3, lr_min=2e-5):
        """One data-parallel Adam step on this rank's batch (x (b, 7), target
        (b, n_out) normalised, on the network's device); returns the mean
        loss over all ranks' rows."""
        rows = torch.tensor([float(x.shape[0])], dtype=torch.float64, device=self._device())
        self._sum(rows)
        n_total = float(rows[0])
        loss, grad = self.net.loss_grad(x, target)
        # mean over local rows -> sum over local rows -> mean over all rows
        grad.mul_(float(x.shape[0]))
        self._sum(grad)
        grad.div_(n_total)
        lsum = torch.tensor([loss * float(x.shape[0])], dtype=torch.float64, device=self._device())
        self._sum(lsum)
        self.net.step = int(step)
        self.net.adam(cosine_lr(step, total_steps, lr_max, lr_min))
        return float(lsum[0]) / n_total

    def fit(self, x, target, steps, batch, lr_max=2e-3, lr_min=2e-5, first_step=0, total_steps=None):
        """``steps`` data-parallel steps over this rank's rows: x (n, 7) on the
        network's device, target (n, n_out) in physical units (host or
        device).  ``batch``: rows per rank and step; n is trimmed to a
        multiple of it.  Sets the normalisation from all ranks' targets first
        (when ``first_step`` is 0).  Returns the per-step mean losses."""
        t = target.detach().cpu().numpy() if isinstance(target, torch.Tensor) else np.asarray(target)
        n = (x.shape[0] // batch) * batch
        if n == 0:
            raise ValueError(f"need at least {batch} rows per rank")
        if first_step == 0:
            self.set_normalisation(t[:n])
        tn = torch.from_numpy(((t[:n] - self.net.shift) / self.net.scale).astype(np.float32)).to(self._device())
        xs = x[:n].contiguous()
        nb = n // batch
        total = int(total_steps if total_steps is not None else first_step + steps)
        losses = []
        for k in range(first_step, first_step + int(steps)):
            r0 = (k % nb) * batch
            losses.append(self.step(xs[r0:r0 + batch], tn[r0:r0 + batch], k, total, lr_max, lr_min))
        self.net.step = first_step + int(steps)
        return np.asarray(losses)
