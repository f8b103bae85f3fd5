"""Data-parallel training of the tail network (world size 2, gloo, CPU).

The trainer's collective logic -- the normalisation reduced over all ranks'
targets, each step's gradient summed over the ranks weighted by their rows,
the same Adam step and learning rate on every rank -- runs here with the
float64 CPU oracle of the network standing in for the GPU kernels (which do
not exist on this host).  Two ranks with half the rows each must end with the
parameters of one process training on the concatenated batches, and both
ranks with the same parameters."""

import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import mlp_oracle as M
from tod_generation_mapbased_beam_b200 import dp_train

DIMS = (8, 16, 2, 3)  # n_freq, width, depth, n_out
ROWS, BATCH, STEPS = 96, 16, 7


class OracleNet:
    """The network of todgpu_mlp_* in float64 numpy (oracle), with the
    attributes the trainer uses."""

    def __init__(self, seed=0):
        F, H, D, O = DIMS
        rng = np.random.default_rng(seed)
        self.freq = torch.from_numpy(rng.standard_normal((F, 7)))
        _, _, n = M.param_offsets(F, H, D, O)
        self.params = torch.from_numpy(rng.uniform(-0.3, 0.3, n))
        self.grad = torch.zeros(n, dtype=torch.float64)
        self.m = np.zeros(n)
        self.v = np.zeros(n)
        self.step = 0
        self.shift = np.zeros(O)
        self.scale = np.ones(O)

    def loss_grad(self, x, target):
        feat = M.features(x.numpy(), self.freq.numpy(), bf16=False)
        loss, g = M.loss_grad(self.params.numpy(), DIMS, feat, target.numpy().astype(np.float64), bf16=False)
        self.grad.copy_(torch.from_numpy(g))
        return loss, self.grad

    def adam(self, lr):
        self.step += 1
        p, self.m, self.v = M.adam_step(self.params.numpy(), self.m, self.v, self.grad.numpy(), self.step, lr)
        self.params.copy_(torch.from_numpy(p))


def _data():
    rng = np.random.default_rng(11)
    th = np.arccos(rng.uniform(-1, 1, ROWS))
    ph = rng.uniform(0, 2 * np.pi, ROWS)
    ps = rng.uniform(0, 2 * np.pi, ROWS)
    x = torch.from_numpy(M.inputs(th, ph, ps))
    target = np.stack([np.sin(3 * th) * np.cos(ph), np.cos(2 * ps) * th, ph * 0.1 + ps * 0.01], -1) * 1e-7
    return x, target


def _shard(rank, world):
    """Rank r's rows: batch k of rank r is rows [k B, (k+1) B) of its half, so
    that the two ranks' k-th batches together are the single process's k-th
    batch of 2 B rows (rows interleaved by batch)."""
    x, t = _data()
    nb = ROWS // (BATCH * world)
    idx = np.concatenate([np.arange(k * BATCH * world + rank * BATCH, k * BATCH * world + (rank + 1) * BATCH)
                          for k in range(nb)])
    return x[idx], t[idx]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        net = OracleNet(seed=rank)  # different starting points: sync_parameters makes them rank 0's
        tr = dp_train.DataParallelTrainer(net)
        tr.sync_parameters()
        x, t = _shard(rank, world)
        losses = tr.fit(x, t, STEPS, BATCH)
        got = [None] * world
        dist.all_gather_object(got, net.params.numpy().copy())
        if rank == 0:
            np.savez(path, params0=got[0], params1=got[1], losses=losses, shift=net.shift, scale=net.scale)
    finally:
        dist.destroy_process_group()


def test_two_rank_steps_equal_one_rank_on_the_concatenated_batches(tmp_path):
    world = 2
    path = str(tmp_path / "dp.npz")
    mp.start_processes(_worker, args=(world, _free_port(), path), nprocs=world, join=True, start_method="spawn")
    res = np.load(path)
    assert np.array_equal(res["params0"], res["params1"])

    # one process, batches of 2 B rows: the k-th is both ranks' k-th batches
    net = OracleNet(seed=0)
    x, t = _data()
    net.shift = t.mean(0)
    sd = t.std(0)
    net.scale = np.where(sd > 0, sd, 1.0)
    tn = torch.from_numpy((t - net.shift) / net.scale)
    nb = ROWS // (2 * BATCH)
    losses = []
    for k in range(STEPS):
        r0 = (k % nb) * 2 * BATCH
        loss, _ = net.loss_grad(x[r0:r0 + 2 * BATCH], tn[r0:r0 + 2 * BATCH].float())
        losses.append(loss)
        net.step = k
        net.adam(dp_train.cosine_lr(k, STEPS, 2e-3, 2e-5))
    np.testing.assert_allclose(res["shift"], net.shift, rtol=1e-12)
    np.testing.assert_allclose(res["scale"], net.scale, rtol=1e-12)
    np.testing.assert_allclose(res["losses"], losses, rtol=1e-9)
    ref = net.params.numpy()
    assert np.abs(res["params0"] - ref).max() <= 1e-10 * np.abs(ref).max()
    # and training moved the parameters
    assert np.abs(ref - OracleNet(seed=0).params.numpy()).max() > 1e-4


def test_cosine_lr_matches_the_kernel_schedule():
    assert dp_train.cosine_lr(0, 100, 2e-3, 2e-5) == np.float32(2e-3)
    assert abs(dp_train.cosine_lr(100, 100, 2e-3, 2e-5) - 2e-5) < 1e-9
    mid = dp_train.cosine_lr(50, 100, 2e-3, 2e-5)
    assert abs(mid - (2e-5 + (2e-3 - 2e-5) * 0.5)) < 1e-9


def test_single_process_trainer_is_plain_training():
    """Without a process group the trainer is the plain step sequence."""
    net = OracleNet(seed=3)
    x, t = _data()
    tr = dp_train.DataParallelTrainer(net)
    assert tr.world == 1
    tr.fit(x, t, 3, BATCH)
    net2 = OracleNet(seed=3)
    net2.shift, net2.scale = t.mean(0), t.std(0)
    tn = torch.from_numpy(((t - net2.shift) / net2.scale).astype(np.float32))
    for k in range(3):
        net2.loss_grad(x[k * BATCH:(k + 1) * BATCH], tn[k * BATCH:(k + 1) * BATCH])
        net2.step = k
        net2.adam(dp_train.cosine_lr(k, 3, 2e-3, 2e-5))
    np.testing.assert_allclose(net.params.numpy(), net2.params.numpy(), rtol=0, atol=1e-14)
