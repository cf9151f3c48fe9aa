"""Data-parallel training of the surrogate (pacuda_b200.unweight.train_data_parallel) on two gloo
ranks on the CPU: the host logic (shards, one all-reduce of the gradient per step, the same Adam
step on every rank) with the CPU oracle standing in for the device network, against one process
training on the union of the shards."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import surrogate_oracle as O
from pacuda_b200 import unweight

INPUTS, BATCH, STEPS = 7, 64, 3


class OracleNet:
    """The network's gradient and Adam entry points on the CPU oracle (test infrastructure)."""

    def __init__(self, params):
        self.p = params.astype(np.float32).copy()
        self.m1 = np.zeros_like(self.p)
        self.m2 = np.zeros_like(self.p)
        self.step = 0

    def gradients(self, x, y):
        g, loss = O.gradients(self.p, x.numpy(), y.numpy())
        return torch.from_numpy(g.astype(np.float32)), torch.tensor([loss], dtype=torch.float32)

    def apply_gradients(self, grad, lr):
        self.step += 1
        self.p, self.m1, self.m2 = O.adam(self.p, self.m1, self.m2, grad.numpy().astype(np.float32), np.float32(lr),
                                          self.step, INPUTS)


def _data(seed=3):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (2 * BATCH, INPUTS)).astype(np.float32)
    y = rng.normal(size=2 * BATCH).astype(np.float32)
    p = rng.uniform(-0.1, 0.1, O.param_count()).astype(np.float32)
    p[: O.WIDTH * O.IN].reshape(O.WIDTH, O.IN)[:, INPUTS:] = 0.0
    return x, y, p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    x, y, p = _data()
    shard = slice(rank * BATCH, (rank + 1) * BATCH)
    net = OracleNet(p)
    unweight.train_data_parallel(net, torch.from_numpy(x[shard]), torch.from_numpy(y[shard]), dist, epochs=STEPS,
                                 batch=BATCH, lr=1e-3, lr_end=1e-3)
    np.save(os.path.join(out, f"rank{rank}.npy"), net.p)
    dist.destroy_process_group()


def test_two_ranks_train_like_one_process(tmp_path):
    port = 29500 + os.getpid() % 1000
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    a, b = np.load(tmp_path / "rank0.npy"), np.load(tmp_path / "rank1.npy")
    assert np.array_equal(a, b)  # every rank applies the same averaged gradient
    # one process on the union: each step's gradient is the mean over both shards' points (the
    # ranks' random orders differ within a shard, but a shard is one batch, so the set is the same)
    x, y, p = _data()
    net = OracleNet(p)
    for _ in range(STEPS):
        g0, _ = O.gradients(net.p, x[:BATCH], y[:BATCH])
        g1, _ = O.gradients(net.p, x[BATCH:], y[BATCH:])
        net.apply_gradients(torch.from_numpy(((g0 + g1) / 2).astype(np.float32)), 1e-3)
    assert np.allclose(a, net.p, rtol=0, atol=1e-6)
