"""The multi-process paths on the CPU with gloo, world size 2: data-parallel
training of the warm-start network (watersim-v1_b200/dp_train.py) against a
fake solver with the same interface, and bench.py's max-over-ranks timing.
No GPU is involved: the fake solver keeps its weights and gradients in torch
CPU tensors, a linear least-squares model standing in for the network."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "watersim-v1_b200"))
sys.path.insert(0, ROOT)

NW, NPAIR = 12, 40


def _data(rank):
    rng = np.random.default_rng(100 + rank)
    X = rng.standard_normal((NPAIR, NW))
    y = X @ np.linspace(-1, 1, NW) + 0.1 * rng.standard_normal(NPAIR) + rank
    return X, y


class FakeSolver:
    """unet_* interface over a linear model: loss per pair (x.w - y/G)^2."""

    def __init__(self, rank, seed=5):
        self.X, self.y = _data(rank)
        self.w = torch.tensor(np.random.default_rng(seed).standard_normal(NW) * 0.1)
        self.g = torch.zeros(NW, dtype=torch.float64)
        self.m = np.zeros(NW)
        self.v = np.zeros(NW)
        self.step = 0
        self.gain = 0.0

    def unet_train(self, steps, batch, lr, seed):
        assert steps == 0
        self.gain = float(np.sqrt(np.mean(self.y ** 2)))

    def unet_info(self):
        return {"gain": self.gain}

    def unet_set_gain(self, g):
        self.gain = g

    def unet_accumulate(self, samples, seed):
        idx = np.random.default_rng(seed).integers(0, NPAIR, samples)
        w = self.w.numpy()
        r = self.X[idx] @ w - self.y[idx] / self.gain
        self.g.copy_(torch.from_numpy(2 * (r[:, None] * self.X[idx]).sum(0)))
        return float((r ** 2).sum())

    def unet_grads(self):
        return self.g

    def unet_apply(self, lr, total):
        self.step += 1
        g = self.g.numpy() / total
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.999 * self.v + 0.001 * g * g
        mh, vh = self.m / (1 - 0.9 ** self.step), self.v / (1 - 0.999 ** self.step)
        self.w -= torch.from_numpy(lr * mh / (np.sqrt(vh) + 1e-8))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import dp_train
        import bench
        fs = FakeSolver(rank)
        G = dp_train.agree_gain(fs)
        loss = dp_train.train_data_parallel(fs, steps=6, batch=3, lr=0.05, seed=9)
        slow = bench.reduce_max(1.0 + rank, "cpu")
        out[rank] = (fs.w.numpy().copy(), G, loss, slow)
    finally:
        dist.destroy_process_group()


def test_data_parallel_training_world2():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    w0, G0, L0, s0 = out[0]
    w1, G1, L1, s1 = out[1]
    np.testing.assert_array_equal(w0, w1)                  # identical replicas
    assert G0 == G1 and L0 == L1
    assert s0 == s1 == 2.0                                 # max over ranks
    # single-process replay: the summed gradients of both ranks' draws
    ranks = [FakeSolver(r) for r in range(world)]
    G = float(np.sqrt(np.mean([np.mean(_data(r)[1] ** 2) for r in range(world)])))
    assert G0 == pytest.approx(G, rel=1e-12)
    ref = FakeSolver(0)
    for fs in ranks:
        fs.gain = G
    ref.gain = G
    for it in range(6):
        total = np.zeros(NW)
        for r, fs in enumerate(ranks):
            fs.w = ref.w.clone()
            fs.unet_accumulate(3, (9 * 1000003 + it * world + r) & 0xffffffff)
            total += fs.g.numpy()
        ref.g.copy_(torch.from_numpy(total))
        ref.unet_apply(0.05, 3 * world)
    np.testing.assert_allclose(w0, ref.w.numpy(), rtol=1e-12, atol=1e-14)
