"""Data-parallel training of the proposal network (brian_b200/dp.py).

CPU: two gloo ranks, each a network copy whose gradients come from the FP64
oracle (oracle/mlp.py) and whose Adam is a float32 restatement, train on
halves of each global batch: the two copies stay equal bit for bit, and
they match one process training on the whole global batch to float
rounding.  GPU: with one rank the data-parallel steps equal bg_mlp_train
bit for bit; two ranks on one GPU (gloo all-reduce through host memory)
keep equal copies and match one process on the global batch."""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
YDIM = 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _data(n, seed=3):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, 64)).astype(np.float32), rng.uniform(-1, 1, (n, YDIM)).astype(np.float32)


def _params(seed=4):
    import oracle.mlp as om
    return om.init_params(np.random.default_rng(seed), YDIM)


class OracleWorker(object):
    """A network copy on the host: oracle gradients, float32 Adam with the
    device's constants and the trained rows of the output layer."""

    def __init__(self, P, X, Y):
        self.P = [(W.astype(np.float32).copy(), b.astype(np.float32).copy()) for W, b in P]
        self.m = [(np.zeros_like(W), np.zeros_like(b)) for W, b in self.P]
        self.v = [(np.zeros_like(W), np.zeros_like(b)) for W, b in self.P]
        self.X, self.Y, self.rows, self.t = X, Y, len(X), 0

    def epoch_order(self, seed, epoch):
        self.perm = np.random.Generator(np.random.PCG64([seed, epoch])).permutation(self.rows)

    def step_gradients(self, batch, row0):
        import oracle.mlp as om
        idx = self.perm[row0:row0 + batch]
        loss, dW, db, _ = om.gradients(self.P, self.X[idx], self.Y[idx], YDIM)
        flat = np.concatenate([np.concatenate([dW[l].ravel(), db[l]]) for l in range(4)]).astype(np.float32)
        return float(loss), flat

    def as_tensor(self, g):
        import torch
        return torch.from_numpy(g)

    def apply_gradients(self, g, lr, scale):
        self.t += 1
        b1, b2, eps = np.float32(0.9), np.float32(0.999), np.float32(1e-8)
        c1, c2 = np.float32(1) - b1 ** np.float32(self.t), np.float32(1) - b2 ** np.float32(self.t)
        off = 0
        for l in range(4):
            rows_train = 2 * YDIM if l == 3 else self.P[l][0].shape[0]
            for k in range(2):
                p, m, v = self.P[l][k], self.m[l][k], self.v[l][k]
                gk = g[off:off + p.size].reshape(p.shape) * np.float32(scale)
                off += p.size
                sl = slice(0, rows_train)
                m[sl] = b1 * m[sl] + (np.float32(1) - b1) * gk[sl]
                v[sl] = b2 * v[sl] + (np.float32(1) - b2) * gk[sl] * gk[sl]
                p[sl] -= np.float32(lr) * (m[sl] / c1) / (np.sqrt(v[sl] / c2) + eps)


def _flat(P):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in P])


def _cpu_rank(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    from brian_b200.dp import train_data_parallel
    X, Y = _data(2048)
    w = OracleWorker(_params(), X, Y)
    losses = train_data_parallel(w, 2, 1024, 1e-3, 11)
    np.savez(os.path.join(out_dir, "r%d.npz" % rank), p=_flat(w.P), losses=losses)
    dist.destroy_process_group()


def test_two_ranks_on_cpu():
    from brian_b200.dp import train_data_parallel
    X, Y = _data(2048)
    whole = OracleWorker(_params(), X, Y)
    want_losses = train_data_parallel(whole, 2, 1024, 1e-3, 11)
    want = _flat(whole.P)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_cpu_rank, args=(2, _free_port(), d), nprocs=2, join=True, start_method="spawn")
        r0, r1 = (np.load(os.path.join(d, "r%d.npz" % r)) for r in range(2))
        assert np.array_equal(r0["p"], r1["p"])                     # the copies stay equal
        moved = np.abs(want - _flat(_params())).max()
        assert moved > 1e-3                                         # training moved the weights
        np.testing.assert_allclose(r0["p"], want, rtol=0, atol=1e-5)
        np.testing.assert_allclose(r0["losses"], want_losses, rtol=0, atol=1e-6)


@pytest.mark.gpu
def test_one_rank_equals_train_on_gpu(gpu_table):
    from brian_b200._lib import MLPHandle
    from brian_b200.dp import ProposalWorker, train_data_parallel
    X, Y = _data(16384)
    hs = []
    for _ in range(2):
        h = MLPHandle(YDIM)
        for l, (W, b) in enumerate(_params()):
            h.set_params(l, W, b)
        h.set_data(X, Y)
        hs.append(h)
    loss_a, _ = hs[0].train(2, 4096, 1e-3, 17)
    loss_b = train_data_parallel(ProposalWorker(hs[1]), 2, 4096, 1e-3, 17)
    for l in range(4):
        for x, y in zip(hs[0].get_params(l), hs[1].get_params(l)):
            assert np.array_equal(x, y), l
    np.testing.assert_allclose(loss_a, loss_b, rtol=1e-6)
    for h in hs:
        h.close()


def _gpu_rank(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    from brian_b200._lib import MLPHandle
    from brian_b200.dp import ProposalWorker, train_data_parallel
    X, Y = _data(16384)
    h = MLPHandle(YDIM)
    for l, (W, b) in enumerate(_params()):
        h.set_params(l, W, b)
    h.set_data(X, Y)
    losses = train_data_parallel(ProposalWorker(h), 2, 8192, 1e-3, 17)
    np.savez(os.path.join(out_dir, "r%d.npz" % rank), p=_flat([h.get_params(l) for l in range(4)]), losses=losses)
    h.close()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_on_one_gpu(gpu_table):
    from brian_b200._lib import MLPHandle
    from brian_b200.dp import ProposalWorker, train_data_parallel
    X, Y = _data(16384)
    h = MLPHandle(YDIM)
    for l, (W, b) in enumerate(_params()):
        h.set_params(l, W, b)
    h.set_data(X, Y)
    want_losses = train_data_parallel(ProposalWorker(h), 2, 8192, 1e-3, 17)
    want = _flat([h.get_params(l) for l in range(4)])
    h.close()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gpu_rank, args=(2, _free_port(), d), nprocs=2, join=True, start_method="spawn")
        r0, r1 = (np.load(os.path.join(d, "r%d.npz" % r)) for r in range(2))
        assert np.array_equal(r0["p"], r1["p"])
        assert np.abs(want - _flat(_params())).max() > 1e-3
        # local means of 4096 rows summed and halved against the mean of
        # 8192 rows: float32 sums in another order, through Adam's step
        np.testing.assert_allclose(r0["p"], want, rtol=0, atol=2e-4)
        np.testing.assert_allclose(r0["losses"], want_losses, rtol=1e-3)
