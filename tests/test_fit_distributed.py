"""distributed_modelfitting across two gloo ranks on the CPU: each rank
fits its own block of targets (a stand-in fit that reports which targets
and inputs it was given) and every rank ends with all results in target
order."""
import importlib
import os
import socket
import sys
import tempfile

import numpy as np
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, G, out_dir):
    sys.path.insert(0, os.path.dirname(HERE))
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    mf = importlib.import_module("brian_b200.modelfitting")
    calls = []

    def fake_fit(data=None, input=None, **kw):
        trains = mf._split_data(data)
        calls.append((len(trains), kw.get("device"), kw.get("popsize")))
        pos = [{"tau": float(np.mean(t)), "first_input": float(np.asarray(x)[0])} for t, x in zip(trains, input)]
        fit = [float(len(t)) for t in trains]
        if len(pos) == 1:
            return mf.OptimizationResult(pos[0], fit[0], {"rank": rank})
        return mf.OptimizationResult(pos, fit, {"rank": rank})

    mf.modelfitting = fake_fit
    rng = np.random.default_rng(0)
    trains = [np.sort(rng.uniform(0, 1, 3 + j)) for j in range(G)]
    data = [(j, t) for j in range(G) for t in trains[j]]
    inputs = [np.full(10, float(j)) for j in range(G)]
    res = mf.distributed_modelfitting(data=data, input=inputs, popsize=64, maxiter=3)
    np.save(os.path.join(out_dir, "r%d.npy" % rank),
            np.array([[p["tau"], p["first_input"], f] for p, f in zip(res.best_pos, res.best_fit)]))
    np.save(os.path.join(out_dir, "c%d.npy" % rank), np.array(calls))
    dist.destroy_process_group()


def test_two_ranks_gather_in_target_order():
    G, world = 7, 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), G, d), nprocs=world, join=True, start_method="spawn")
        rng = np.random.default_rng(0)
        trains = [np.sort(rng.uniform(0, 1, 3 + j)) for j in range(G)]
        want = np.array([[np.mean(t), float(j), float(len(t))] for j, t in enumerate(trains)])
        for r in range(world):
            np.testing.assert_allclose(np.load(os.path.join(d, "r%d.npy" % r)), want, rtol=0, atol=0)
        c0, c1 = np.load(os.path.join(d, "c0.npy")), np.load(os.path.join(d, "c1.npy"))
        # rank 0: targets 0-2 on device 0; rank 1: targets 3-6 (device from LOCAL_RANK, 0 when unset)
        assert c0.tolist() == [[3, 0, 64]] and c1.tolist() == [[4, 0, 64]]
