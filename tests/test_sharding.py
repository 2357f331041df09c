"""Column-sharded STDP scale-up over two gloo ranks on the CPU (the oracle
engine on each rank): the gathered weights, spikes, traces and states equal
the single-process run of the whole network bit for bit."""
import os
import socket
import sys
import tempfile

import numpy as np
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
KW = dict(seed=31, nin=300, nout=50, rate_lo=100.0, rate_hi=500.0)
STEPS = 400


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, os.path.dirname(HERE))
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    import oracle
    import brian_b200 as b
    from brian_b200.network import engine
    from brian_b200.sharding import stdp_scaleup_sharded
    b.clear()
    with engine(oracle.table()):
        res = stdp_scaleup_sharded(STEPS, **KW)
    np.savez(os.path.join(out_dir, "r%d.npz" % rank), **{k: v for k, v in res.items() if k != "world_size"})
    dist.destroy_process_group()


def _whole():
    import oracle
    import brian_b200 as b
    from brian_b200 import workloads
    from brian_b200.network import engine
    b.clear()
    b.reinit_default_clock()
    with engine(oracle.table()):
        d = workloads.stdp_scaleup(spike_record=KW["nout"], **KW)
        d["net"].run(STEPS * 1e-4)
        a_pre, a_post = d["stdp"]._traces()
        s, i = d["M"]._record()
        out = {"W": d["C"]._weights().reshape(KW["nin"], KW["nout"]).copy(), "steps": s.copy(),
               "idx": i.astype(np.int64), "A_pre": a_pre.copy(), "A_post": a_post.copy(),
               "v": np.array(d["outputs"].v)}
        d["net"]._invalidate()
    return out


def test_two_ranks_equal_whole_network():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d), nprocs=world, join=True, start_method="spawn")
        want = _whole()
        assert len(want["idx"]) > 500 and np.any(want["W"] != want["W"][0, 0])
        for r in range(world):
            got = np.load(os.path.join(d, "r%d.npz" % r))
            for k in want:
                assert np.array_equal(got[k], want[k]), (r, k)


def test_shard_ranges_partition():
    from brian_b200.sharding import shard_range
    for n in (1, 7, 4096):
        for w in (1, 2, 3, 8):
            r = [shard_range(n, k, w) for k in range(w)]
            assert r[0][0] == 0 and r[-1][1] == n and all(a[1] == b_[0] for a, b_ in zip(r, r[1:]))
