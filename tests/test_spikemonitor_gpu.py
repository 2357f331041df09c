"""SpikeMonitor on the stepped path (monitor.py:156-166): a group of more
spike-history words than one pass of the monitor kernel covers (8192
words), and monitors on subgroups that start and end inside a word, record
the same spikes in the same order as the oracle."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms
from brian_b200.network import engine


def _run(table, n=300001, steps=40):
    b.clear()
    b.reinit_default_clock()
    rng = np.random.Generator(np.random.PCG64(11))
    prev = b.get_global_preference("persistent")
    b.set_global_preferences(persistent=False)
    try:
        with engine(table):
            P = b.PoissonGroup(n, rates=rng.uniform(20, 200, n), seed=7)
            A, B, C = P.subgroup(7), P.subgroup(n - 12), P.subgroup(5)
            mons = [b.SpikeMonitor(x) for x in (P, A, B, C)]
            net = b.Network(P, *mons)
            net.run(steps // 2 * 0.1 * ms)
            net.run(steps // 2 * 0.1 * ms)
            out = [tuple(np.asarray(v).copy() for v in m._record()) for m in mons]
            net._invalidate()
    finally:
        b.set_global_preferences(persistent=prev)
    return out


def test_subgroup_monitors_on_oracle(oracle_table):
    out = _run(oracle_table, n=20001, steps=20)
    whole = out[0]
    assert len(whole[1]) > 100
    # the subgroups' records are the whole group's, shifted and split
    idx = np.asarray(whole[1])
    assert sum(len(o[1]) for o in out[1:]) == len(idx)


@pytest.mark.gpu
def test_large_group_monitors_gpu_equals_oracle(oracle_table, gpu_table):
    ref = _run(oracle_table)
    got = _run(gpu_table)
    assert len(ref[0][1]) > 10000
    for r, g in zip(ref, got):
        for x, y in zip(r, g):
            np.testing.assert_array_equal(x, y)
