"""Spike-history semantics pinned against the reference's own C++
SpikeContainer (brian/utils/ccircular/circular.cpp, compiled from the
reference tree by oracle/build.py into oracle/_ref/).

A SpikeMonitor with a delay on a subgroup reads get_spikes(delay, origin, N)
every step (neurongroup.py:521-533); the oracle's and the reference's answers
must agree spike for spike.  LS[0:period] (the Refractoriness clamp set,
reset.py:311-332) must be the union of the last `period` pushes.
"""
import ctypes as ct

import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms
from brian_b200.network import engine


def _ref():
    import oracle
    lib = oracle.reference_spike_container()
    if lib is None:
        pytest.skip("reference SpikeContainer not built (reference tree absent)")
    return lib


def _gen_spikes(rng, n, steps, p):
    out = []
    for t in range(steps):
        idx = np.nonzero(rng.random(n) < p)[0]
        out.append(idx)
    return out


@pytest.mark.parametrize("delay,origin,size", [(0, 0, 50), (3, 10, 25), (7, 31, 19)])
def test_delayed_subgroup_spikes_match_reference_container(oracle_table, delay, origin, size):
    lib = _ref()
    rng = np.random.Generator(np.random.PCG64(delay * 100 + origin))
    n, steps = 50, 120
    spikes = _gen_spikes(rng, n, steps, 0.15)
    depth = delay + 2
    h = lib.ref_sc_create(depth)
    want = []
    buf = (ct.c_long * n)()
    for t in range(steps):
        arr = (ct.c_long * max(1, len(spikes[t])))(*[int(i) for i in spikes[t]])
        lib.ref_sc_push(h, arr, len(spikes[t]))
        k = lib.ref_sc_get_spikes(h, delay, origin, size, buf, n)
        want += [(t, int(buf[j])) for j in range(k)]
    lib.ref_sc_destroy(h)
    # mid-step times: the generator fires at step ceil(t/dt) (directcontrol.py:233)
    pairs = [(int(i), (t - 0.5) * 0.1 * ms) for t in range(steps) for i in spikes[t]]
    with engine(oracle_table):
        G = b.SpikeGeneratorGroup(n, pairs)
        M = b.SpikeMonitor(G[origin:origin + size], delay=(delay + 0.5) * 0.1 * ms)
        b.Network(G, M).run(steps * 0.1 * ms)
        s, i = M._record()
    got = list(zip(s.tolist(), i.tolist()))
    assert got == want


def test_refractory_window_is_union_of_recent_pushes():
    lib = _ref()
    rng = np.random.Generator(np.random.PCG64(5))
    n, period = 40, 6
    h = lib.ref_sc_create(period + 2)
    hist = []
    buf = (ct.c_long * (n * period))()
    for t in range(60):
        sp = np.nonzero(rng.random(n) < 0.1)[0]
        hist.append(set(sp.tolist()))
        arr = (ct.c_long * max(1, len(sp)))(*[int(i) for i in sp])
        lib.ref_sc_push(h, arr, len(sp))
        k = lib.ref_sc_getslice(h, 0, period, buf, n * period)
        got = sorted(buf[j] for j in range(k))
        want = sorted(i for s in hist[-period:] for i in s)
        assert got == want
    lib.ref_sc_destroy(h)
