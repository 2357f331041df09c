"""The reference's testcorrectness/test_synapses_vs_connection.py:16-105
restated: a SpikeGeneratorGroup drives half of a group through a
Connection (plain, constant delay, or a DelayConnection with per-pair
delays) and the other half through Synapses ('v+=w') with the same weights
and delays; the two halves' voltage traces must be equal bit for bit.  It
pins when the synaptic code runs: in the 'synapses' slot of the step in
which the queue row comes due (network.py:365-380), right after the
connections."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms
from brian_b200.network import engine

N = 10


def _traces(tab, mode):
    b.clear()
    b.reinit_default_clock()
    spikes = [(i, i * ms) for i in range(N)]
    source = b.SpikeGeneratorGroup(N, spikes)
    targets = b.NeuronGroup(2 * N, model="dv/dt = -v / (1 * ms) : 1", threshold=10, reset=0)
    target_syn, target_conn = targets[:N], targets[N:]
    if mode == "none":
        duration = (N + 1) * ms
        conn = b.Connection(source, target_conn)
        conn.connect_one_to_one(source, target_conn, weight=1.1)
        syn = b.Synapses(source, target_syn, model="w:1", pre="v+=w")
        syn.connect_one_to_one(source, target_syn)
        syn.w = 1.1
    elif mode == "constant":
        delay = 5 * ms
        duration = (N + 1) * ms + delay
        conn = b.Connection(source, target_conn, delay=delay)
        conn.connect_one_to_one(source, target_conn, weight=1.1)
        syn = b.Synapses(source, target_syn, model="w:1", pre="v+=w", max_delay=delay)
        syn.connect_one_to_one(source, target_syn)
        syn.w = 1.1
        syn.delay = delay
    else:
        flat = np.array([i * ms for i in range(N)])
        delays = np.eye(N) * flat
        duration = (N + 1) * ms + delays.max()
        conn = b.Connection(source, target_conn, delay=True, max_delay=flat.max())
        conn.connect_one_to_one(source, target_conn, weight=1.1, delay=delays)
        syn = b.Synapses(source, target_syn, model="w:1", pre="v+=w", max_delay=flat.max())
        syn.connect_one_to_one(source, target_syn)
        syn.w = 1.1
        syn.delay = flat
    mon = b.StateMonitor(targets, "v", record=True)
    net = b.Network(source, targets, conn, syn, mon)
    if tab is None:
        net.run(duration)
        return mon.values
    with engine(tab):
        net.run(duration)
        return mon.values


def _check(v):
    assert np.any(v[:N] != 0)
    for i in range(N):
        assert np.array_equal(v[i], v[N + i]), i


@pytest.mark.parametrize("mode", ["none", "constant", "variable"])
def test_synapses_equal_connection_oracle(oracle_table, mode):
    _check(_traces(oracle_table, mode))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["none", "constant", "variable"])
def test_synapses_equal_connection_gpu(gpu_table, mode):
    _check(_traces(None, mode))
