"""Synapses on the oracle and the host side of the class.

The known-answer cases are worked out by hand from the reference's
SpikeQueue (spikequeue.py:209-216 next/peek, 270-302 insert, 340-363
propagate), Synapses.update (synapses.py:808-827) and the schedule
(network.py:365-380: connections, after_connections, synapses, resets): a
spike of step s through a synapse of delay d bins is inserted in the
connections slot at the queue row due d steps later and applied in the
synapses slot of step s + d; the events reaching one target are applied one
after the other in queue order.
"""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms
from brian_b200.network import engine

import scenarios

DT = 1e-4


def _fresh():
    b.clear()
    b.reinit_default_clock()
    np.random.seed(1234)


def _kat(tab, steps=12):
    src = b.SpikeGeneratorGroup(3, [(0, 2 * DT), (1, 2 * DT), (2, 4 * DT), (0, 5 * DT)])
    P = b.NeuronGroup(2, model="v : 1")
    P.v = [1.0, 0.0]
    S = b.Synapses(src, P, model="w : 1", pre="v += w")
    S[0, 0] = True          # synapse 0
    S[1, 0] = True          # synapse 1
    S[2, 1] = 2             # synapses 2, 3
    S.w = [2.0 ** -53, 2.0 ** -52, 0.25, 0.5]
    S.delay[0] = 3 * DT + 1e-9     # int(value/dt) = 3
    S.delay[1] = 3 * DT + 1e-9
    S.delay[2] = 0.0
    S.delay[3] = 1 * DT + 1e-9
    M = b.StateMonitor(P, "v", record=True)
    net = b.Network(src, P, S, M)
    with engine(tab):
        net.run(steps * DT)
        steps_, vals = M._record()
    return np.asarray(steps_), np.asarray(vals).reshape(len(steps_), 2)


def test_known_answer(oracle_table):
    _fresh()
    steps, v = _kat(oracle_table)
    v0 = np.full(12, 1.0)
    # spikes of step 2 through synapses 0 and 1 (delay 3) arrive at step 5,
    # in queue order: source 0 first: (1 + 2^-53) + 2^-52
    x = (1.0 + 2.0 ** -53) + 2.0 ** -52
    v0[5:] = x
    # the second spike of source 0 (step 5) arrives at step 8
    v0[8:] = x + 2.0 ** -53
    v1 = np.zeros(12)
    v1[4:] = 0.25            # step 4, delay 0 -> step 4
    v1[5:] = 0.25 + 0.5      # step 4, delay 1 -> step 5
    np.testing.assert_array_equal(steps, np.arange(12))
    np.testing.assert_array_equal(v[:, 0], v0)
    np.testing.assert_array_equal(v[:, 1], v1)
    # the order matters: applying synapse 1 first gives another value
    assert (1.0 + 2.0 ** -52) + 2.0 ** -53 != x


def kat_insertion_order(tab, steps=10):
    """Source 1 spikes at step 2 through a delay of 3, source 0 at step 4
    through a delay of 1: both events reach target 0 at step 5, the one
    inserted first (source 1) applied first."""
    src = b.SpikeGeneratorGroup(2, [(1, 2 * DT), (0, 4 * DT)])
    P = b.NeuronGroup(1, model="v : 1")
    P.v = 1.0
    S = b.Synapses(src, P, model="w : 1", pre="v += w")
    S[0, 0] = True
    S[1, 0] = True
    S.w = [2.0 ** -52, 2.0 ** -53]
    S.delay[0] = 1 * DT + 1e-9
    S.delay[1] = 3 * DT + 1e-9
    M = b.StateMonitor(P, "v", record=True)
    net = b.Network(src, P, S, M)
    with engine(tab):
        net.run(steps * DT)
        _, vals = M._record()
    return np.asarray(vals).ravel()


def expected_insertion_order(steps=10):
    v = np.full(steps, 1.0)
    v[5:] = (1.0 + 2.0 ** -53) + 2.0 ** -52
    return v


def expected_known_answer():
    v0 = np.full(12, 1.0)
    x = (1.0 + 2.0 ** -53) + 2.0 ** -52
    v0[5:] = x
    v0[8:] = x + 2.0 ** -53
    v1 = np.zeros(12)
    v1[4:] = 0.25
    v1[5:] = 0.25 + 0.5
    return v0, v1


def test_insertion_order(oracle_table):
    _fresh()
    v = kat_insertion_order(oracle_table)
    np.testing.assert_array_equal(v, expected_insertion_order())
    assert (1.0 + 2.0 ** -52) + 2.0 ** -53 != v[-1]


def test_creation_order_and_delays():
    _fresh()
    G = b.NeuronGroup(5, model="v : 1")
    H = b.NeuronGroup(4, model="v : 1")
    S = b.Synapses(G, H, model="w : 1\nu : 1", pre="v += w")
    S[0:2, 1:3] = True
    np.testing.assert_array_equal(S.presynaptic, [0, 0, 1, 1])
    np.testing.assert_array_equal(S.postsynaptic, [1, 2, 1, 2])
    S[4, 0] = 2
    np.testing.assert_array_equal(S.presynaptic[4:], [4, 4])
    S[2:4, :] = "j == i"
    np.testing.assert_array_equal(S.presynaptic[6:], [2, 3])
    np.testing.assert_array_equal(S.postsynaptic[6:], [2, 3])
    S.w = "i + 10*j"
    np.testing.assert_array_equal(S.w[:], S.presynaptic + 10.0 * S.postsynaptic)
    S.delay = 0.25e-3
    assert np.all(S._delay == int(0.25e-3 / b.defaultclock.dt))
    np.testing.assert_array_equal(S.w[0, 1], [10.0])
    assert len(S) == 8


def test_unsupported_forms():
    _fresh()
    G = b.NeuronGroup(5, model="v : 1")
    with pytest.raises(NotImplementedError):
        b.Synapses(G, G, model="w : 1", pre="v += w", post="v_post += w")
    with pytest.raises(NotImplementedError):
        b.Synapses(G, G, model="dw/dt = -w/(5*ms) : 1", pre="v += w")
    with pytest.raises(ValueError):
        b.Synapses(G, G, model="w : 1", pre="v_pre += w")
    S = b.Synapses(G, G, model="w : 1", pre="v += w", max_delay=0.2e-3)
    S[:, :] = True
    S.delay = 0.5e-3
    with pytest.raises(ValueError):
        S._queue_check()


def test_two_runs_continue(oracle_table):
    _fresh()
    with engine(oracle_table):
        one = scenarios.synapses_cuba(N=600, steps=600)
    _fresh()
    with engine(oracle_table):
        two = scenarios.synapses_cuba(N=600, steps=600, runs=2)
    assert len(one["spk0.idx"]) > 50
    scenarios.compare(one, two)


def test_save_load_connectivity(tmp_path):
    _fresh()
    G = b.NeuronGroup(30, model="v : 1")
    S = b.Synapses(G, G, model="w : 1", pre="v += w")
    S.connect_random(sparseness=0.3)
    S.delay = "rand() * 1*ms"
    fn = str(tmp_path / "conn.npz")
    S.save_connectivity(fn)
    T = b.Synapses(G, G, model="w : 1", pre="v += w")
    T.load_connectivity(fn)
    np.testing.assert_array_equal(T.presynaptic, S.presynaptic)
    np.testing.assert_array_equal(T.postsynaptic, S.postsynaptic)
    np.testing.assert_array_equal(T._delay, S._delay)
    assert set(np.load(fn).files) == {"presynaptic", "postsynaptic", "_delay_pre", "_delay_post"}


def test_edge_cases(oracle_table):
    _fresh()
    src = b.SpikeGeneratorGroup(2, [(0, 1 * DT), (1, 2 * DT)])
    P = b.NeuronGroup(6, model="v : 1")
    empty = b.Synapses(src, P, model="w : 1", pre="v += w")            # no synapses at all
    sub = b.Synapses(src, P[2:5], model="w : 1", pre="v -= 2*w")       # a subgroup as target
    sub[0, 1] = True                                                   # -> neuron 3 of P
    sub[1, 2] = True                                                   # -> neuron 4 of P
    sub.w = [0.25, 0.5]
    M = b.StateMonitor(P, "v", record=True)
    net = b.Network(src, P, empty, sub, M)
    with engine(oracle_table):
        net.run(6 * DT)
        _, vals = M._record()
    vals = np.asarray(vals).reshape(6, 6)
    want = np.zeros((6, 6))
    want[1:, 3] = -0.5          # spike of step 1, delay 0 -> applied at step 1
    want[2:, 4] = -1.0          # spike of step 2 -> step 2
    np.testing.assert_array_equal(vals, want)


def test_order_in_network_does_not_matter(oracle_table):
    """Synapses run in their own slot after the connections, wherever they
    sit among the groups (network.py:472-483)."""
    out = []
    for order in ("GSH", "GHS"):
        _fresh()
        G = b.SpikeGeneratorGroup(3, [(0, 1 * DT), (2, 3 * DT)])
        H = b.NeuronGroup(3, model="dv/dt = -v/(2*ms) : 1")
        S = b.Synapses(G, H, model="w : 1", pre="v += w")
        S[:, :] = True
        S.w = "0.1 + i + 10*j"
        M = b.StateMonitor(H, "v", record=True)
        objs = {"G": G, "S": S, "H": H}
        net = b.Network(*[objs[c] for c in order], M)
        with engine(oracle_table):
            net.run(6 * DT)
            out.append(np.asarray(M._record()[1]).copy())
    np.testing.assert_array_equal(out[0], out[1])
    assert np.any(out[0] != 0)
