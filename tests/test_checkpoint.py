"""Checkpoint / resume: run(T1); pickle the network; unpickle; run(T2)
equals run(T1); run(T2) on the network that was never pickled, bit for bit (Network.__reduce__, network.py:652;
SpikeContainer.__reduce__, utils/circular.py:249-269).  The engine's dynamic
state -- delay rings, spike histories, refractory bookkeeping, STDP traces,
counters -- is saved through bg_net_save_state and loaded into the engine
the unpickled network builds."""
import pickle

import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms, mV
from brian_b200.connections import fixed_indegree_csr
from brian_b200.network import engine


def _cuba_delay(monitors=True, refractory=0.0, N=1500):
    eqs = b.Equations("dv/dt=(ge+gi-(v-El))/taum : volt\ndge/dt=-ge/taue : volt\ndgi/dt=-gi/taui : volt",
                      taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    P = b.NeuronGroup(N, model=eqs, threshold=-50 * mV, reset=-60 * mV, refractory=refractory)
    ne = int(0.8 * N)
    rng = np.random.Generator(np.random.PCG64(4))
    objs = [P]
    for src, n, k, w, var, sd in ((P.subgroup(ne), ne, 40, 0.3e-2, "ge", 1), (P.subgroup(N - ne), N - ne, 10,
                                                                             -1.2e-2, "gi", 2)):
        rowptr, cols = fixed_indegree_csr(n, N, k, seed=sd)
        C = b.DelayConnection(src, P, var, max_delay=5 * ms)
        C.connect_csr(rowptr, cols, w, delay_steps=rng.integers(1, 51, size=len(cols)).astype(np.uint8))
        objs.append(C)
    P.v = -60 * mV + rng.random(N) * 11 * mV
    if monitors:
        objs += [b.SpikeMonitor(P), b.StateMonitor(P, "v", record=[0, 5, N - 1])]
    return b.Network(*objs)


def _stdp():
    eqs = b.Equations("dv/dt=(ge*(Ee-vr)+El-v)/taum : volt\ndge/dt=-ge/taue : 1", taum=10 * ms, taue=5 * ms,
                      Ee=0 * mV, vr=-60 * mV, El=-74 * mV)
    rng = np.random.Generator(np.random.PCG64(8))
    inp = b.PoissonGroup(300, rates=rng.uniform(5, 25, 300) * 20, seed=3)
    out = b.NeuronGroup(40, model=eqs, threshold=-54 * mV, reset=-60 * mV)
    out.v = -60 * mV
    C = b.Connection(inp, out, "ge", structure="dense", dtype=np.float32)
    C.connect(W=rng.uniform(0, 0.01, (300, 40)))
    S = b.ExponentialSTDP(C, 20 * ms, 20 * ms, 0.01, -0.0105, wmax=0.01)
    return b.Network(inp, out, C, S, b.SpikeMonitor(out))


def _snapshot(net):
    out = {}
    for k, o in enumerate(net._order):
        if isinstance(o, b.NeuronGroup):
            for v in o._names:
                out["g%d.%s" % (k, v)] = np.array(getattr(o, v))
        elif isinstance(o, b.Connection):
            out["w%d" % k] = o._weights().astype(np.float64).copy()
        elif isinstance(o, b.SpikeMonitor):
            out["spk%d" % k] = tuple(x.copy() for x in o._record())
        elif isinstance(o, b.StateMonitor):
            out["st%d" % k] = tuple(x.copy() for x in o._record())
    for k, s in enumerate(net.stdps):
        out["stdp%d" % k] = tuple(x.copy() for x in s._traces())
    out["clock"] = net.clock._n
    return out


def _equal(a, c):
    assert a.keys() == c.keys()
    for k in a:
        x, y = a[k], c[k]
        if isinstance(x, tuple):
            assert all(np.array_equal(p, q) for p, q in zip(x, y)), k
        else:
            assert np.array_equal(x, y), k


def checkpoint_roundtrip(build, t1, t2, table=None):
    def go():
        b.clear()
        b.reinit_default_clock()
        net = build()
        net.run(t1 * 0.1 * ms)
        net.run(t2 * 0.1 * ms)
        whole = _snapshot(net)
        net._invalidate()
        b.clear()
        b.reinit_default_clock()
        net = build()
        net.run(t1 * 0.1 * ms)
        blob = pickle.dumps(net)
        net._invalidate()
        del net
        b.clear()
        net2 = pickle.loads(blob)
        net2.run(t2 * 0.1 * ms)
        resumed = _snapshot(net2)
        net2._invalidate()
        return whole, resumed
    if table is None:
        return go()
    with engine(table):
        return go()


CASES = {"delay-monitors": (lambda: _cuba_delay(), 317, 450),
         "delay-persistent": (lambda: _cuba_delay(monitors=False), 400, 333),
         "refractory": (lambda: _cuba_delay(refractory=3 * ms), 250, 260),
         "stdp": (_stdp, 300, 400)}


@pytest.mark.parametrize("case", sorted(CASES))
def test_checkpoint_oracle(oracle_table, case):
    build, t1, t2 = CASES[case]
    whole, resumed = checkpoint_roundtrip(build, t1, t2, oracle_table)
    _equal(whole, resumed)


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_checkpoint_gpu(gpu_table, case):
    build, t1, t2 = CASES[case]
    whole, resumed = checkpoint_roundtrip(build, t1, t2)
    _equal(whole, resumed)


def test_state_refused_by_another_network(oracle_table):
    with engine(oracle_table):
        b.clear()
        net = _cuba_delay(N=1500)
        net.run(50 * 0.1 * ms)
        blob = net._binding.rt.save_state()
        net._invalidate()
        b.clear()
        other = _cuba_delay(N=1400)
        other.prepare()
        with pytest.raises(Exception):
            other._binding.rt.load_state(blob)
        other._invalidate()


def _synapses():
    np.random.seed(21)                      # connect_random and rand() draw from numpy's global generator
    G = b.NeuronGroup(300, model="dv/dt = -v/(10*ms) : volt", threshold=5 * mV, reset=0 * mV)
    src = b.PoissonGroup(200, rates=120.0, seed=3)
    S = b.Synapses(src, G, model="w : volt", pre="v += w")
    S.connect_random(sparseness=0.2)
    S.w = "0.2*mV * (1 + (i % 3))"
    S.delay = "rand() * 3*ms"
    return b.Network(src, G, S, b.SpikeMonitor(G), b.StateMonitor(G, "v", record=[0, 7]))


@pytest.mark.parametrize("events", [None, True], ids=["by-size", "events"])
def test_checkpoint_synapses_oracle(oracle_table, events):
    b.set_global_preferences(synapse_events=events)
    try:
        whole, resumed = checkpoint_roundtrip(_synapses, 213, 190, oracle_table)
    finally:
        b.set_global_preferences(synapse_events=None)
    assert len(whole["spk3"][1]) > 100
    _equal(whole, resumed)


@pytest.mark.gpu
@pytest.mark.parametrize("events", [None, True], ids=["by-size", "events"])
def test_checkpoint_synapses_gpu(gpu_table, events):
    """Synapses with delays up to 3 ms resumed 21.3 ms into the run: the
    event path rebuilds the spike lists of the last 30 steps from the loaded
    spike history."""
    b.set_global_preferences(synapse_events=events)
    try:
        whole, resumed = checkpoint_roundtrip(_synapses, 213, 190)
    finally:
        b.set_global_preferences(synapse_events=None)
    assert len(whole["spk3"][1]) > 100
    _equal(whole, resumed)


def _synapses_self():
    """CUBA through Synapses onto its own group (the engine's persistent
    kernel for Synapses when the event path is forced)."""
    np.random.seed(5)
    eqs = b.Equations("dv/dt=(ge+gi-(v-El))/taum : volt\ndge/dt=-ge/taue : volt\ndgi/dt=-gi/taui : volt",
                      taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    N = 2500
    P = b.NeuronGroup(N, model=eqs, threshold=-50 * mV, reset=-60 * mV)
    Pe, Pi = P.subgroup(2000), P.subgroup(500)
    rng = np.random.Generator(np.random.PCG64(6))
    Se = b.Synapses(Pe, P, model="w : volt", pre="ge += w", max_delay=5 * ms)
    Si = b.Synapses(Pi, P, model="w : volt", pre="gi -= w")
    Se.connect_random(sparseness=0.02)
    Si.connect_random(sparseness=0.02)
    Se.w = 1.62 * mV * (0.5 + rng.random(len(Se)))
    Si.w = 9 * mV * (0.5 + rng.random(len(Si)))
    Se.delay = rng.random(len(Se)) * 4 * ms
    Si.delay = rng.random(len(Si)) * 4 * ms
    P.v = -60 * mV + rng.random(N) * 10 * mV
    return b.Network(P, Se, Si, b.SpikeMonitor(P), b.StateMonitor(P, "v", record=[0, 1, N - 1]))


@pytest.mark.gpu
@pytest.mark.parametrize("events", [None, True], ids=["by-size", "events"])
def test_checkpoint_synapses_self_gpu(gpu_table, events):
    """One group with Synapses onto itself (with the event path forced: the
    persistent kernel for Synapses), resumed mid-run from a saved state."""
    b.set_global_preferences(synapse_events=events)
    try:
        whole, resumed = checkpoint_roundtrip(_synapses_self, 237, 180)
    finally:
        b.set_global_preferences(synapse_events=None)
    assert len(whole["spk3"][1]) > 100
    _equal(whole, resumed)
