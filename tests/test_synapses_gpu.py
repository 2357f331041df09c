"""Synapses on the GPU: the known answers and bit-exact parity with the
oracle (spikes, states, state monitors)."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200.network import engine

import scenarios
import test_synapses_oracle as kat


def _both(fn, oracle_table, **kw):
    out = []
    for tab in (oracle_table, None):
        b.clear()
        b.reinit_default_clock()
        np.random.seed(1234)
        if tab is None:
            out.append(fn(**kw))
        else:
            with engine(tab):
                out.append(fn(**kw))
    return out


@pytest.mark.gpu
def test_known_answers_gpu(gpu_table):
    kat._fresh()
    steps, v = kat._kat(gpu_table)
    v0, v1 = kat.expected_known_answer()
    np.testing.assert_array_equal(v[:, 0], v0)
    np.testing.assert_array_equal(v[:, 1], v1)
    kat._fresh()
    np.testing.assert_array_equal(kat.kat_insertion_order(gpu_table), kat.expected_insertion_order())


@pytest.fixture(params=[None, True, False], ids=["by-size", "events", "pull"])
def delivery(request):
    """The Synapses delivery the engine picks by size (the pull for most of
    these networks, the persistent kernel for Synapses for those of its
    shape), the event path forced, and the pull forced."""
    b.set_global_preferences(synapse_events=request.param)
    yield request.param
    b.set_global_preferences(synapse_events=None)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(runs=2), dict(two_statements=False, multi=False),
                                dict(N=6000, p=0.01, steps=1500)])
def test_synapses_bit_exact(oracle_table, gpu_table, kw, delivery):
    ref, gpu = _both(scenarios.synapses_cuba, oracle_table, **kw)
    assert len(ref["spk0.idx"]) > 100
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
def test_synapse_weights_changed_between_runs(oracle_table, gpu_table, delivery):
    def fn():
        from brian_b200 import ms, mV
        G = b.NeuronGroup(300, model="dv/dt = -v/(10*ms) : volt", threshold=-50 * mV, reset=-60 * mV)
        src = b.PoissonGroup(200, rates=40.0, seed=3)
        S = b.Synapses(src, G, model="w : volt", pre="v += w")
        S.connect_random(sparseness=0.2)
        S.w = 0.5 * mV
        S.delay = "rand() * 2*ms"
        M = b.SpikeMonitor(G)
        St = b.StateMonitor(G, "v", record=[0, 5])
        net = b.Network(src, G, S, M, St)
        net.run(20 * ms)
        S.w = "w * (1 + (i % 3))"
        net.run(20 * ms)
        return scenarios._result(net, groups=[G], spikemons=[M], statemons=[St])
    ref, gpu = _both(fn, oracle_table)
    assert len(ref["spk0.idx"]) > 10
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("rate,sparseness,delay", [(200.0, 0.6, "rand() * 2*ms"), (40.0, 1.0, "1*ms")])
def test_synapses_event_bins_and_pull_fallback(oracle_table, gpu_table, rate, sparseness, delay, delivery):
    """Dense, busy synapses: some steps bring more events to a block of
    targets than its bin holds (and, with one delay for all synapses, every
    source has more than 256 synapses of one delay), so those steps are
    delivered by the pull and the others by the event bins -- equal to the
    oracle bit for bit either way."""
    def fn():
        from brian_b200 import ms, mV
        G = b.NeuronGroup(1200, model="dv/dt = -v/(10*ms) : volt", threshold=5 * mV, reset=0 * mV)
        src = b.PoissonGroup(400, rates=rate, seed=5)
        S = b.Synapses(src, G, model="w : volt", pre="v += w")
        S.connect_random(sparseness=sparseness)
        S.w = "0.01*mV * (1 + (i % 7))"
        S.delay = delay
        M = b.SpikeMonitor(G)
        St = b.StateMonitor(G, "v", record=[0, 700, 1199])
        net = b.Network(src, G, S, M, St)
        net.run(60 * ms)
        return scenarios._result(net, groups=[G], spikemons=[M], statemons=[St])
    ref, gpu = _both(fn, oracle_table)
    assert len(ref["spk0.idx"]) > 100
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(runs=3, steps=2400), dict(multi=False, N=5000, p=0.01, steps=1200),
                                dict(multi=False, N=40000, p=0.001, steps=600)])
def test_synapses_persistent_kernel(oracle_table, gpu_table, kw):
    """One group with Synapses onto itself (one statement each) on the event
    path runs in the persistent kernel for Synapses (one launch per run, one
    grid-wide wait per step): spikes, states and the StateMonitor equal the
    oracle's."""
    b.set_global_preferences(synapse_events=True)
    try:
        ref, gpu = _both(scenarios.synapses_cuba, oracle_table, report_persistent=True, two_statements=False, **kw)
    finally:
        b.set_global_preferences(synapse_events=None)
    assert ref.pop("persistent_threads") == 0 and gpu.pop("persistent_threads") > 0
    assert len(ref["spk0.idx"]) > 100
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("delay", ["1*ms", "rand() * 2*ms"])
def test_synapses_persistent_overflow(oracle_table, gpu_table, delay):
    """The persistent kernel for Synapses on a dense, busy network onto
    itself: every source has 750 synapses, so with one delay a source has
    more than 256 synapses of that delay, and with random delays a step's
    events exceed what a bin holds; those steps are delivered by the pull's
    test inside the same launch.  Spikes, states and the StateMonitor equal
    the oracle's."""
    def fn():
        from brian_b200 import ms, mV
        G = b.NeuronGroup(1500, model="dv/dt = (20*mV - v)/(10*ms) : volt", threshold=10 * mV, reset=0 * mV)
        G.v = np.random.rand(1500) * 10 * mV
        S = b.Synapses(G, G, model="w : volt", pre="v += w")
        S.connect_random(sparseness=0.5)
        S.w = "0.002*mV * (1 + (i % 7))"
        S.delay = delay
        M = b.SpikeMonitor(G)
        St = b.StateMonitor(G, "v", record=[0, 700, 1499])
        net = b.Network(G, S, M, St)
        net.run(30 * ms)
        out = scenarios._result(net, groups=[G], spikemons=[M], statemons=[St])
        out["persistent_threads"] = net.stats().get("persistent_threads", 0)
        return out
    ref, gpu = _both(fn, oracle_table)
    assert ref.pop("persistent_threads") == 0 and gpu.pop("persistent_threads") > 0
    assert len(ref["spk0.idx"]) > 10000
    scenarios.compare(ref, gpu)
