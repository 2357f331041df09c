"""Synapses with code (synapses.py:149-330, 400-510): event-driven traces
(`dx/dt = -x/tau : 1 (event-driven)`), presynaptic code that changes
synaptic and postsynaptic variables, postsynaptic code, lastupdate.

On the oracle: the STDP pairing rule as known answers worked out from the
equations (a pre spike 5 ms before a post spike potentiates by
dApre exp(-5 ms/taupre); the reverse order depresses by dApost exp(-5 ms /
taupost)), to within one ulp of numpy's exp.  On the GPU: a Poisson-driven
network with per-synapse delays, STDP in Synapses and two runs (weights
changed between them) equals the oracle bit for bit (spikes, states,
synaptic variables)."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms, mV
from brian_b200.network import engine

TAUPRE = TAUPOST = 20 * ms
WMAX = 0.01
DAPRE = 0.01 * WMAX
DAPOST = -1.05 * DAPRE
MODEL = """w : 1
dApre/dt = -Apre/taupre : 1 (event-driven)
dApost/dt = -Apost/taupost : 1 (event-driven)"""


def _pair(table, t_pre, t_post, w0=0.005):
    b.clear()
    b.reinit_default_clock()
    taupre, taupost, wmax, dApre, dApost = TAUPRE, TAUPOST, WMAX, DAPRE, DAPOST
    with engine(table):
        P = b.SpikeGeneratorGroup(1, [(0, t_pre)])
        Q = b.SpikeGeneratorGroup(1, [(0, t_post)])
        S = b.Synapses(P, Q, model=MODEL, pre="Apre += dApre; w = clip(w + Apost, 0, wmax)",
                       post="Apost += dApost; w = clip(w + Apre, 0, wmax)")
        S[:, :] = True
        S.w = w0
        net = b.Network(P, Q, S)
        net.run(30 * ms)
        out = float(np.array(S.w)[0]), float(np.array(S.Apre)[0]), float(np.array(S.Apost)[0]), \
            float(np.array(S.lastupdate)[0])
        net._invalidate()
    return out


def test_pairing_known_answers(oracle_table):
    w, apre, apost, lu = _pair(oracle_table, 10 * ms, 15 * ms)
    dt = 1e-4
    want = 0.005 + DAPRE * np.exp(-(150 * dt - 100 * dt) / TAUPRE)
    assert w == pytest.approx(want, rel=1e-15, abs=0)
    assert apost == DAPOST and lu == 150 * dt
    w, apre, apost, lu = _pair(oracle_table, 15 * ms, 10 * ms)
    want = 0.005 + DAPOST * np.exp(-(150 * dt - 100 * dt) / TAUPOST)
    assert w == pytest.approx(want, rel=1e-15, abs=0)
    assert apre == DAPRE and lu == 150 * dt
    # weights stay in [0, wmax]
    w, *_ = _pair(oracle_table, 10 * ms, 15 * ms, w0=WMAX)
    assert w == WMAX


def test_unsupported_code_is_refused(oracle_table):
    b.clear()
    P = b.NeuronGroup(2, model="v : 1")
    with pytest.raises(NotImplementedError):
        b.Synapses(P, P, model="w : 1", post="v_post += w")
    with pytest.raises(ValueError):
        b.Synapses(P, P, model="w : 1", pre="v_pre += w")
    with pytest.raises(NotImplementedError):
        b.Synapses(P, P, model="dx/dt = -x/(10*ms) : 1", pre="v += x")


def _network(table, steps=(1500, 1000), seed=9):
    b.clear()
    b.reinit_default_clock()
    rng = np.random.Generator(np.random.PCG64(seed))
    np.random.seed(seed)                    # connect_random draws from numpy's global generator
    taupre, taupost, wmax, dApre, dApost = TAUPRE, TAUPOST, WMAX, DAPRE, DAPOST
    with engine(table):
        inp = b.PoissonGroup(60, rates=rng.uniform(10, 40, 60), seed=seed)
        eqs = b.Equations("dv/dt=(ge-(v+70*mV))/(10*ms) : volt\ndge/dt=-ge/(5*ms) : volt")
        out = b.NeuronGroup(12, model=eqs, threshold=-54 * mV, reset=-70 * mV)
        out.v = -70 * mV + 10 * mV * rng.random(12)
        S = b.Synapses(inp, out, model=MODEL, pre="ge += w*0.8; Apre += dApre; w = clip(w + Apost, 0, wmax)",
                       post="Apost += dApost; w = clip(w + Apre, 0, wmax)", max_delay=3 * ms)
        S.connect_random(inp, out, 0.7)
        S.w = rng.uniform(0, WMAX, len(S))
        S.delay = rng.integers(0, 30, len(S)) * 0.1 * ms
        M = b.SpikeMonitor(out)
        net = b.Network(inp, out, S, M)
        net.run(steps[0] * 0.1 * ms)
        w = np.array(S.w)
        S.w[:10] = w[:10] * 0.5
        net.run(steps[1] * 0.1 * ms)
        r = {"spk": M._record(), "v": np.array(out.v), "ge": np.array(out.ge)}
        for n in ("w", "Apre", "Apost", "lastupdate"):
            r[n] = np.array(getattr(S, n))
        net._invalidate()
    return r


def test_network_on_oracle(oracle_table):
    r = _network(oracle_table)
    assert len(r["spk"][1]) > 100
    assert np.any(r["w"] == 0) or np.any(r["w"] == WMAX) or np.ptp(r["w"]) > 0


@pytest.mark.gpu
def test_network_gpu_equals_oracle(oracle_table, gpu_table):
    ref = _network(oracle_table)
    got = _network(gpu_table)
    for k in ref:
        if isinstance(ref[k], tuple):
            for x, y in zip(ref[k], got[k]):
                np.testing.assert_array_equal(x, y, err_msg=k)
        else:
            np.testing.assert_array_equal(ref[k], got[k], err_msg=k)


@pytest.mark.gpu
def test_pairing_gpu_equals_oracle(oracle_table, gpu_table):
    for t1, t2 in ((10 * ms, 15 * ms), (15 * ms, 10 * ms), (12 * ms, 12 * ms)):
        assert _pair(oracle_table, t1, t2) == _pair(gpu_table, t1, t2)
