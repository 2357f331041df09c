"""Failure detection without a GPU fault: a bounded inter-block wait that
runs out (one block of the persistent kernel holds back its arrivals, a flag
nothing else sets), a non-finite state found by the end-of-run scan, and
connection rows refused by the range checks.  Each failure comes back as an
error status with the device still usable."""
import numpy as np
import pytest

import scenarios
import brian_b200 as b
from brian_b200 import ms, mV
from brian_b200._lib import EngineError
from brian_b200.connections import fixed_indegree_csr
from brian_b200.network import engine

BG_EINVAL, BG_ETIMEOUT, BG_ENUMERIC, BG_ESTATE = -1, -4, -5, -6


def _cuba_delay_net(N=6000, seed=3, v0=None):
    eqs = b.Equations("dv/dt=(ge+gi-(v-El))/taum : volt\ndge/dt=-ge/taue : volt\ndgi/dt=-gi/taui : volt",
                      taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    P = b.NeuronGroup(N, model=eqs, threshold=-50 * mV, reset=-60 * mV)
    ne = int(0.8 * N)
    rng = np.random.Generator(np.random.PCG64(seed))
    conns = []
    for src, n, k, w, var, sd in ((P.subgroup(ne), ne, 80, 0.162e-2, "ge", 1), (P.subgroup(N - ne), N - ne, 20,
                                                                               -0.9e-2, "gi", 2)):
        rowptr, cols = fixed_indegree_csr(n, N, k, seed=sd)
        C = b.DelayConnection(src, P, var, max_delay=5 * ms)
        C.connect_csr(rowptr, cols, w, delay_steps=rng.integers(1, 51, size=len(cols)).astype(np.uint8))
        conns.append(C)
    P.v = -60 * mV + rng.random(N) * 10 * mV if v0 is None else v0
    return b.Network(P, *conns), P


@pytest.mark.gpu
def test_bounded_wait_runs_out(oracle_table, gpu_table):
    b.set_global_preferences(spin_limit=20000)
    try:
        net, P = _cuba_delay_net()
        net.prepare(configure=lambda rt: rt.debug_hold_arrival(2))
        assert net.stats()["persistent_threads"] > 0
        with pytest.raises(EngineError) as e:
            net.run(100 * 0.1 * ms)
        assert e.value.code == BG_ETIMEOUT, e.value
        # the network refuses to go on from an inconsistent state
        with pytest.raises(EngineError) as e:
            net.run(10 * 0.1 * ms)
        assert e.value.code == BG_ESTATE
        net._invalidate()
    finally:
        b.set_global_preferences(spin_limit=None)
    # nothing was left running: the device serves the next network, which
    # matches the oracle bit for bit
    out = []
    for tab in (oracle_table, None):
        b.clear()
        b.reinit_default_clock()
        np.random.seed(1234)
        if tab is None:
            out.append(scenarios.cuba_delay(monitors=False, N=6000, steps=500))
        else:
            with engine(tab):
                out.append(scenarios.cuba_delay(monitors=False, N=6000, steps=500))
    for r in out:
        r.pop("launches"), r.pop("persistent_threads")
    scenarios.compare(out[0], out[1])


@pytest.mark.gpu
@pytest.mark.parametrize("persistent", [True, False])
def test_nonfinite_state_reported(gpu_table, persistent):
    v0 = -60 * mV + np.random.default_rng(5).random(6000) * 10 * mV
    v0[1234] = np.nan
    b.set_global_preferences(check_finite=True, persistent=persistent)
    try:
        net, P = _cuba_delay_net(v0=v0)
        with pytest.raises(EngineError) as e:
            net.run(50 * 0.1 * ms)
        assert e.value.code == BG_ENUMERIC
        assert "group 0, variable 0, neuron 1234" in str(e.value)
        net._invalidate()
        # without the check the same network runs (NaN never crosses threshold)
        b.set_global_preferences(check_finite=False)
        b.clear()
        net, P = _cuba_delay_net(v0=v0)
        net.run(50 * 0.1 * ms)
        assert np.isnan(np.asarray(P.v)[1234])
        net._invalidate()
    finally:
        b.set_global_preferences(check_finite=False, persistent=True)


@pytest.mark.gpu
@pytest.mark.parametrize("bad", ["target", "order", "delay"])
def test_connection_rows_refused(gpu_table, bad):
    """Rows with a target beyond the group, targets out of ascending order or
    a delay at the ring depth are refused with BG_EINVAL before any kernel
    reads them."""
    N = 2000
    eqs = b.Equations("dv/dt=(ge-(v-El))/taum : volt\ndge/dt=-ge/taue : volt", taum=20 * ms, taue=5 * ms,
                      El=-49 * mV)
    P = b.NeuronGroup(N, model=eqs, threshold=-50 * mV, reset=-60 * mV)
    rowptr, cols = fixed_indegree_csr(N, N, 10, seed=9)
    cols = cols.copy()
    d = np.ones(len(cols), np.uint8)
    k = int(rowptr[40]) + 3
    if bad == "target":
        cols[k] = N
    elif bad == "order":
        cols[k], cols[k + 1] = cols[k + 1], cols[k]
    else:
        d[k] = 51                           # max_delay 5 ms: 51 ring rows, delays 0..50
    C = b.DelayConnection(P, P, "ge", max_delay=5 * ms)
    with pytest.raises((EngineError, ValueError)) as e:
        # (a delay beyond max_delay is already refused by the Python front end)
        C.connect_csr(rowptr, cols, 0.1e-3, delay_steps=d)
        net = b.Network(P, C)
        net.run(10 * 0.1 * ms)
    if isinstance(e.value, EngineError):
        assert e.value.code == BG_EINVAL, e.value


@pytest.mark.gpu
def test_bounded_wait_runs_out_synapses(oracle_table, gpu_table):
    """The same for the persistent kernel for Synapses: one block holds back
    its arrivals, every wait runs out, the run fails with BG_ETIMEOUT and
    the device runs the next network bit for bit like the oracle."""
    b.set_global_preferences(spin_limit=20000)
    try:
        b.clear()
        b.reinit_default_clock()
        np.random.seed(1234)
        P = b.NeuronGroup(6000, model="dv/dt = (20*mV - v)/(10*ms) : volt", threshold=10 * mV, reset=0 * mV)
        P.v = np.random.rand(6000) * 10 * mV
        S = b.Synapses(P, P, model="w : volt", pre="v += w")
        S.connect_random(sparseness=0.01)
        S.w = 0.01 * mV
        S.delay = "rand() * 2*ms"
        net = b.Network(P, S)
        net.prepare(configure=lambda rt: rt.debug_hold_arrival(2))
        assert net.stats()["persistent_threads"] > 0
        with pytest.raises(EngineError) as e:
            net.run(100 * 0.1 * ms)
        assert e.value.code == BG_ETIMEOUT, e.value
        with pytest.raises(EngineError) as e:
            net.run(10 * 0.1 * ms)
        assert e.value.code == BG_ESTATE
        net._invalidate()
    finally:
        b.set_global_preferences(spin_limit=None)
    out = []
    for tab in (oracle_table, None):
        b.clear()
        b.reinit_default_clock()
        np.random.seed(1234)
        if tab is None:
            out.append(scenarios.synapses_cuba(two_statements=False, steps=500, report_persistent=True))
        else:
            with engine(tab):
                out.append(scenarios.synapses_cuba(two_statements=False, steps=500, report_persistent=True))
    assert out[0].pop("persistent_threads") == 0 and out[1].pop("persistent_threads") > 0
    scenarios.compare(out[0], out[1])
