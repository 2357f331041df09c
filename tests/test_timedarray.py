"""TimedArray / TimedArraySetter (timedarray.py): the array's own semantics
(construction, slicing, calling with a time) as the reference's
testinterface/test_timedarray.py states them, the setter on the oracle
(a parameter that follows the array exactly, on a clock grid, on explicit and
irregular times, per neuron, on a subgroup), and the CUDA engine against the
oracle bit for bit, including a network driven through a TimedArray input."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms, mV, second
from brian_b200.network import engine


def test_construction_and_call():
    ar = np.array([0, 2, 4, 6])

    def check(ta, start, dt):
        for k, v in enumerate(ar):
            assert ta(start + dt * k) == v
        for k, v in enumerate(ar[:-1]):
            assert ta(start + dt * (k + 0.4)) == v

    ta = b.TimedArray(ar)
    assert ta.clock is b.defaultclock
    check(ta, 0.0, b.defaultclock.dt)
    clk = b.Clock(dt=0.25 * ms)
    ta = b.TimedArray(ar, clock=clk)
    assert ta.clock is clk
    check(ta, 0.0, clk.dt)
    check(b.TimedArray(ar, dt=0.5 * ms), 0.0, 0.5 * ms)
    check(b.TimedArray(ar, start=1 * ms, dt=0.5 * ms), 1 * ms, 0.5 * ms)
    with pytest.raises(ValueError):
        b.TimedArray(ar, start=1 * ms, dt=0.5 * ms, clock=b.Clock())
    times = np.arange(len(ar)) * 0.25 * ms
    b.TimedArray(ar, times=times)
    with pytest.raises(ValueError):
        b.TimedArray(ar, times=times, clock=b.Clock())


def test_access():
    ar = np.array([0, 2, 4, 6])
    ta = b.TimedArray(ar)
    assert ta[1] == ar[1]
    assert (ta[:] == ar).all() and (ta.times == ta[:].times).all()
    assert (ta[:2].times == ta.times[:2]).all()
    idx = np.array([0, 2])
    assert (ta[idx] == ar[idx]).all() and (ta[idx].times == ta.times[idx]).all()
    assert (ta(np.arange(len(ar)) * b.defaultclock.dt) == ar).all()
    assert ta(1 * second) == ar[-1]                                  # clamped to the last value
    ar2 = np.array([[0, 1], [2, 3], [4, 5], [6, 7]])
    ta2 = b.TimedArray(ar2)
    assert len(ta2(0 * second)) == 2
    assert (ta2(1 * second) == ar2[-1]).all()
    assert (ta2(np.array([0 * second, 2 * b.defaultclock.dt])) == np.array([ar2[0, 0], ar2[2, 1]])).all()
    import pickle
    tp = pickle.loads(pickle.dumps(b.TimedArray(ar, dt=0.5 * ms)))
    assert (tp == ar).all() and tp._dt == 0.5 * ms and tp(1 * ms) == 4


def _param_group(table, arr_fn, duration=5 * ms, n=1, record=(0,), sub=None):
    """G with model 'p : 1' whose p follows arr_fn(); StateMonitor of p."""
    b.clear()
    b.reinit_default_clock()
    with engine(table):
        G = b.NeuronGroup(n, model="p : 1")
        target = G if sub is None else G[sub[0]:sub[1]]
        target.p = arr_fn()
        mon = b.StateMonitor(G, "p", record=list(record))
        net = b.Network(G, mon)
        net.run(duration)
        out = mon._record()
        net._invalidate()
    return out


def _cases():
    dt = 0.1 * ms
    ar = np.arange(0, 50) * 3.0
    return {
        "clock": (lambda: b.TimedArray(ar), ar),
        "times": (lambda: b.TimedArray(ar, times=np.arange(50) * dt), ar),
        "irregular": (lambda: b.TimedArray(np.array([1.0, 5.0]), times=np.array([0 * ms, 3 * ms])),
                      np.where(np.arange(50) * dt < 3 * ms, 1.0, 5.0)),
        "start_dt": (lambda: b.TimedArray(ar[:20], start=0 * second, dt=0.25 * ms * 0.4), np.r_[ar[:20], [ar[19]] * 30]),
        "offset": (lambda: b.TimedArray(ar[:30], start=1 * ms, dt=dt), None),
    }


@pytest.mark.parametrize("case", ["clock", "times", "irregular", "start_dt", "offset"])
def test_setter_on_oracle(oracle_table, case):
    make, want = _cases()[case]
    steps, vals = _param_group(oracle_table, make)
    assert len(steps) == 50
    if want is not None:
        np.testing.assert_array_equal(vals[:, 0], want)
    else:
        # a setter on a clock that starts at 1 ms: p stays 0 before it, then
        # follows the array (row 0 at 1 ms)
        np.testing.assert_array_equal(vals[:10, 0], 0.0)
        np.testing.assert_array_equal(vals[10:40, 0], np.arange(30) * 3.0)


def test_setter_per_neuron_and_subgroup(oracle_table):
    ar = np.arange(40 * 3, dtype=float).reshape(40, 3)
    steps, vals = _param_group(oracle_table, lambda: b.TimedArray(ar), duration=4 * ms, n=5, record=range(5),
                               sub=(1, 4))
    np.testing.assert_array_equal(vals[:, 1:4], ar)
    np.testing.assert_array_equal(vals[:, [0, 4]], 0.0)


def _driven(table, steps=3000, seed=5, precision=64):
    """20 LIF neurons whose input current I (a parameter) follows a noisy
    TimedArray of 1500 samples on the default clock, one value for all; a
    second group of 10 gets one column per neuron on explicit times."""
    b.clear()
    b.reinit_default_clock()
    rng = np.random.Generator(np.random.PCG64(seed))
    eqs = b.Equations("dv/dt = (I - v)/tau : volt\nI : volt", tau=10 * ms)
    with engine(table):
        G = b.NeuronGroup(20, model=eqs, threshold=-50 * mV, reset=-70 * mV)
        G.v = -70 * mV
        G.I = b.TimedArray(-60 * mV + 30 * mV * rng.random(1500))
        H = b.NeuronGroup(10, model=eqs, threshold=-50 * mV, reset=-70 * mV)
        H.v = -65 * mV
        tt = np.sort(rng.uniform(0, 0.4, 60))
        H.I = b.TimedArray(-70 * mV + 35 * mV * rng.random((60, 10)), times=tt)
        M, MH = b.SpikeMonitor(G), b.SpikeMonitor(H)
        S = b.StateMonitor(G, "v", record=[0, 7, 19])
        net = b.Network(G, H, M, MH, S)
        net.run(steps // 2 * 0.1 * ms)
        net.run(steps // 2 * 0.1 * ms)
        out = {"spk": M._record(), "spkH": MH._record(), "v": S._record()[1], "G.v": np.array(G.v),
               "H.v": np.array(H.v), "G.I": np.array(G.I), "H.I": np.array(H.I)}
        net._invalidate()
    return out


def test_driven_network_on_oracle(oracle_table):
    r = _driven(oracle_table)
    assert len(r["spk"][1]) > 50 and len(r["spkH"][1]) > 20


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["clock", "times", "irregular", "start_dt", "offset"])
def test_setter_gpu_equals_oracle(oracle_table, gpu_table, case):
    make, _ = _cases()[case]
    a = _param_group(oracle_table, make)
    g = _param_group(gpu_table, make)
    for x, y in zip(a, g):
        np.testing.assert_array_equal(x, y)


@pytest.mark.gpu
def test_driven_network_bit_exact(oracle_table, gpu_table):
    ref = _driven(oracle_table)
    got = _driven(gpu_table)
    for k in ref:
        x, y = (ref[k], got[k])
        if isinstance(x, tuple):
            for xx, yy in zip(x, y):
                np.testing.assert_array_equal(xx, yy, err_msg=k)
        else:
            np.testing.assert_array_equal(x, y, err_msg=k)
