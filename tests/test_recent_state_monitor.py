"""RecentStateMonitor (monitor.py:991-1141) as a ring view over the
records: the same records as a StateMonitor, the reference's ring indexing
(slot r mod num_duration, current_time_index, has_looped) and past values
(current_time_index - 1 - int(invdt*times)) mod num_duration."""
import numpy as np

import brian_b200 as b
from brian_b200 import ms
from brian_b200.network import engine

DT = 1e-4


def _net(tab, steps, duration=1 * ms):
    b.clear()
    b.reinit_default_clock()
    G = b.NeuronGroup(3, model="dv/dt = -v/(10*ms) : 1")
    G.v = [1.0, 2.0, 3.0]
    R = b.RecentStateMonitor(G, "v", duration=duration)
    S = b.StateMonitor(G, "v", record=True)
    net = b.Network(G, R, S)
    with engine(tab):
        net.run(steps * DT)
        return R, S, R.values, R.times, R.current_time_index, R.has_looped, S.values.T, S.times, \
            R.get_past_values(np.array([0.0, 1.5 * DT, 4 * DT])), R[2]


def test_before_and_after_wrap(oracle_table):
    M = int(1 * ms / DT) + 1
    assert M == 11
    R, S, vals, times, cur, looped, full, ftimes, past, v2 = _net(oracle_table, 5)
    assert cur == 5 and not looped
    np.testing.assert_array_equal(vals, full)
    np.testing.assert_array_equal(times, ftimes)
    R, S, vals, times, cur, looped, full, ftimes, past, v2 = _net(oracle_table, 25)
    assert cur == 25 % M and looped
    np.testing.assert_array_equal(vals, full[-M:])
    np.testing.assert_array_equal(times, ftimes[-M:])
    np.testing.assert_array_equal(v2, full[-M:, 2])
    # neuron k looks lag int(times[k]/dt) records back from the last one
    lags = np.array([0.0, 1.5 * DT, 4 * DT]) * (1.0 / DT)
    for k in range(3):
        assert past[k] == full[-1 - int(lags[k]), k]


def test_isi_histogram(oracle_table):
    """ISIHistogramMonitor (monitor.py:430-504): intervals 5 ms -> bin 0,
    15 and 12 ms -> bin 1, 26 ms and the two first spikes (negative
    intervals from the 1000 s start) -> the last bin."""
    b.clear()
    b.reinit_default_clock()
    G = b.SpikeGeneratorGroup(2, [(0, 1 * ms), (1, 2 * ms), (0, 6 * ms), (1, 14 * ms), (0, 21 * ms),
                                  (1, 40 * ms)])
    H = b.ISIHistogramMonitor(G, [0 * ms, 10 * ms, 20 * ms])
    net = b.Network(G, H)
    with engine(oracle_table):
        net.run(45 * ms)
        np.testing.assert_array_equal(H.count, [1, 2, 3])
    np.testing.assert_array_equal(H.bins, [0, 0.01, 0.02])
