"""ExponentialSTDP on a DelayConnection: the oracle against a replay of the
reference's own bookkeeping.

The replay restates stdp.py:296-368 (the immediate and delayed updaters
and their code strings), DelayedSTDPUpdater.propagate (stdp.py:77-89) and
RecentStateMonitor (monitor.py:991-1099: records at the end of each step
into slot current_time_index, get_past_values_sequence indexes
(current_time_index - 1 - array(invdt * times, dtype=int)) % M) in numpy,
driven by the spike trains the oracle recorded.  Given the same spikes, its
weights and traces must equal the oracle's bit for bit.  It computes the
lags itself from the delays in seconds, independently of the engine's host
code.
"""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200.network import engine

import scenarios

DT = 1e-4
_PRE_ADD = {"all": True, "nearest": False, "nearest_pre": False, "nearest_post": True}
_POST_ADD = {"all": True, "nearest": False, "nearest_pre": False, "nearest_post": False}


def _run_oracle(oracle_table, **kw):
    b.clear()
    b.reinit_default_clock()
    np.random.seed(1234)
    with engine(oracle_table):
        return scenarios.stdp_delay(**kw)


def _by_step(steps_arr, idx_arr, nsteps):
    out = [[] for _ in range(nsteps)]
    for s, i in zip(steps_arr, idx_arr):
        out[int(s)].append(int(i))
    return [np.array(x, dtype=np.int64) for x in out]


def replay(res, Nin, Nout, nsteps, interactions):
    rowptr, cols, d = res["rowptr"], res["cols"], res["d"]
    w = res["w_init"].copy()
    a_pre, c_pre, a_post, c_post = res["decay"]
    gmax = 0.01
    Ap, Am = 0.01 * gmax, -0.0105 * gmax
    wmin, wmax = float("%e" % 0.0), float("%e" % gmax)          # stdp.py:325, '%e' in the code string
    md = int(5e-3 / DT) + 1                                      # delayconnection.py:94
    max_delay = md * DT                                          # stdp.py:297
    D = int(max_delay / DT)                                      # monitor.py:142
    M = int(((md + 1) * DT) / (1 * DT)) + 1                      # monitor.py:1024-1026
    maxd = float("%.12g" % max_delay)                            # str(float) in stdp.py:78
    inv = 1.0 / DT
    rows = np.repeat(np.arange(Nin), np.diff(rowptr))
    col_syn = [np.nonzero(cols == j)[0] for j in range(Nout)]    # ascending source per column
    sin = _by_step(res["spk1.steps"], res["spk1.idx"], nsteps)
    sout = _by_step(res["spk0.steps"], res["spk0.idx"], nsteps)
    A_pre, A_post = np.zeros(Nin), np.zeros(Nout)
    Vpre, Vpost = np.zeros((M, Nin)), np.zeros((M, Nout))
    cur = 0
    for t in range(nsteps):
        A_pre = a_pre * A_pre + c_pre
        A_post = a_post * A_post + c_post
        for i in sin[t]:                                         # immediate presynaptic updater
            A_pre[i] = A_pre[i] + Ap if _PRE_ADD[interactions] else Ap
        if t >= D:                                               # delayed presynaptic updater
            sp = sin[t - D]
            seqs = [maxd - d[rowptr[i]:rowptr[i + 1]] for i in sp]
            vals = [Vpost[(cur - 1 - np.array(inv * tm, dtype=int)) % M, cols[rowptr[i]:rowptr[i + 1]]]
                    for i, tm in zip(sp, seqs)]
            for i, v in zip(sp, vals):
                seg = slice(rowptr[i], rowptr[i + 1])
                w[seg] = np.clip(w[seg] + v, wmin, wmax)
        so = sout[t]                                             # postsynaptic updater
        vals = [Vpre[(cur - 1 - np.array(inv * d[col_syn[j]], dtype=int)) % M, rows[col_syn[j]]] for j in so]
        for j in so:
            A_post[j] = A_post[j] + Am if _POST_ADD[interactions] else Am
        for j, v in zip(so, vals):
            k = col_syn[j]
            w[k] = np.clip(w[k] + v, wmin, wmax)
        Vpre[cur] = A_pre                                        # RecentStateMonitors, when='end'
        Vpost[cur] = A_post
        cur = (cur + 1) % M
    return w, A_pre, A_post


@pytest.mark.parametrize("interactions", ["all", "nearest_pre", "nearest_post"])
def test_oracle_matches_reference_bookkeeping(oracle_table, interactions):
    Nin, Nout, nsteps = 150, 24, 1500
    res = _run_oracle(oracle_table, Nin=Nin, Nout=Nout, steps=nsteps, interactions=interactions)
    assert len(res["spk0.idx"]) > 20 and len(res["spk1.idx"]) > 1000
    w, A_pre, A_post = replay(res, Nin, Nout, nsteps, interactions)
    assert not np.array_equal(w, res["w_init"])
    np.testing.assert_array_equal(w, res["w0"])
    np.testing.assert_array_equal(A_pre, res["stdp0.pre"])
    np.testing.assert_array_equal(A_post, res["stdp0.post"])


def test_lags_are_not_complements(oracle_table):
    """The delayed presynaptic lookup int((1/dt)*(max_delay-d)) is not
    (max_delay bins) - int((1/dt)*d) for most float delays: the case the
    replay above would catch if the engine used the complement."""
    res = _run_oracle(oracle_table, Nin=60, Nout=10, steps=10)
    md = int(5e-3 / DT) + 1
    maxd = float("%.12g" % (md * DT))
    d = res["d"]
    pre = np.array((1.0 / DT) * (maxd - d), dtype=int)
    post = np.array((1.0 / DT) * d, dtype=int)
    assert np.mean(pre != int(md * DT / DT) - post) > 0.5


def test_two_runs_continue(oracle_table):
    """Two runs of half the duration give the run of the whole duration
    (the trace records and their ring index carry over)."""
    one = _run_oracle(oracle_table, Nin=100, Nout=16, steps=800)
    two = _run_oracle(oracle_table, Nin=100, Nout=16, steps=800, runs=2)
    scenarios.compare(one, two)
