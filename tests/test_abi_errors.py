"""Argument checks of the Synapses and STDP entry points, on the oracle's
copy of the ABI (the engine's checks are the same; the engine needs a
device to create a network)."""
import numpy as np
import pytest

from brian_b200._lib import Runtime, EngineError


def _rt(oracle_table):
    rt = Runtime(table=oracle_table, dt=1e-4)
    g = rt.group_add(np.zeros((2, 4)))
    return rt, g


def test_synapses_argument_checks(oracle_table):
    rt, g = _rt(oracle_table)
    ok = dict(pre=[0, 1], post=[1, 2], delay=[0, 3], op_var=[0], op_sub=[0], terms=np.ones((1, 2)))
    sid = rt.synapses_add(g, 0, 4, g, 0, 4, **ok)
    assert sid == 0
    bad = [dict(ok, post=[1, 4]),                       # target beyond the range
           dict(ok, pre=[-1, 0]),                       # negative source
           dict(ok, delay=[0, -2]),                     # negative delay
           dict(ok, op_var=[2]),                        # no such state variable
           dict(ok, op_var=[0] * 5, op_sub=[0] * 5, terms=np.ones((5, 2)))]   # more than four statements
    for kw in bad:
        with pytest.raises(EngineError):
            rt.synapses_add(g, 0, 4, g, 0, 4, **kw)
    with pytest.raises(EngineError):
        rt.synapses_add(g, 2, 4, g, 0, 4, **ok)        # source range past the group


def test_stdp_argument_checks(oracle_table):
    rt, g = _rt(oracle_table)
    rowptr, cols = np.array([0, 1, 2, 2, 2]), np.array([1, 2], dtype=np.int32)
    c64 = rt.conn_add(g, 0, 4, g, 0, 4, 0, rowptr, cols, np.array([0.5, 0.5]))
    c32 = rt.conn_add(g, 0, 4, g, 0, 4, 0, rowptr, cols, np.array([0.5, 0.5], dtype=np.float32))
    cd = rt.conn_add(g, 0, 4, g, 0, 4, 0, rowptr, cols, np.array([0.5, 0.5]), delays=np.array([1, 2], np.uint8),
                     ring_depth=5)
    decay = np.array([0.9, 0.0, 0.9, 0.0])
    s = rt.stdp_add(c64, decay, 0.01, -0.01, 0.0, 1.0, 0, 0, 0)
    rt.stdp_set_update(s, 1, 2, 1.0)
    with pytest.raises(EngineError):
        rt.stdp_set_update(s, 3, 0, 1.0)                # no such update form
    s32 = rt.stdp_add(c32, decay, 0.01, -0.01, 0.0, 1.0, 0, 0, 0)
    with pytest.raises(EngineError):
        rt.stdp_set_update(s32, 1, 0, 1.0)              # multiplicative needs FP64 weights
    with pytest.raises(EngineError):                    # lags must lie within the trace history
        rt.stdp_add_delayed(cd, decay, 0.01, -0.01, 0.0, 1.0, 0, 5, 4, [0, 4], [0, 1])
    with pytest.raises(EngineError):                    # a plain connection is not a DelayConnection
        rt.stdp_add_delayed(c64, decay, 0.01, -0.01, 0.0, 1.0, 0, 5, 4, [0, 1], [0, 1])
    rt.stdp_add_delayed(cd, decay, 0.01, -0.01, 0.0, 1.0, 0, 5, 7, [0, 4], [1, 2])
    rt.prepare()
    with pytest.raises(EngineError):
        rt.stdp_set_update(s, 0, 0, 1.0)                # after prepare
