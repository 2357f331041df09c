"""FP32 state against FP64 on the plain CUBA network (4000 LIF, p = 0.02,
zero delay, 1 s).  The network is chaotic: the FP32 run repeats the FP64
spikes exactly until a neuron sits within rounding distance of the
threshold (5-25 ms in, depending on the seed), and from there the two
trajectories part like any two runs with different initial states.  So the
spike-timing bar (gamma >= 0.95, delta 4 ms) is checked over the first
50 ms, the traces before the first differing spike must agree to float
precision, and over the whole second the population rate must agree within
3 %."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import workloads
from brian_b200.statistics import precision_agreement


def _run(prec, seed=1, steps=10000):
    b.set_global_preferences(precision=prec)
    try:
        b.clear()
        b.reinit_default_clock()
        net, P, M, S = workloads.cuba4000(seed=seed)
        net.run(steps * 1e-4)
        out = (tuple(x.copy() for x in M._record()), S._record()[1].copy())
        net._invalidate()
        return out
    finally:
        b.set_global_preferences(precision=64)


@pytest.mark.gpu
def test_cuba4000_fp32_tracks_fp64(gpu_table):
    (r64, v64), (r32, v32) = _run(64), _run(32)
    rep = precision_agreement(r64, r32, 4000, 1.0, v64, v32)
    assert rep["spikes_fp64"] > 10000
    assert rep["gamma_mean_by_window_ms"]["50"] >= 0.95, rep
    assert rep["rate_rel_err"] < 0.03, rep
    # before the first differing spike the traces agree to float precision
    s0 = rep["first_differing_step"]
    assert s0 is not None and s0 > 20
    d = np.abs(v32[:s0] - v64[:s0])
    assert d.max() < 1e-6, d.max()
