"""The STDP scale-up network at full size (10 000 Poisson inputs onto 4096
LIF outputs, all to all, dense f32 W = 41 M plastic synapses,
ExponentialSTDP; examples/plasticity/STDP1.py:8-58 scaled up): the CUDA
engine against the oracle over a shortened run.  Weights, traces, spikes and
states equal bit for bit."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import workloads
from brian_b200.network import engine


def _run(table, steps, nout=4096, runs=1):
    b.clear()
    b.reinit_default_clock()

    def go():
        d = workloads.stdp_scaleup(seed=77, nout=nout, spike_record=nout, record=[0, 1, 2, nout - 1],
                                   input_monitor=True)
        for _ in range(runs):
            d["net"].run(steps // runs * 1e-4)
        a_pre, a_post = d["stdp"]._traces()
        out = {"W": d["C"]._weights().copy(), "A_pre": a_pre.copy(), "A_post": a_post.copy(),
               "v": np.array(d["outputs"].v), "ge": np.array(d["outputs"].ge),
               "spk": d["M"]._record(), "inp": d["Mi"]._record(), "trace": d["S"]._record()}
        d["net"]._invalidate()
        return out
    if table is None:
        return go()
    with engine(table):
        return go()


@pytest.mark.gpu
def test_stdp_scaleup_bit_exact(oracle_table, gpu_table):
    ref = _run(oracle_table, 240, runs=2)
    gpu = _run(None, 240, runs=2)
    # the outputs fire at hundreds of spikes per step, so nearly every
    # column takes postsynaptic updates every step
    assert len(ref["spk"][1]) > 100000 and len(ref["inp"][1]) > 1000
    for k in ("spk", "inp", "trace"):
        for x, y in zip(ref[k], gpu[k]):
            assert np.array_equal(x, y), k
    for k in ("W", "A_pre", "A_post", "v", "ge"):
        assert np.array_equal(ref[k], gpu[k]), k
