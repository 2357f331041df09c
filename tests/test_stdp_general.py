"""STDP from equations and code strings (stdp.py:92-449): the exponential
additive rule written by hand runs exactly as ExponentialSTDP
(stdp.py:452-539, which the reference builds from the same strings), on a
plain and on a delayed connection; other rules are refused."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms
from brian_b200.network import engine

import scenarios


def _run(tab, fn, **kw):
    b.clear()
    b.reinit_default_clock()
    np.random.seed(1234)
    with engine(tab):
        return fn(**kw)


@pytest.mark.parametrize("dense", [True, False])
def test_general_equals_exponential(oracle_table, dense):
    a = _run(oracle_table, scenarios.stdp, dense=dense, steps=1500)
    g = _run(oracle_table, scenarios.stdp, dense=dense, steps=1500, general=True)
    assert not np.array_equal(a["w0"], 0 * a["w0"])
    scenarios.compare(a, g)


@pytest.mark.parametrize("interactions", ["all", "nearest", "nearest_post"])
def test_general_equals_exponential_delayed(oracle_table, interactions):
    a = _run(oracle_table, scenarios.stdp_delay, Nin=120, Nout=20, steps=1200, interactions=interactions)
    g = _run(oracle_table, scenarios.stdp_delay, Nin=120, Nout=20, steps=1200, interactions=interactions,
             general=True)
    scenarios.compare(a, g)


def test_engine_parameters():
    G = b.NeuronGroup(4, model="v : 1")
    C = b.Connection(G, G, "v", structure="dense")
    C.connect(W=np.full((4, 4), 0.5))
    taup, taum, gmax = 16.8 * ms, 33.7 * ms, 2.0
    dA_pre, dA_post = 0.005, -0.00525
    S = b.STDP(C, "dA_pre/dt=-A_pre/taup : 1\ndA_post/dt=-A_post/taum : 1", pre="A_pre+=dA_pre; w+=A_post",
               post="A_post=dA_post; w+=A_pre", wmin=0.1, wmax=gmax)
    E = b.ExponentialSTDP(C, taup, taum, dA_pre / gmax, dA_post / gmax, interactions="nearest_post",
                          wmin=0.1, wmax=gmax)
    np.testing.assert_array_equal(S.decay, E.decay)
    assert (S.Ap, S.Am, S.wmin, S.wmax, S.interactions) == (E.Ap, E.Am, E.wmin, E.wmax, E.interactions)
    assert isinstance(E, b.STDP)


@pytest.mark.parametrize("pre,post", [("A_pre+=0.01; w*=(2+A_post)", "A_post+=-0.01; w+=A_pre"),
                                      ("A_pre+=0.01; w+=A_post; w+=0.1", "A_post+=-0.01; w+=A_pre"),
                                      ("A_pre=0.01; w+=A_post", "A_post+=-0.01; w+=A_pre"),
                                      ("A_pre+=A_pre; w+=A_post", "A_post+=-0.01; w+=A_pre")])
def test_unsupported_rules(pre, post):
    G = b.NeuronGroup(4, model="v : 1")
    C = b.Connection(G, G, "v")
    C.connect_full(G, G, weight=0.1)
    with pytest.raises(NotImplementedError):
        b.STDP(C, "dA_pre/dt=-A_pre/(10*ms) : 1\ndA_post/dt=-A_post/(10*ms) : 1", pre=pre, post=post, wmax=1.0)
