"""ExponentialSTDP update='multiplicative' and 'mixed' (stdp.py:510-533) on
the oracle, against the reference's own code strings.

The replay builds the pre and post code the way the reference does for a
connection without delays (stdp.py:370-414: 'for _i in spikes:', the
presynaptic variables indexed by _i, w replaced by w[_i,:] / w[:,_i], the
clip line with the bounds formatted by '%e', constants frozen by repr,
optimiser.py:53-88) and executes it with numpy on a dense weight matrix,
driven by the spike trains the oracle recorded; the trace groups decay by
their 1x1 propagators.  Weights and traces must equal the oracle's bit for
bit.
"""
import re

import numpy as np
import pytest

import brian_b200 as b
from brian_b200.network import engine

import scenarios


def _run(tab, **kw):
    b.clear()
    b.reinit_default_clock()
    np.random.seed(1234)
    with engine(tab):
        return scenarios.stdp(**kw)


def _codes(update, gmax, Ap=0.01, Am=-0.0105):
    """The reference's ExponentialSTDP strings for interactions='all'."""
    pre, post = "A_pre+=Ap", "A_post+=Am"
    if update == "multiplicative":
        pre += "\nw*=(1+A_post)" if Am < 0 else "\nw+=(wmax-w)*A_post"
        post += "\nw*=(1+A_pre)" if Ap < 0 else "\nw+=(wmax-w)*A_pre"
    else:   # mixed with Am < 0 < Ap
        Ap *= gmax
        pre += "\nw*=(1+A_post)"
        post += "\nw+=A_pre"
    consts = {"Ap": repr(float(Ap)), "Am": repr(float(Am)), "wmax": repr(float(gmax))}

    def gen(code, own, widx):
        out = "for _i in spikes:\n"
        for ln in code.split("\n"):
            for k, v in consts.items():
                ln = re.sub(r"\b%s\b" % k, v, ln)
            ln = re.sub(r"\b%s\b" % own, own + "[_i]", ln)
            ln = re.sub(r"\bw\b", widx, ln)
            out += "    " + ln + "\n"
        out += "    %s=clip(%s,%e,%e)\n" % (widx, widx, 0.0, gmax)
        return out

    return gen(pre, "A_pre", "w[_i,:]"), gen(post, "A_post", "w[:,_i]")


def _replay(res, Nin, Nout, nsteps, update, gmax=0.01):
    w = res["w_init"].reshape(Nin, Nout).copy()
    a_pre, c_pre, a_post, c_post = res["decay"]
    pre_code, post_code = _codes(update, gmax)
    sin = [[] for _ in range(nsteps)]
    sout = [[] for _ in range(nsteps)]
    for s_, i in zip(res["spk1.steps"], res["spk1.idx"]):
        sin[int(s_)].append(int(i))
    for s_, j in zip(res["spk0.steps"], res["spk0.idx"]):
        sout[int(s_)].append(int(j))
    ns = {"A_pre": np.zeros(Nin), "A_post": np.zeros(Nout), "w": w, "clip": np.clip}
    for t in range(nsteps):
        ns["A_pre"][:] = a_pre * ns["A_pre"] + c_pre
        ns["A_post"][:] = a_post * ns["A_post"] + c_post
        ns["spikes"] = sin[t]
        exec(pre_code, ns)
        ns["spikes"] = sout[t]
        exec(post_code, ns)
    return w.ravel(), ns["A_pre"], ns["A_post"]


@pytest.mark.parametrize("update", ["multiplicative", "mixed"])
def test_update_forms_match_reference_code(oracle_table, update):
    Nin, Nout, nsteps = 120, 16, 1500
    res = _run(oracle_table, Nin=Nin, Nout=Nout, steps=nsteps, dense=True, wdtype=np.float64, update=update)
    assert len(res["spk0.idx"]) > 20
    w, A_pre, A_post = _replay(res, Nin, Nout, nsteps, update)
    assert not np.array_equal(w, res["w_init"])
    np.testing.assert_array_equal(w, res["w0"])
    np.testing.assert_array_equal(A_pre, res["stdp0.pre"])
    np.testing.assert_array_equal(A_post, res["stdp0.post"])


def test_forms_differ_and_fp32_refused(oracle_table):
    add = _run(oracle_table, Nin=80, Nout=10, steps=800, dense=True, wdtype=np.float64)
    mul = _run(oracle_table, Nin=80, Nout=10, steps=800, dense=True, wdtype=np.float64, update="multiplicative")
    assert not np.array_equal(add["w0"], mul["w0"])
    with pytest.raises(Exception):
        _run(oracle_table, Nin=80, Nout=10, steps=10, dense=True, wdtype=np.float32, update="multiplicative")


def test_delayed_multiplicative_runs(oracle_table):
    b.clear()
    b.reinit_default_clock()
    np.random.seed(1234)
    with engine(oracle_table):
        r = scenarios.stdp_delay(Nin=100, Nout=12, steps=800, update="multiplicative")
    assert not np.array_equal(r["w0"], r["w_init"])
    assert np.all(r["w0"] >= 0) and np.all(r["w0"] <= 0.01)
