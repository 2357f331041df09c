"""The reference's testinterface/test_synapses.py construction and access
tests (test_construction_single_synapses, test_construction_multiple_synapses,
test_construction_and_access, :23-300) restated for the host class."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms
from brian_b200.network import engine


def _group():
    b.clear()
    b.reinit_default_clock()
    G = b.NeuronGroup(20, model="v:1")
    return G, G[:10], G[10:]


def test_construction_single_synapses(oracle_table):
    G, s1, s2 = _group()
    syn = b.Synapses(G, model="w:1")
    assert syn.source is syn.target
    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    assert syn.source is s1 and syn.target is s2
    syn[:, :] = True
    assert len(syn) == 10 * 10
    with pytest.raises(ValueError):
        syn[0, 0] = False
    syn.w[:, :] = 2
    syn.delay[:, :] = 1 * ms
    assert all(syn.w[i, j] == 2 for i in range(10) for j in range(10))
    assert all(syn.delay[i, j] == 1 * ms for i in range(10) for j in range(10))

    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    syn[:, :] = "i == j"
    syn.w[:, :] = 2
    assert len(syn) == 10
    for i in range(10):
        for j in range(10):
            if i == j:
                assert syn.w[i, j] == 2
            else:
                assert len(syn.w[i, j]) == 0
    net = b.Network(G, syn)
    with engine(oracle_table):
        net.run(b.defaultclock.dt)
    with pytest.raises(AttributeError):
        syn[0, 1] = True

    for args, kw in (((s1, s2), {}), ((s1,), {}), ((), {"post": s2}), ((), {})):
        syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
        syn.connect_one_to_one(*args, **kw)
        assert len(syn) == 10
    with pytest.raises(TypeError):
        syn.connect_one_to_one(G[:2], G[:1])

    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    syn[:, :] = 0.0
    assert len(syn) == 0
    syn.connect_random(s1, s2, 0.0)
    assert len(syn) == 0
    for make in (lambda S: S.__setitem__((slice(None), slice(None)), 1.0),
                 lambda S: S.connect_random(s1, s2, 1.0),
                 lambda S: S.connect_random(s1, sparseness=1.0),
                 lambda S: S.connect_random(post=s2, sparseness=1.0),
                 lambda S: S.connect_random(sparseness=1.0)):
        syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
        make(syn)
        assert len(syn) == 100
    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    for bad in (1.3, -0.3):
        with pytest.raises(ValueError):
            syn.connect_random(s1, s2, bad)
        with pytest.raises(ValueError):
            syn[:, :] = bad

    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    syn[np.arange(5), np.arange(5)] = True
    syn.w[np.arange(5), np.arange(5)] = 2
    syn.delay[np.arange(5), np.arange(5)] = 5 * ms
    assert len(syn) == 25
    assert all(syn.w[i, j] == 2 for i in range(5) for j in range(5))
    assert all(syn.delay[i, j] == 5 * ms for i in range(5) for j in range(5))
    assert all(len(syn.w[i, j]) == 0 for i in range(5, 10) for j in range(5, 10))
    b.Synapses(s1, s2, model="", pre="v+=1")


def test_construction_multiple_synapses():
    G, s1, s2 = _group()
    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    syn[:, :] = 3
    assert len(syn) == 300
    syn.w[:, :] = 2
    syn.delay[:, :] = 1 * ms
    assert all(syn.w[i, j, k] == 2 for i in range(10) for j in range(10) for k in range(3))
    assert all(syn.delay[i, j, k] == 1 * ms for i in range(10) for j in range(10) for k in range(3))
    assert len(syn.w[2, 3, 1]) == 1 and len(syn.w[2, 3, 3]) == 0


def test_construction_and_access():
    G, s1, s2 = _group()
    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    syn[3, 4] = True
    syn.w[3, 4] = 0.25
    syn.delay[3, 4] = 1 * ms
    for i in range(10):
        for j in range(10):
            if (i, j) == (3, 4):
                assert syn.w[i, j] == 0.25 and syn.delay[i, j] == 1 * ms
            else:
                assert len(syn.w[i, j]) == 0 and len(syn.delay[i, j]) == 0
    with pytest.raises(ValueError):
        syn[3, 10] = True
    with pytest.raises(ValueError):
        syn[10, 4] = True
    for key in ((3, slice(None)), (slice(None), 4)):
        syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
        syn[key] = True
        syn.w[key] = 0.25
        syn.delay[key] = 1 * ms
        assert len(syn) == 10
        assert (syn.w[key] == 0.25).all() and (syn.delay[key] == 1 * ms).all()


def test_string_initialisation():
    """test_construction_and_access, :300-322: string expressions of i
    (and n, numpy, units) for variables and delays; delays are whole
    multiples of dt (truncated)."""
    G, s1, s2 = _group()
    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    syn[:, 4] = True
    syn.w[:, 4] = "(i % 2 == 0) * 0.5 + 0.5"
    syn.delay[:, 4] = "(i % 2 == 0) * 0.5 * ms + 0.5 * ms"
    assert (syn.w[::2, 4] == 1).all() and (syn.w[1::2, 4] == 0.5).all()
    assert (syn.delay[::2, 4] == 1 * ms).all() and (syn.delay[1::2, 4] == 0.5 * ms).all()
    syn = b.Synapses(s1, s2, model="w:1", pre="v += w")
    syn[:, 4] = True
    syn.w[:, 4] = "0.5 + 0.5 * np.cos(i / (1.0 * n) * np.pi)"
    syn.delay[:, 4] = "0.0005 + 0.0005 * np.cos(i / (1.0 * n) * np.pi)"
    assert (syn.w[:, 4] == 0.5 + 0.5 * np.cos(np.arange(10) / 10.0 * np.pi)).all()
    delays = 0.5 * ms + 0.5 * ms * np.cos(np.arange(10) / 10.0 * np.pi)
    dt = b.defaultclock.dt
    assert (syn.delay[:, 4] == (delays / dt).astype(int) * dt).all()
