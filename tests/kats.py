"""Known-answer tests of the reference test suite, restated for this API.

Each function runs on the active engine and asserts the reference's
expected values.  Sources (Brian 1.4.4, brian/tests/):
  tutorial1c ........... testcorrectness/test_from_tutorial1c.py:3-39
  epsp ................. testcorrectness/test_epsp.py:3-63
  exponential_current .. testcorrectness/test_exponential_current.py:3-58
  connection_values .... testinterface/test_connection.py:89-203
  propagation .......... testfeatures/test_propagation.py:3-35
  stdp_pairing ......... testinterface/test_stdp.py:6-39 (linear neuron model;
                         the reference's conductance model is nonlinear)
  monitor_semantics .... testinterface/test_monitor.py (SpikeMonitor times,
                         StateMonitor timestep, subgroup origin)
"""
import numpy as np

import brian_b200 as b
from brian_b200 import ms, mV, second, msecond, mvolt, volt


def tutorial1c():
    tau, Vt, Vr, El = 20 * msecond, -50 * mvolt, -60 * mvolt, -49 * mvolt
    G = b.NeuronGroup(N=40, model=b.Equations("dV/dt = -(V-El)/tau : volt", tau=tau, El=El), threshold=Vt, reset=Vr)
    G.V = El
    M = b.SpikeMonitor(G)
    b.Network(G, M).run(1 * second)
    assert M.nspikes == 840, M.nspikes


def epsp():
    taum, taupsp, y0 = 10 * ms, 0.325 * ms, 4.86 * mV
    P = b.NeuronGroup(N=1, model=b.Equations("""
        dV/dt = (-V+x)*(1./taum) : volt
        dx/dt = (-x+y)*(1./taupsp) : volt
        dy/dt = -y*(1./taupsp) : volt""", taum=taum, taupsp=taupsp), threshold=100 * mV, reset=0 * mV)
    Pinit = b.SpikeGeneratorGroup(1, [(0, 0 * ms)])
    C = b.Connection(Pinit, P, "y")
    C.connect_full(Pinit, P, y0)
    M = b.StateMonitor(P, "V", record=0)
    b.Network(P, Pinit, C, M).run(10 * ms)
    V = M[0]
    Vi = int(np.argmax(V))
    assert abs(V[Vi] - 0.136889 * mvolt) < 0.001 * mvolt, V[Vi]
    assert abs(M.times[Vi] - 1.69735 * msecond) < max(0.1 * ms, 0.00001 * ms), M.times[Vi]


def exponential_current():
    taum, taue, taui, Vt, Vr = 20 * ms, 1 * ms, 10 * ms, 10 * mV, 0 * mV
    G1 = b.SpikeGeneratorGroup(2, [(0, 0 * ms)])
    G2 = b.NeuronGroup(N=1, model=b.Equations("""
        dV/dt = (-V+ge-gi)/taum : volt
        dge/dt = -ge/taue : volt
        dgi/dt = -gi/taui : volt""", taum=taum, taue=taue, taui=taui), threshold=Vt, reset=Vr)
    G2.V = Vr
    C1 = b.Connection(G1, G2, "ge")
    C2 = b.Connection(G1, G2, "gi")
    C1[0, 0] = 3 * mV
    C2[1, 0] = 3 * mV
    Mv = b.StateMonitor(G2, "V", record=True)
    b.Network(G1, G2, C1, C2, Mv).run(100 * ms)
    t = Mv.times
    Vpred = (np.exp(-t / taum) - np.exp(-t / taue)) * taue * (3 * mV) / (taum - taue)
    assert np.max(np.abs(Vpred - Mv[0])) < 0.00001


def connection_values():
    G1 = b.SpikeGeneratorGroup(2, [(0, 1 * msecond), (1, 3 * msecond)])
    G2 = b.NeuronGroup(2, model=b.Equations("da/dt = 0.*hertz : 1.\ndb/dt = 0.*hertz : 1."), threshold=10.,
                       reset=0.)
    C = b.Connection(G1, G2)
    C.connect_full(G1, G2, weight=2.)
    assert all(C[i, j] == 2. for i in range(2) for j in range(2))
    C = b.Connection(G1, G2)
    C.connect_one_to_one(G1, G2)
    assert C[0, 0] == 1. and C[1, 1] == 1. and C[0, 1] == 0. and C[1, 0] == 0.
    Ca = b.Connection(G1, G2, "a")
    Cb = b.Connection(G1, G2, "b")
    Ca[0, 0] = 1.
    Ca[0, 1] = 1.
    Ca[1, 0] = 1.
    Cb[0, 1] = 1.
    Cb[1, 0] = 1.
    Cb[1, 1] = 1.
    net = b.Network(G1, G2, Ca, Cb)
    net.run(2 * msecond)
    assert np.array_equal(G2.a, [1., 1.]) and np.array_equal(G2.b, [0., 1.]), (G2.a, G2.b)
    net.run(2 * msecond)
    assert np.array_equal(G2.a, [2., 1.]) and np.array_equal(G2.b, [1., 2.]), (G2.a, G2.b)


def propagation():
    dt = b.defaultclock.dt
    H = b.NeuronGroup(1, model=b.Equations("V:1\nmod:1"), threshold=1, reset=0)
    H.V = 2
    H.mod = 1
    G = [b.NeuronGroup(10, model=b.Equations("V:1"), threshold=1, reset=0) for _ in range(12)]
    M = [b.SpikeMonitor(g) for g in G]
    Cs = [b.Connection(H, G[0], "V", weight=2),
          b.Connection(H, G[1], "V", weight=2, structure="dense"),
          b.Connection(H, G[2], "V", weight=2, structure="dynamic"),
          b.Connection(H, G[3], "V", weight=2, modulation="mod"),
          b.Connection(H, G[4], "V", weight=2, structure="dense", modulation="mod"),
          b.Connection(H, G[5], "V", weight=2, structure="dynamic", modulation="mod"),
          b.Connection(H, G[6], "V", weight=2, delay=True),
          b.Connection(H, G[7], "V", weight=2, delay=True, structure="dense"),
          b.Connection(H, G[8], "V", weight=2, delay=True, structure="dynamic"),
          b.Connection(H, G[9], "V", weight=2, delay=True, modulation="mod"),
          b.Connection(H, G[10], "V", weight=2, delay=True, structure="dense", modulation="mod"),
          b.Connection(H, G[11], "V", weight=2, delay=True, structure="dynamic", modulation="mod")]
    for c in Cs[6:]:
        c.delay[0, :] = np.arange(10) * dt + dt / 2
    b.Network(H, *(G + Cs + M)).run(2 * ms)
    for k, m in enumerate(M):
        i, t = m.it
        assert len(i), k
        j = np.array((t + dt / 2) / dt, dtype=int)
        assert np.array_equal(i, np.arange(10)), (k, i)
        if k < 6:
            assert np.all(j == 1), (k, j)
        else:
            assert np.array_equal(j, 1 + np.arange(10)), (k, j)


def stdp_pairing():
    inp = b.SpikeGeneratorGroup(1, [(0, 1 * ms)])
    G = b.NeuronGroup(1, model=b.Equations("dv/dt = (60*mV*ge + (-80*mV - v)) / (5 * ms) : volt\n"
                                           "dge/dt = -ge / (5 * ms) : 1"), threshold=-50 * mV, reset=-80 * mV)
    G.v = -51 * mV
    con = b.Connection(inp, G, "ge", weight=1)
    stdp = b.ExponentialSTDP(con, 10 * ms, 10 * ms, 0.1, 0.1, wmax=10.0)
    post = b.SpikeMonitor(G)
    b.Network(inp, G, con, stdp, post).run(4 * ms)
    assert post.nspikes >= 1
    assert con.W[0, 0] > 1, con.W[0, 0]


def monitor_semantics():
    G = b.SpikeGeneratorGroup(6, [(1, 0.5 * ms), (4, 0.5 * ms), (2, 1.0 * ms), (5, 2.0 * ms)])
    Ms = b.SpikeMonitor(G)
    Msub = b.SpikeMonitor(G[2:6])
    Md = b.SpikeMonitor(G, delay=0.35 * ms)   # int(3.5) = 3 bins
    H = b.NeuronGroup(3, model=b.Equations("dx/dt = 1/(10*ms) : 1"))
    Sx = b.StateMonitor(H, "x", record=[2, 0], timestep=4)
    b.Network(G, H, Ms, Msub, Md, Sx).run(3 * ms)
    dt = b.defaultclock.dt
    i, t = Ms.it
    assert np.array_equal(i, [1, 4, 2, 5]) and np.allclose(t, [5 * dt, 5 * dt, 10 * dt, 20 * dt])
    i2, t2 = Msub.it
    assert np.array_equal(i2, [2, 0, 3]) and np.allclose(t2, [5 * dt, 10 * dt, 20 * dt])
    i3, t3 = Md.it
    assert np.array_equal(i3, [1, 4, 2, 5]) and np.allclose(t3, [8 * dt, 8 * dt, 13 * dt, 23 * dt])
    assert len(Sx.times) == 8 and np.allclose(Sx.times, np.arange(0, 30, 4) * dt)
    assert Sx.values.shape == (2, 8)
    assert np.allclose(Sx[0], Sx[2])


ALL = [tutorial1c, epsp, exponential_current, connection_values, propagation, stdp_pairing, monitor_semantics]
