"""NetworkBatch: independent networks in one launch (one block each) against
the oracle running every network alone, bit for bit -- spikes, states,
StateMonitor rows and event counters -- with uneven durations, several runs,
both ring placements (shared memory and the engine's ring in global memory)
and every block shape and lanes-per-row setting."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms, mV
from brian_b200.connections import fixed_indegree_csr
from brian_b200.network import engine

import scenarios

EQS = """
dv/dt  = (ge+gi-(v-El))/taum : volt
dge/dt = -ge/taue : volt
dgi/dt = -gi/taui : volt
"""


def _net(kind, n, seed, record=(0, 1), timestep=1, sub_monitor=False):
    """One small network on its own clock.  kind "cuba": Bernoulli p = 0.02
    zero-delay Connections (CUBA.py); "delay": fixed in-degree
    DelayConnections with delays 1..50 steps; "exc": one Connection only."""
    clk = b.Clock(dt=0.1 * ms)
    eqs = b.Equations(EQS, taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    P = b.NeuronGroup(n, model=eqs, threshold=-50 * mV, reset=-60 * mV, clock=clk)
    ne = int(0.8 * n)
    Pe, Pi = P.subgroup(ne), P.subgroup(n - ne)
    rng = np.random.Generator(np.random.PCG64(seed))
    objs = [P]
    if kind == "cuba":
        for src, w, var, sd in ((Pe, 1.62 * mV, "ge", seed), (Pi, -9 * mV, "gi", seed + 1)):
            C = b.Connection(src, P, var)
            C.connect_random(src, P, 0.02, weight=w, seed=sd)
            objs.append(C)
    elif kind == "exc":
        C = b.Connection(Pe, P, "ge")
        C.connect_random(Pe, P, 0.05, weight=1.2 * mV, seed=seed)
        objs.append(C)
    else:
        k = 60
        for src, m, kk, w, var, sd in ((Pe, ne, int(0.8 * k), 0.4e-2, "ge", seed), (Pi, n - ne, k - int(0.8 * k), -1.5e-2,
                                                                                        "gi", seed + 1)):
            rowptr, cols = fixed_indegree_csr(m, n, kk, seed=sd)
            C = b.DelayConnection(src, P, var, max_delay=5 * ms, dtype=np.float32)
            C.connect_csr(rowptr, cols, w, delay_steps=rng.integers(1, 51, size=len(cols)).astype(np.uint8))
            objs.append(C)
    P.v = -60 * mV + rng.random(n) * 10 * mV
    M = b.SpikeMonitor(Pi if sub_monitor else P)
    S = b.StateMonitor(P, "v", record=[r % n for r in record], timestep=timestep)
    objs += [M, S]
    net = b.Network(*objs)
    return net, P, M, S


SPECS = [dict(kind="cuba", n=4000, seed=11, record=(0, 3999, 7)),
         dict(kind="cuba", n=2500, seed=12, record=(2499, 0), timestep=2, sub_monitor=True),
         dict(kind="delay", n=1000, seed=13),                       # rings in global memory (too large)
         dict(kind="delay", n=300, seed=14, record=(299,)),          # rings in shared memory
         dict(kind="exc", n=4096, seed=15, sub_monitor=True),
         dict(kind="cuba", n=33, seed=16)]


def _result(net, P, M, S):
    s, i = M._record()
    st, v = S._record()
    g, c = net._binding.rt.counters(1, len(net.connections))
    return {"v": np.array(P.v), "ge": np.array(P.ge), "gi": np.array(P.gi), "spk.steps": s.copy(),
            "spk.idx": i.copy(), "st.steps": st.copy(), "st.vals": v.copy(), "spikes": g.copy(), "events": c.copy()}


def _oracle(oracle_table, specs, durations_list):
    out = []
    with engine(oracle_table):
        for spec, durs in zip(specs, zip(*durations_list)):
            net, P, M, S = _net(**spec)
            for d in durs:
                net.run(d * 0.1 * ms)
            out.append(_result(net, P, M, S))
            net._invalidate()
    return out


def _batched(specs, durations_list, shape=None, autotune=False):
    built = [_net(**spec) for spec in specs]
    batch = b.NetworkBatch([x[0] for x in built])
    if shape is not None:
        batch.set_shape(*shape)
    for k, durs in enumerate(durations_list):
        if autotune and k == 1:
            batch.autotune(50)
        batch.run([d * 0.1 * ms for d in durs])
    res = [_result(*x) for x in built]
    info = batch.shape()
    batch.close()
    for x in built:
        x[0]._invalidate()
    return res, info


@pytest.mark.gpu
def test_batch_uneven_durations_bit_exact(oracle_table, gpu_table):
    durations = [[3000, 2000, 2500, 1234, 3000, 700], [500, 1700, 0, 999, 1, 2300]]
    ref = _oracle(oracle_table, SPECS, durations)
    got, info = _batched(SPECS, durations, autotune=True)
    assert sum(len(r["spk.idx"]) for r in ref) > 5000
    for k, (r, g) in enumerate(zip(ref, got)):
        try:
            scenarios.compare(r, g)
        except AssertionError as e:
            raise AssertionError("network %d (%s): %s" % (k, SPECS[k], e))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("lanes", [4, 32])
def test_batch_every_shape_bit_exact(oracle_table, gpu_table, shape, lanes):
    specs = [dict(kind="cuba", n=500, seed=21, record=(1, 499)), dict(kind="delay", n=300, seed=22),
             dict(kind="exc", n=512, seed=23, sub_monitor=True)]
    durations = [[800, 600, 900]]
    ref = _oracle(oracle_table, specs, durations)
    got, info = _batched(specs, durations, shape=(shape, lanes))
    assert info["shape"] == shape and info["lanes"] == lanes
    for r, g in zip(ref, got):
        scenarios.compare(r, g)


@pytest.mark.gpu
def test_network_continues_alone_after_batch(oracle_table, gpu_table):
    """Batch run, then each network runs alone on the engine: the same as the
    oracle's run(T1) + run(T2) (rings, monitors and counters carry over)."""
    specs = [dict(kind="delay", n=1000, seed=31), dict(kind="cuba", n=2000, seed=32, timestep=3)]
    ref = _oracle(oracle_table, specs, [[1200, 1500], [800, 400]])
    built = [_net(**spec) for spec in specs]
    batch = b.NetworkBatch([x[0] for x in built])
    batch.run([1200 * 0.1 * ms, 1500 * 0.1 * ms])
    built[0][0].run(800 * 0.1 * ms)
    built[1][0].run(400 * 0.1 * ms)
    for r, x in zip(ref, built):
        scenarios.compare(r, _result(*x))
        x[0]._invalidate()
    batch.close()


@pytest.mark.gpu
def test_batch_refuses_what_it_cannot_run(gpu_table):
    from brian_b200._lib import EngineError
    net, P, M, S = _net("cuba", 500, 1)
    eqs = b.Equations(EQS, taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    clk = b.Clock(dt=0.1 * ms)
    Q = b.NeuronGroup(100, model=eqs, threshold=-50 * mV, reset=-60 * mV, refractory=5 * ms, clock=clk)
    other = b.Network(Q)
    with pytest.raises(EngineError) as e:
        b.NetworkBatch([net, other]).run(10 * 0.1 * ms)
    assert "network 1" in str(e.value) and "refractor" in str(e.value)
    big, *_ = _net("exc", 5000, 2)
    with pytest.raises(EngineError) as e:
        b.NetworkBatch([big]).run(10 * 0.1 * ms)
    assert "4096" in str(e.value)
    for x in (net, other, big):
        x._invalidate()
