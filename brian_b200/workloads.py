"""Seeded synthetic networks of the benchmark configurations, built with the
public API (the same calls a user of the reference writes).

- ``cuba4000``: the plain CUBA network of examples/misc/CUBA.py:25-74 --
  4000 LIF neurons (3200 exc / 800 inh), Bernoulli p = 0.02 connectivity,
  we = 1.62 mV, wi = -9 mV, zero delay, v0 uniform in [Vr, Vt], a
  SpikeMonitor and the v trace of 10 neurons.
- ``cuba_scaled_inputs`` / ``cuba_scaled``: CUBA with delays at scale --
  262 144 LIF neurons, fixed in-degree 1000 (800 exc + 200 inh), f32
  weights 0.162 mV / -0.9 mV, u8 delays uniform in 1..50 steps.
- ``stdp_scaleup``: examples/plasticity/STDP1.py:8-58 scaled up -- 10 000
  Poisson inputs at rates uniform in [5, 25] Hz onto 4096 LIF outputs, all
  to all (dense f32 W, w0 uniform in [0, gmax]), ExponentialSTDP with
  taupre = taupost = 20 ms, gmax = 0.01, dApre = 0.01 gmax, dApost =
  -1.05 dApre.

All values are SI floats, dt = 0.1 ms.  The random inputs come from numpy's
PCG64 generator (and the engine's counter-based generator for the Poisson
spikes and the fixed in-degree rows), so a seed fixes the network.
"""
import numpy as np

from .units import ms, mV

__all__ = ["cuba4000", "cuba_scaled_inputs", "cuba_scaled", "stdp_scaleup", "CUBA_EQS", "STDP_EQS"]

CUBA_EQS = """
dv/dt  = (ge+gi-(v-El))/taum : volt
dge/dt = -ge/taue : volt
dgi/dt = -gi/taui : volt
"""

STDP_EQS = """
dv/dt=(ge*(Ee-vr)+El-v)/taum : volt
dge/dt=-ge/taue : 1
"""


def _b():
    import brian_b200 as b
    return b


def cuba4000(seed=1, n=4000, p=0.02, record=10, refractory=0.0):
    """CUBA-4000 (FP64 in the reference): returns (net, P, M, S)."""
    b = _b()
    eqs = b.Equations(CUBA_EQS, taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    Vt, Vr = -50 * mV, -60 * mV
    P = b.NeuronGroup(n, model=eqs, threshold=Vt, reset=Vr, refractory=refractory)
    ne = int(0.8 * n)
    Pe, Pi = P.subgroup(ne), P.subgroup(n - ne)
    Ce = b.Connection(Pe, P, "ge")
    Ce.connect_random(Pe, P, p, weight=1.62 * mV, seed=seed)
    Ci = b.Connection(Pi, P, "gi")
    Ci.connect_random(Pi, P, p, weight=-9 * mV, seed=seed + 1)
    rng = np.random.Generator(np.random.PCG64(seed + 2))
    P.v = Vr + rng.random(n) * (Vt - Vr)
    M = b.SpikeMonitor(P)
    S = b.StateMonitor(P, "v", record=list(range(record)))
    net = b.Network(P, Ce, Ci, M, S)
    return net, P, M, S


def cuba_scaled_inputs(seed, n=262144, indegree=1000, builder=None):
    """Host arrays of the scaled CUBA network: CSR rows of both connections
    (fixed in-degree, drawn by `builder(n_src, n_tgt, k, seed)`, by default
    the engine's host-side bg_fixed_indegree_csr), u8 delays and v0."""
    ne = int(0.8 * n)
    ke = int(0.8 * indegree)
    if builder is None:
        from ._lib import fixed_indegree_csr_native as builder
    rng = np.random.Generator(np.random.PCG64(seed))
    exc = builder(ne, n, ke, seed * 2 + 1)
    inh = builder(n - ne, n, indegree - ke, seed * 2 + 2)
    d_exc = rng.integers(1, 51, size=len(exc[1]), dtype=np.uint8)
    d_inh = rng.integers(1, 51, size=len(inh[1]), dtype=np.uint8)
    v0 = -60e-3 + rng.random(n) * (-50e-3 - -60e-3)
    return dict(n=n, ne=ne, exc=exc, inh=inh, d_exc=d_exc, d_inh=d_inh, v0=v0)


def cuba_scaled(inp, spike_monitor=False, record=None):
    """The scaled CUBA network of `inp`: returns (net, P, (Ce, Ci), M, S); M a
    SpikeMonitor on the whole group when asked, S a StateMonitor of v on the
    neurons `record` when given."""
    b = _b()
    eqs = b.Equations(CUBA_EQS, taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    P = b.NeuronGroup(inp["n"], model=eqs, threshold=-50 * mV, reset=-60 * mV)
    Pe = P.subgroup(inp["ne"])
    Pi = P.subgroup(inp["n"] - inp["ne"])
    Ce = b.DelayConnection(Pe, P, "ge", max_delay=5 * ms, dtype=np.float32)
    Ce.connect_csr(inp["exc"][0], inp["exc"][1], np.float32(0.162e-3), delay_steps=inp["d_exc"])
    Ci = b.DelayConnection(Pi, P, "gi", max_delay=5 * ms, dtype=np.float32)
    Ci.connect_csr(inp["inh"][0], inp["inh"][1], np.float32(-0.9e-3), delay_steps=inp["d_inh"])
    P.v = inp["v0"]
    objs = [P, Ce, Ci]
    M = S = None
    if spike_monitor:
        M = b.SpikeMonitor(P)
        objs.append(M)
    if record is not None:
        S = b.StateMonitor(P, "v", record=list(record))
        objs.append(S)
    return b.Network(*objs), P, (Ce, Ci), M, S


def stdp_scaleup(seed=2024, nin=10000, nout=4096, gmax=0.01, rate_lo=5.0, rate_hi=25.0, spike_record=0,
                 record=None, input_monitor=False, out_range=None):
    """The STDP scale-up network.  Returns a dict with the network and its
    objects: net, inputs, outputs, C (dense Connection), stdp, M (SpikeMonitor
    of the first `spike_record` outputs, or None), S (StateMonitor of v on
    the outputs `record`, or None), Mi (SpikeMonitor of the inputs when
    asked), w0 (the initial weights, float64).

    out_range=(lo, hi) builds the shard of outputs [lo, hi): the same inputs
    (the Poisson spikes are a function of (seed, step, index), so every
    shard draws them alike) onto those outputs with their columns of the
    full network's initial weights.  The outputs do not interact, so the
    shards of a partition together run exactly the full network."""
    b = _b()
    eqs = b.Equations(STDP_EQS, taum=10 * ms, taue=5 * ms, Ee=0 * mV, vr=-60 * mV, El=-74 * mV)
    rng = np.random.Generator(np.random.PCG64(seed))
    rates = rng.uniform(rate_lo, rate_hi, nin)
    inputs = b.PoissonGroup(nin, rates=rates, seed=seed + 1)
    lo, hi = (0, nout) if out_range is None else out_range
    outputs = b.NeuronGroup(hi - lo, model=eqs, threshold=-54 * mV, reset=-60 * mV)
    outputs.v = -60 * mV
    w0 = rng.uniform(0, gmax, (nin, nout))[:, lo:hi]
    C = b.Connection(inputs, outputs, "ge", structure="dense", dtype=np.float32)
    C.connect(W=w0)
    stdp = b.ExponentialSTDP(C, 20 * ms, 20 * ms, 0.01, -0.0105, wmax=gmax)
    objs = [inputs, outputs, C, stdp]
    M = S = Mi = None
    if spike_record:
        M = b.SpikeMonitor(outputs.subgroup(spike_record))
        objs.append(M)
    if record is not None:
        S = b.StateMonitor(outputs, "v", record=list(record))
        objs.append(S)
    if input_monitor:
        Mi = b.SpikeMonitor(inputs)
        objs.append(Mi)
    return dict(net=b.Network(*objs), inputs=inputs, outputs=outputs, C=C, stdp=stdp, M=M, S=S, Mi=Mi, w0=w0,
                rates=rates, gmax=gmax)
