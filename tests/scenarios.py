"""Network scenarios shared by the oracle tests and the GPU parity tests.

Each function builds a network with the public API, runs it on whatever
engine is active (``brian_b200.network.engine``) and returns plain arrays.
"""
import numpy as np

import brian_b200 as b
from brian_b200 import ms, mV, second, Hz
from brian_b200.connections import fixed_indegree_csr


def _result(net, groups=(), spikemons=(), statemons=(), conns=(), stdps=()):
    out = {}
    for k, g in enumerate(groups):
        for v in g._names:
            out["g%d.%s" % (k, v)] = np.array(getattr(g, v))
    for k, m in enumerate(spikemons):
        s, i = m._record()
        out["spk%d.steps" % k] = s.copy()
        out["spk%d.idx" % k] = i.copy()
    for k, m in enumerate(statemons):
        s, v = m._record()
        out["st%d.steps" % k] = s.copy()
        out["st%d.vals" % k] = v.copy()
    for k, c in enumerate(conns):
        out["w%d" % k] = c._weights().astype(np.float64).copy()
    for k, s in enumerate(stdps):
        a, p = s._traces()
        out["stdp%d.pre" % k] = a.copy()
        out["stdp%d.post" % k] = p.copy()
    return out


def cuba(N=4000, steps=10000, seed=1, p=0.02, record=10, refractory=0.0, runs=1, timestep=1, persistent=True):
    """Config 1: CUBA-4000, FP64, zero delay (examples/misc/CUBA.py:25-74);
    `runs` > 1 splits the steps into that many equal run() calls; `record`
    is the number of leading neurons whose v is recorded, or their list;
    `timestep` the StateMonitor's recording period in steps.  Without
    refractoriness the engine runs it in its persistent kernel unless
    `persistent` is False."""
    taum, taue, taui = 20 * ms, 5 * ms, 10 * ms
    Vt, Vr, El = -50 * mV, -60 * mV, -49 * mV
    eqs = b.Equations("""
    dv/dt  = (ge+gi-(v-El))/taum : volt
    dge/dt = -ge/taue : volt
    dgi/dt = -gi/taui : volt
    """, taum=taum, taue=taue, taui=taui, El=El)
    P = b.NeuronGroup(N, model=eqs, threshold=Vt, reset=Vr, refractory=refractory)
    Ne = int(0.8 * N)
    Pe = P.subgroup(Ne)
    Pi = P.subgroup(N - Ne)
    we, wi = 1.62 * mV, -9 * mV
    Ce = b.Connection(Pe, P, "ge")
    Ce.connect_random(Pe, P, p, weight=we, seed=seed)
    Ci = b.Connection(Pi, P, "gi")
    Ci.connect_random(Pi, P, p, weight=wi, seed=seed + 1)
    rng = np.random.Generator(np.random.PCG64(seed + 2))
    P.v = Vr + rng.random(N) * (Vt - Vr)
    M = b.SpikeMonitor(P)
    S = b.StateMonitor(P, "v", record=list(range(record)) if np.isscalar(record) else list(record),
                       timestep=timestep)
    net = b.Network(P, Ce, Ci, M, S)
    assert steps % runs == 0
    prev = b.get_global_preference("persistent")
    b.set_global_preferences(persistent=persistent)
    try:
        for _ in range(runs):
            net.run(steps // runs * 0.1 * ms)
    finally:
        b.set_global_preferences(persistent=prev)
    out = _result(net, groups=[P], spikemons=[M], statemons=[S])
    out["persistent_threads"] = net.stats().get("persistent_threads", 0)
    return out


def cuba_delay(N=3000, indegree=100, steps=2000, seed=3, wdtype=np.float32, we=0.162e-2, wi=-0.9e-2,
               hetero_weights=False, monitors=True, dmin=1, runs=1, persistent=True, coupled=False,
               burst=False):
    """Config 2 in miniature: fixed in-degree (80% exc / 20% inh), integer
    delays uniform in 1..50 steps, DelayConnections into ge and gi."""
    taum, taue, taui = 20 * ms, 5 * ms, 10 * ms
    Vt, Vr, El = -50 * mV, -60 * mV, -49 * mV
    # coupled: gi is also driven by ge, so the update matrix is not "first
    # row full, the rest diagonal"
    eqs = b.Equations("""
    dv/dt  = (ge+gi-(v-El))/taum : volt
    dge/dt = -ge/taue : volt
    dgi/dt = %s/taui : volt
    """ % ("(0.25*ge-gi)" if coupled else "-gi"), taum=taum, taue=taue, taui=taui, El=El)
    P = b.NeuronGroup(N, model=eqs, threshold=Vt, reset=Vr)
    Ne = int(0.8 * N)
    Pe, Pi = P.subgroup(Ne), P.subgroup(N - Ne)
    ke = int(0.8 * indegree)
    rng = np.random.Generator(np.random.PCG64(seed))
    conns = []
    for src, n, k, w, var, sd in ((Pe, Ne, ke, we, "ge", seed + 10), (Pi, N - Ne, indegree - ke, wi, "gi", seed + 20)):
        rowptr, cols = fixed_indegree_csr(n, N, k, seed=sd)
        d = rng.integers(dmin, 51, size=len(cols)).astype(np.uint8)
        C = b.DelayConnection(src, P, var, max_delay=5 * ms, dtype=wdtype)
        wv = (w * (0.5 + rng.random(len(cols)))) if hetero_weights else w
        C.connect_csr(rowptr, cols, wv, delay_steps=d)
        conns.append(C)
    P.v = Vr + rng.random(N) * (Vt - Vr)
    if burst:
        # every neuron a hair below threshold: the whole group fires within
        # the first steps, far more spikes per block and step than one batch
        P.v = Vt - 1e-7 * rng.random(N)
    if not monitors or monitors == "spikes":
        # no monitors (or spike monitors only): the engine may take its
        # persistent single-launch path
        prev = b.get_global_preference("persistent")
        b.set_global_preferences(persistent=persistent)
        # monitors="spikes": spike monitors only (the whole group and the
        # inhibitory subgroup), which the persistent kernel records itself
        mons = [b.SpikeMonitor(P), b.SpikeMonitor(Pi)] if monitors == "spikes" else []
        try:
            net = b.Network(P, conns[0], conns[1], *mons)
            for _ in range(runs):
                net.run(steps * 0.1 * ms / runs)
        finally:
            b.set_global_preferences(persistent=prev)
        out = _result(net, groups=[P], spikemons=mons)
        g, c = net._binding.rt.counters(1, 2)
        out["spikes"], out["events"] = g.copy(), c.copy()
        st = net.stats()
        out["launches"] = st["launches"]
        out["persistent_threads"] = st.get("persistent_threads", 0)
        return out
    M = b.SpikeMonitor(P)
    S = b.StateMonitor(P, "v", record=[0, 1, N - 1])
    net = b.Network(P, conns[0], conns[1], M, S)
    net.run(steps * 0.1 * ms)
    return _result(net, groups=[P], spikemons=[M], statemons=[S])


def cuba_large(N=200000, indegree=1000, steps=300, seed=2024, runs=1, precision=64):
    """The benchmark network at scale: N LIF neurons (80 % exc / 20 % inh),
    fixed in-degree `indegree` (80 % exc), f32 shared weights 0.162 mV /
    -0.9 mV, u8 delays uniform in 1..50 steps, seeded v0 in [Vr, Vt] (the
    CUBA-262k construction), a SpikeMonitor on the whole group; connectivity
    drawn by the engine's host-side builder (the same on both engines)."""
    from brian_b200._lib import fixed_indegree_csr_native
    ne = int(0.8 * N)
    ke = int(0.8 * indegree)
    rng = np.random.Generator(np.random.PCG64(seed))
    exc = fixed_indegree_csr_native(ne, N, ke, seed * 2 + 1)
    inh = fixed_indegree_csr_native(N - ne, N, indegree - ke, seed * 2 + 2)
    d_exc = rng.integers(1, 51, size=len(exc[1]), dtype=np.uint8)
    d_inh = rng.integers(1, 51, size=len(inh[1]), dtype=np.uint8)
    v0 = -60e-3 + rng.random(N) * (-50e-3 - -60e-3)
    eqs = b.Equations("""
    dv/dt  = (ge+gi-(v-El))/taum : volt
    dge/dt = -ge/taue : volt
    dgi/dt = -gi/taui : volt
    """, taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    P = b.NeuronGroup(N, model=eqs, threshold=-50 * mV, reset=-60 * mV)
    Pe, Pi = P.subgroup(ne), P.subgroup(N - ne)
    Ce = b.DelayConnection(Pe, P, "ge", max_delay=5 * ms, dtype=np.float32)
    Ce.connect_csr(exc[0], exc[1], np.float32(0.162e-3), delay_steps=d_exc)
    Ci = b.DelayConnection(Pi, P, "gi", max_delay=5 * ms, dtype=np.float32)
    Ci.connect_csr(inh[0], inh[1], np.float32(-0.9e-3), delay_steps=d_inh)
    P.v = v0
    M = b.SpikeMonitor(P)
    net = b.Network(P, Ce, Ci, M)
    for _ in range(runs):
        net.run(steps // runs * 0.1 * ms)
    out = _result(net, groups=[P], spikemons=[M])
    g, c = net._binding.rt.counters(1, 2)
    out["spikes"], out["events"] = g.copy(), c.copy()
    st = net.stats()
    out["launches"] = st["launches"]
    out["persistent_threads"] = st.get("persistent_threads", 0)
    net._invalidate()
    return out


def coba(N=2000, steps=2000, seed=7, method=None, implicit=False, order=1, string_threshold=True,
         string_reset=True, delays=True, empirical=False, linear=False):
    """A conductance-based (nonlinear) network: v driven by ge*(Ee-v) and
    gi*(Ei-v), integrated by the generated scheme of `method`/`implicit`/
    `order`; a condition string threshold and a two-statement string reset,
    or EmpiricalThreshold with no reset; sparse excitatory and (delayed)
    inhibitory connections; spike and state monitors."""
    taum, taue, taui = 20 * ms, 5 * ms, 10 * ms
    Ee, Ei, El, Vt, Vr = 0 * mV, -80 * mV, -49 * mV, -50 * mV, -60 * mV
    # linear: current-based instead (exact update, generated threshold/reset)
    eqs = b.Equations("""
    dv/dt  = (%s + (El-v))/taum : volt
    dge/dt = -ge/taue : 1
    dgi/dt = -gi/taui : 1
    """ % ("0.01*ge*volt - 0.04*gi*volt" if linear else "ge*(Ee-v) + gi*(Ei-v)"),
                       taum=taum, taue=taue, taui=taui, Ee=Ee, Ei=Ei, El=El, volt=1.0)
    if empirical:
        thr, rst = b.EmpiricalThreshold(threshold=Vt, refractory=3 * ms), None
    else:
        thr = "v > Vt + 2*mV*ge" if string_threshold else Vt
        rst = "v = Vr\nge = ge*0.5" if string_reset else Vr
    P = b.NeuronGroup(N, model=eqs, threshold=thr, reset=rst, method=method, implicit=implicit, order=order)
    Ne = int(0.8 * N)
    Pe, Pi = P.subgroup(Ne), P.subgroup(N - Ne)
    rng = np.random.Generator(np.random.PCG64(seed))
    rowe, cole = fixed_indegree_csr(Ne, N, 40, seed=seed + 1)
    rowi, coli = fixed_indegree_csr(N - Ne, N, 10, seed=seed + 2)
    Ce = b.Connection(Pe, P, "ge")
    Ce.connect_csr(rowe, cole, 0.05 * (0.5 + rng.random(len(cole))))
    if delays:
        Ci = b.DelayConnection(Pi, P, "gi", max_delay=2 * ms)
        Ci.connect_csr(rowi, coli, 0.2, delay_steps=rng.integers(1, 21, len(coli)).astype(np.uint8))
    else:
        Ci = b.Connection(Pi, P, "gi")
        Ci.connect_csr(rowi, coli, 0.2)
    P.v = Vr + rng.random(N) * (Vt - Vr + 2 * mV)
    M = b.SpikeMonitor(P)
    S = b.StateMonitor(P, "v", record=[0, 1, N - 1])
    net = b.Network(P, Ce, Ci, M, S)
    net.run(steps * 0.1 * ms)
    return _result(net, groups=[P], spikemons=[M], statemons=[S])


def cobahh(steps=10000):
    """The reference's COBAHH regression (dev/tests/correctness/
    test_optimizations.py:58-128): 4000 Hodgkin-Huxley neurons, exponential
    Euler (implicit=True), EmpiricalThreshold(-20 mV, 3 ms), the fixed 0/1
    excitatory/inhibitory matrices of tests/golden/cobahh.npz, deterministic
    initial state; returns the spike monitor's (steps, indices)."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cobahh.npz"))
    nS, msiemens, ufarad, umetre, cm, siemens = 1e-9, 1e-3, 1e-6, 1e-6, 1e-2, 1.0
    area = 20000 * umetre ** 2
    Cm = (1 * ufarad * cm ** -2) * area
    gl = (5e-5 * siemens * cm ** -2) * area
    El, EK, ENa = -60 * mV, -90 * mV, 50 * mV
    g_na = (100 * msiemens * cm ** -2) * area
    g_kd = (30 * msiemens * cm ** -2) * area
    VT = -63 * mV
    taue, taui = 5 * ms, 10 * ms
    Ee, Ei = 0 * mV, -80 * mV
    eqs = b.Equations("""
    dv/dt = (gl*(El-v)+ge*(Ee-v)+gi*(Ei-v)-g_na*(m*m*m)*h*(v-ENa)-g_kd*(n*n*n*n)*(v-EK))/Cm : volt
    dm/dt = alpham*(1-m)-betam*m : 1
    dn/dt = alphan*(1-n)-betan*n : 1
    dh/dt = alphah*(1-h)-betah*h : 1
    dge/dt = -ge*(1./taue) : siemens
    dgi/dt = -gi*(1./taui) : siemens
    alpham = 0.32*(mV**-1)*(13*mV-v+VT)/(exp((13*mV-v+VT)/(4*mV))-1.)/ms : Hz
    betam = 0.28*(mV**-1)*(v-VT-40*mV)/(exp((v-VT-40*mV)/(5*mV))-1)/ms : Hz
    alphah = 0.128*exp((17*mV-v+VT)/(18*mV))/ms : Hz
    betah = 4./(1+exp((40*mV-v+VT)/(5*mV)))/ms : Hz
    alphan = 0.032*(mV**-1)*(15*mV-v+VT)/(exp((15*mV-v+VT)/(5*mV))-1.)/ms : Hz
    betan = .5*exp((10*mV-v+VT)/(40*mV))/ms : Hz
    """, gl=gl, El=El, Ee=Ee, Ei=Ei, g_na=g_na, ENa=ENa, g_kd=g_kd, EK=EK, Cm=Cm, VT=VT, taue=taue, taui=taui)
    P = b.NeuronGroup(4000, model=eqs, threshold=b.EmpiricalThreshold(threshold=-20 * mV, refractory=3 * ms),
                      implicit=True, freeze=True)
    Pe, Pi = P.subgroup(3200), P.subgroup(800)
    Ce = b.Connection(Pe, P, "ge")
    Ce.connect_csr(g["ce_rowptr"], g["ce_cols"].astype(np.int32), 6 * nS)
    Ci = b.Connection(Pi, P, "gi")
    Ci.connect_csr(g["ci_rowptr"], g["ci_cols"].astype(np.int32), 67 * nS)
    x = np.arange(4000, dtype=float) / 4000
    P.v = El + ((x - 0.5) * 20 - 5) * mV
    P.ge = ((x - 0.5) * 6 + 4) * 10. * nS
    P.gi = ((x - 0.5) * 48 + 20) * 10. * nS
    M = b.SpikeMonitor(P)
    net = b.Network(P, Ce, Ci, M)
    net.run(steps * 0.1 * ms)
    s, i = M._record()
    return {"steps": s.copy(), "idx": i.copy(), "golden_steps": g["spk_step"], "golden_idx": g["spk_i"]}


def _stdp_rule(C, gmax, general, interactions="all", update="additive"):
    """ExponentialSTDP, or the same rule written as STDP code strings."""
    if not general:
        return b.ExponentialSTDP(C, 20 * ms, 20 * ms, 0.01, -0.0105, wmax=gmax, interactions=interactions,
                                 update=update)
    taup = taum = 20 * ms
    dA_pre, dA_post = 0.01 * gmax, -0.0105 * gmax
    eqs = b.Equations("""
    dA_pre/dt = -A_pre/taup : 1
    dA_post/dt = -A_post/taum : 1""", taup=taup, taum=taum)
    op_pre = "+=" if interactions in ("all", "nearest_post") else "="
    op_post = "+=" if interactions == "all" else "="
    return b.STDP(C, eqs, pre="A_pre %s dA_pre; w += A_post" % op_pre,
                  post="A_post %s dA_post\nw += A_pre" % op_post, wmax=gmax)


def stdp(Nin=400, Nout=32, steps=3000, seed=5, dense=True, rate_lo=5.0, rate_hi=25.0, wdtype=np.float32,
         general=False, update="additive"):
    """Config 3 in miniature: Poisson inputs -> LIF outputs, all-to-all,
    ExponentialSTDP (examples/plasticity/STDP1.py)."""
    taum, taue = 10 * ms, 5 * ms
    Ee, vt, vr, El = 0 * mV, -54 * mV, -60 * mV, -74 * mV
    gmax = 0.01
    eqs = b.Equations("""
    dv/dt=(ge*(Ee-vr)+El-v)/taum : volt
    dge/dt=-ge/taue : 1
    """, taum=taum, taue=taue, Ee=Ee, vr=vr, El=El)
    rng = np.random.Generator(np.random.PCG64(seed))
    inp = b.PoissonGroup(Nin, rates=rng.uniform(rate_lo, rate_hi, Nin) * 20, seed=seed)
    out = b.NeuronGroup(Nout, model=eqs, threshold=vt, reset=vr)
    out.v = vr
    W0 = rng.uniform(0, gmax, (Nin, Nout))
    C = b.Connection(inp, out, "ge", structure="dense" if dense else "sparse", dtype=wdtype)
    if dense:
        C.connect(W=W0)
    else:
        mask = rng.random((Nin, Nout)) < 0.5
        C.connect(W=W0 * mask)
    S = _stdp_rule(C, gmax, general, update=update)
    C.compress()
    w_init = C._weights().astype(np.float64).copy()
    M = b.SpikeMonitor(out)
    Mi = b.SpikeMonitor(inp)
    net = b.Network(inp, out, C, S, M, Mi)
    net.run(steps * 0.1 * ms)
    res = _result(net, groups=[out], spikemons=[M, Mi], conns=[C], stdps=[S])
    res["w_init"], res["decay"] = w_init, np.array(S.decay)
    return res


def stdp_delay(Nin=400, Nout=40, steps=3000, seed=9, p=0.5, wdtype=np.float64, interactions="all", runs=1,
               rate_lo=5.0, rate_hi=25.0, general=False, update="additive"):
    """ExponentialSTDP on a DelayConnection: Poisson inputs -> LIF outputs
    through float delays (seconds) uniform below max_delay = 5 ms, so that
    the per-synapse lags int((1/dt)*(max_delay-d)) and int((1/dt)*d) are
    not complements of each other.  Also returns the connectivity and the
    initial weights (CSR order) for replays of the rule."""
    taum, taue = 10 * ms, 5 * ms
    Ee, vt, vr, El = 0 * mV, -54 * mV, -60 * mV, -74 * mV
    gmax = 0.01
    eqs = b.Equations("""
    dv/dt=(ge*(Ee-vr)+El-v)/taum : volt
    dge/dt=-ge/taue : 1
    """, taum=taum, taue=taue, Ee=Ee, vr=vr, El=El)
    rng = np.random.Generator(np.random.PCG64(seed))
    inp = b.PoissonGroup(Nin, rates=rng.uniform(rate_lo, rate_hi, Nin) * 20, seed=seed)
    out = b.NeuronGroup(Nout, model=eqs, threshold=vt, reset=vr)
    out.v = vr
    mask = rng.random((Nin, Nout)) < p
    W0 = rng.uniform(0, gmax, (Nin, Nout)) * mask
    D = rng.uniform(0.0, 4.99e-3, (Nin, Nout))
    C = b.DelayConnection(inp, out, "ge", max_delay=5 * ms, dtype=wdtype)
    C.connect(inp, out, W0, delay=D)
    S = _stdp_rule(C, gmax, general, interactions, update)
    C.compress()
    extra = {"rowptr": np.array(C._rowptr), "cols": np.array(C._cols), "d": C._delay_seconds().copy(),
             "w_init": C._weights().astype(np.float64).copy(), "decay": np.array(S.decay)}
    M = b.SpikeMonitor(out)
    Mi = b.SpikeMonitor(inp)
    net = b.Network(inp, out, C, S, M, Mi)
    for _ in range(runs):
        net.run(steps * 0.1 * ms / runs)
    res = _result(net, groups=[out], spikemons=[M, Mi], conns=[C], stdps=[S])
    res.update(extra)
    return res


def synapses_cuba(N=2000, steps=2000, seed=11, p=0.02, runs=1, two_statements=True, multi=True,
                  report_persistent=False):
    """CUBA through Synapses: excitatory and inhibitory subgroups onto the
    whole group with per-synapse weights and float delays (0-4 ms); the
    excitatory code has two statements; some pairs get two synapses.
    `report_persistent` adds the threads per block of the engine's
    persistent kernel (0: the stepped path ran)."""
    taum, taue, taui = 20 * ms, 5 * ms, 10 * ms
    Vt, Vr, El = -50 * mV, -60 * mV, -49 * mV
    eqs = b.Equations("""
    dv/dt  = (ge+gi-(v-El))/taum : volt
    dge/dt = -ge/taue : volt
    dgi/dt = -gi/taui : volt
    """, taum=taum, taue=taue, taui=taui, El=El)
    P = b.NeuronGroup(N, model=eqs, threshold=Vt, reset=Vr)
    Ne = int(0.8 * N)
    Pe, Pi = P.subgroup(Ne), P.subgroup(N - Ne)
    rng = np.random.Generator(np.random.PCG64(seed))
    pre_e = "ge += w\nv += 0.05*w" if two_statements else "ge += w"
    Se = b.Synapses(Pe, P, model="w : volt", pre=pre_e, max_delay=5 * ms)
    Si = b.Synapses(Pi, P, model="w : volt", pre="gi -= w")
    Se.connect_random(sparseness=p)
    Si.connect_random(sparseness=p)
    if multi:
        Se[0:20, 0:20] = 2          # pairs with two synapses
    Se.w = 1.62 * mV * (0.5 + rng.random(len(Se)))
    Si.w = 9 * mV * (0.5 + rng.random(len(Si)))
    Se.delay = rng.random(len(Se)) * 4 * ms
    Si.delay = rng.random(len(Si)) * 4 * ms
    P.v = Vr + rng.random(N) * (Vt - Vr)
    M = b.SpikeMonitor(P)
    S = b.StateMonitor(P, "v", record=[0, 1, N - 1])
    net = b.Network(P, Se, Si, M, S)
    for _ in range(runs):
        net.run(steps * 0.1 * ms / runs)
    out = _result(net, groups=[P], spikemons=[M], statemons=[S])
    if report_persistent:
        out["persistent_threads"] = net.stats().get("persistent_threads", 0)
    return out


def kitchen_sink(steps=400, seed=7):
    """Refractoriness, variable threshold/reset, homogeneous delays,
    modulation, dense structure, generators and subgroup monitors."""
    rng = np.random.Generator(np.random.PCG64(seed))
    N = 300
    eqs = b.Equations("""
    dv/dt = (I - v)/tau : volt
    dI/dt = -I/taus : volt
    dvt/dt = (vt0 - vt)/taut : volt
    """, tau=10 * ms, taus=3 * ms, taut=30 * ms, vt0=-50 * mV)
    G = b.NeuronGroup(N, model=eqs, threshold=b.VariableThreshold("vt", "v"), reset=-65 * mV,
                      refractory=2 * ms)
    G.v = -65 * mV + rng.random(N) * 20 * mV
    G.vt = -50 * mV
    G.I = rng.random(N) * 40 * mV
    spk = [(int(i), float(t)) for i, t in zip(rng.integers(0, 50, 600), rng.random(600) * steps * 0.1 * ms)]
    gen = b.SpikeGeneratorGroup(50, spk)
    H = b.NeuronGroup(40, model="dx/dt = -x/(5*ms) : 1\nm : 1", threshold=0.5, reset=b.VariableReset("m", "x"))
    H.x = rng.random(40)
    H.m = rng.random(40) * 0.1
    C1 = b.Connection(gen, G, "I", weight=3 * mV, sparseness=0.3)
    C2 = b.Connection(G, G, "v", delay=1.5 * ms)
    C2.connect_random(G, G, 0.05, weight=lambda i, j: 0.1 * mV * (1 + (i % 7) + (j % 5)), seed=seed)
    C3 = b.Connection(gen, H, "x", structure="dense", weight=rng.random((50, 40)) * 0.2)
    C4 = b.Connection(H, G[100:200], "vt", modulation="m", weight=0.5 * mV, sparseness=0.2)
    C5 = b.DelayConnection(G[:150], H, "x", max_delay=3 * ms)
    C5.connect_random(G[:150], H, 0.1, weight=0.05, seed=seed + 1, delay=(0.1 * ms, 2.9 * ms))
    M1 = b.SpikeMonitor(G)
    M2 = b.SpikeMonitor(G[50:120])
    M3 = b.SpikeMonitor(H, delay=1 * ms)
    S1 = b.StateMonitor(G, "v", record=[3, 0, 250], timestep=3)
    S2 = b.StateMonitor(H, "x", record=True)
    net = b.Network(G, gen, H, C1, C2, C3, C4, C5, M1, M2, M3, S1, S2)
    net.run(steps * 0.05 * ms)
    net.run(steps * 0.05 * ms)
    return _result(net, groups=[G, H], spikemons=[M1, M2, M3], statemons=[S1, S2], conns=[C1, C2, C3, C4, C5])


def compare(a, b_, exact=True):
    """Assert two scenario results agree: identical spikes and steps,
    states equal bit for bit (+0 == -0)."""
    assert set(a) == set(b_), (set(a) ^ set(b_))
    for k in sorted(a):
        x, y = np.asarray(a[k]), np.asarray(b_[k])
        assert x.shape == y.shape, (k, x.shape, y.shape)
        if exact or x.dtype.kind in "iu":
            if not np.array_equal(x, y):
                bad = np.argwhere(x != y)
                raise AssertionError("%s differs at %d positions, first %s: %r vs %r"
                                     % (k, len(bad), bad[0], x[tuple(bad[0])], y[tuple(bad[0])]))
        else:
            np.testing.assert_allclose(x, y, rtol=1e-12, atol=0, err_msg=k)
