"""GPU parity of the batched fitting kernel, gamma and the device swarm
against the numpy oracle (oracle/fitting.py)."""
import numpy as np
import pytest

from brian_b200 import Equations, NeuronGroup, GPUModelFitting, modelfitting, get_spikes, predict
from brian_b200._lib import FitHandle
from brian_b200.codegen import generate_model_code
from brian_b200.statistics import firing_rate
from brian_b200.synthetic import ADAPTIVE_LIF, THRESHOLD, RESET, PARAMS, sample_prior, ou_current
from oracle import fitting as of

pytestmark = pytest.mark.gpu
DT = 1e-4


def _eqs():
    return Equations(ADAPTIVE_LIF, dummy=0.0)


def _case(ns, rng, minlen=2000, maxlen=12000, ntr=60):
    """ns simulations of the adaptive model with random parameters, uneven
    lengths, own OU inputs, random target trains, delays and refractory."""
    state = ["V", "Vt", "R", "tau", "Vt0", "alpha", "tau_t"]
    P = sample_prior(ns, rng)
    S0 = np.zeros((len(state), ns))
    for d, k in enumerate(PARAMS):
        S0[state.index(k)] = P[d]
    S0[1] = S0[4] * rng.uniform(0.8, 1.2, ns)
    nsteps = rng.integers(minlen, maxlen + 1, ns)
    I = np.concatenate([ou_current(int(n), DT, rng) for n in nsteps])
    I_off = np.concatenate([[0], np.cumsum(nsteps)[:-1]])
    trains, offs, ends, pos = [], [], [], 0
    for i in range(ns):
        k = int(rng.integers(0, ntr))
        s = np.sort(rng.choice(int(nsteps[i]), size=k, replace=False))
        tr = np.concatenate([[-10000], s, [int(nsteps[i]) + 10000]])
        trains.append(tr)
        offs.append(pos)
        pos += len(tr)
        ends.append(pos)
    return dict(S0=S0, I=I, I_offset=I_off, nsteps=nsteps, spiketimes=np.concatenate(trains),
                spk_offset=np.array(offs), spk_end=np.array(ends), delay=rng.integers(-30, 31, ns),
                refractory=rng.integers(0, 6, ns))


def _device(code, c, precision, exclusive, delta=40, onset=0, record=0):
    h = FitHandle(code, DT, delta, exclusive=exclusive, precision=precision)
    h.set_input(c["I"])
    h.set_targets(c["spiketimes"])
    if record:
        h.set_record(record)
    h.set_sims(c["S0"], c["I_offset"], c["nsteps"], c["spk_offset"], c["spk_end"], c["delay"], c["refractory"],
               onset)
    return h


@pytest.mark.parametrize("precision,scheme,exclusive", [
    (64, "Euler", True), (32, "Euler", True), (64, "Euler", False), (32, "RK", True), (64, "RK", False)])
def test_fit_kernel_bit_exact(precision, scheme, exclusive):
    rng = np.random.default_rng(100 + precision)
    c = _case(160, rng)
    code = generate_model_code(_eqs(), THRESHOLD, RESET, DT, scalar="float" if precision == 32 else "double",
                               scheme=scheme)
    h = _device(code, c, precision, exclusive, onset=25)
    h.run(0, int(c["nsteps"].max()))
    coinc, nspk, S = h.read(state=True)
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float32 if precision == 32 else np.float64, scheme=scheme)
    r = of.simulate(m, c["S0"], c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"], c["spk_end"],
                    c["delay"], c["refractory"], delta=40, exclusive=exclusive, onset=25)
    assert nspk.sum() > 500
    assert np.array_equal(nspk, r["nspikes"])
    assert np.array_equal(coinc, r["coinc"])
    assert np.array_equal(S, r["state"])


def test_fit_kernel_exponential_euler_close():
    """exp() differs between libm and CUDA in the last ulp, so spike trains
    may drift apart after a near-threshold crossing: counts agree for most
    simulations and states stay close."""
    rng = np.random.default_rng(7)
    c = _case(128, rng)
    code = generate_model_code(_eqs(), THRESHOLD, RESET, DT, scalar="double", scheme="exponential_Euler")
    h = _device(code, c, 64, True)
    h.run(0, int(c["nsteps"].max()))
    coinc, nspk, S = h.read(state=True)
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float64, scheme="exponential_Euler")
    r = of.simulate(m, c["S0"], c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"], c["spk_end"],
                    c["delay"], c["refractory"], delta=40, exclusive=True)
    same = nspk == r["nspikes"]
    assert same.mean() >= 0.95
    assert np.mean(coinc == r["coinc"]) >= 0.95
    rel = np.abs(S[:, same] - r["state"][:, same]) / np.maximum(np.abs(r["state"][:, same]), 1e-12)
    assert np.median(rel) < 1e-9


def test_chunked_launches_and_recorded_spikes():
    rng = np.random.default_rng(3)
    c = _case(96, rng, minlen=3000, maxlen=9000)
    code = generate_model_code(_eqs(), THRESHOLD, RESET, DT, scalar="float")
    whole = _device(code, c, 32, True, record=400)
    whole.run(0, 9000)
    parts = _device(code, c, 32, True, record=400)
    for a in range(0, 9000, 2500):
        parts.run(a, min(a + 2500, 9000))
    a1, b1, s1 = whole.read(state=True)
    a2, b2, s2 = parts.read(state=True)
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2) and np.array_equal(s1, s2)
    cnt, steps = whole.read_spikes()
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float32)
    r = of.simulate(m, c["S0"], c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"], c["spk_end"],
                    c["delay"], c["refractory"], delta=40, exclusive=True, record=True)
    for i in range(96):
        assert list(steps[i, :cnt[i]]) == r["rec"][i]


def _gamma_inputs(c, npart):
    tl, tr = [], []
    for i in range(npart):
        s = c["spiketimes"][c["spk_offset"][i] + 1:c["spk_end"][i] - 1] * DT
        tl.append(len(s))
        tr.append(firing_rate(s))
    return np.array(tl), np.array(tr)


def test_evaluate_gamma_bit_exact():
    rng = np.random.default_rng(9)
    c = _case(128, rng, minlen=4000, maxlen=8000, ntr=80)
    code = generate_model_code(_eqs(), THRESHOLD, RESET, DT, scalar="double")
    h = _device(code, c, 64, True)
    tl, tr = _gamma_inputs(c, 128)
    h.set_gamma(128, 1, tl, tr, 4e-3)
    h.set_params([2, 3, 4, 5, 6, -1])          # R tau Vt0 alpha tau_t delays
    X = np.vstack([sample_prior(128, rng), rng.uniform(-2e-3, 2e-3, 128)])
    g = h.evaluate(X)
    S0 = c["S0"].copy()
    S0[2:7] = X[:5]
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float64)
    r = of.simulate(m, S0, c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"], c["spk_end"],
                    np.rint(X[5] / DT).astype(int), c["refractory"], delta=40, exclusive=True)
    ref = of.gamma(r["coinc"], r["nspikes"], tl, tr, 4e-3)
    assert np.array_equal(np.isnan(g), np.isnan(ref))
    assert np.array_equal(g[~np.isnan(g)], ref[~np.isnan(ref)])


def test_device_swarm_matches_oracle():
    rng = np.random.default_rng(21)
    G, gs = 2, 32
    M = G * gs
    c = _case(M, rng, minlen=2000, maxlen=2000, ntr=20)
    # one input and train per group
    for key in ("I_offset", "spk_offset", "spk_end", "nsteps"):
        c[key] = np.repeat(c[key][::gs][:G], gs)
    c["delay"] = np.zeros(M, int)
    c["refractory"] = np.zeros(M, int)
    code = generate_model_code(_eqs(), THRESHOLD, RESET, DT, scalar="float")
    h = _device(code, c, 32, True)
    tl, tr = _gamma_inputs(c, M)
    h.set_gamma(M, 1, tl, tr, 4e-3)
    h.set_params([2, 3, 4, 5, 6])
    lo = np.array([v[0] for v in [(2.5e7, 5e7), (5e-3, 2e-2), (1.5e-2, 2.5e-2), (2e-3, 1e-2), (5e-2, 2e-1)]])
    hi = lo * np.array([2, 4, 5 / 3, 5, 4])
    X0 = lo.reshape(-1, 1) + (hi - lo).reshape(-1, 1) * rng.random((5, M))
    h.pso_init(gs, X0, lo, hi, 0.7298, 1.49618, 1.49618, 77)
    trace, ms = h.pso_run(4)
    Xd, Vd, Xld, fld = h.pso_state()
    Xg, fg = h.pso_best()
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float32)

    def fun(X):
        S0 = c["S0"].copy()
        S0[2:7] = X
        r = of.simulate(m, S0, c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"], c["spk_end"],
                        None, None, delta=40, exclusive=True)
        return of.gamma(r["coinc"], r["nspikes"], tl, tr, 4e-3)

    Xg_o, fg_o, hist = of.pso_reference(X0, fun, 4, (0.7298, 1.49618, 1.49618), lo, hi, gs, seed=77)
    assert np.array_equal(Xd, hist[-1][0])
    assert np.array_equal(Vd, hist[-1][1])
    assert np.array_equal(Xg, Xg_o)
    assert np.array_equal(fg, fg_o)
    assert np.array_equal(trace, np.array([hh[3] for hh in hist]))
    assert ms.shape == (4,) and np.all(ms > 0)


@pytest.mark.parametrize("slices,overlap,algorithm", [(1, 0.0, None), (4, 0.05, None), (1, 0.0, "PSO")])
def test_modelfitting_recovers_targets(slices, overlap, algorithm):
    """End to end through modelfitting(): 4 targets with their own OU inputs
    and lengths; CMA-ES (the default, as in the reference) and the particle
    swarm find parameter sets with high gamma (also with each input cut into
    4 time slices simulated side by side)."""
    from brian_b200.modelfitting import PSO, CMAES
    from brian_b200.synthetic import FitWorkload
    w = FitWorkload(ntargets=4, dur_min=2.0, dur_max=3.0, seed=5)
    w.build_targets()
    pr = {"R": [2.5e7, 5e7], "tau": [5e-3, 2e-2], "Vt0": [1.5e-2, 2.5e-2], "alpha": [2e-3, 1e-2],
          "tau_t": [5e-2, 2e-1]}
    pr = {k: [v[0], v[0], v[1], v[1]] for k, v in pr.items()}
    res = modelfitting(model=_eqs(), reset=RESET, threshold=THRESHOLD, data=w.data(), input=w.inputs, dt=DT,
                       popsize=512, maxiter=25, delta=4e-3, precision="float", seed=3, slices=slices,
                       overlap=overlap, algorithm=PSO if algorithm == "PSO" else CMAES, **pr)
    assert res.info.get("algorithm", "PSO") == (algorithm or "CMAES")
    assert len(res.best_fit) == 4
    assert np.min(res.best_fit) > 0.5
    assert res.info["trace"].shape == (25, 4)
    # predict() re-simulates the fitted parameters against the targets
    g = predict(model=_eqs(), reset=RESET, threshold=THRESHOLD, data=w.targets[0], input=w.inputs[0], dt=DT,
                delta=4e-3, **res.best_pos[0])
    assert g > 0.4


def test_get_spikes_matches_oracle():
    rng = np.random.default_rng(4)
    P = sample_prior(6, rng)
    inputs = [ou_current(5000, DT, rng) for _ in range(6)]
    sp = get_spikes(model=_eqs(), reset=RESET, threshold=THRESHOLD, input=inputs, dt=DT,
                    **{k: P[d] for d, k in enumerate(PARAMS)})
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float64)
    S0 = np.zeros((7, 6))
    S0[2:7] = P
    spk = np.concatenate([[-10000, 20000]] * 6)
    r = of.simulate(m, S0, np.concatenate(inputs), np.arange(6) * 5000, np.full(6, 5000), spk, np.arange(6) * 2,
                    np.arange(6) * 2 + 2, record=True)
    got = [[int(round(t / DT)) for j, t in sp if j == i] for i in range(6)]
    assert got == [list(x) for x in r["rec"]]


def test_gpu_modelfitting_class_with_neurongroup():
    rng = np.random.default_rng(12)
    N = 64
    G = NeuronGroup(N, model=_eqs(), threshold=THRESHOLD, reset=RESET, method="Euler")
    P = sample_prior(N, rng)
    for d, k in enumerate(PARAMS):
        setattr(G, k, P[d])
    G.Vt = P[2]
    I = ou_current(6000, DT, rng)
    tgt = np.sort(rng.choice(6000, 30, replace=False)) * DT
    spk = np.concatenate([[-1.0], tgt, [1.6]])
    mf = GPUModelFitting(G, _eqs(), I, np.zeros(N, int), spk, np.zeros(N, int), np.zeros(N), 0.0, 4e-3)
    mf.launch(0.6, stepsize=0.1)
    total = int(0.6 / DT)           # the reference's step count for a duration
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float64)
    S0 = np.zeros((7, N))
    S0[1] = P[2]
    S0[2:7] = P
    r = of.simulate(m, S0, I, np.zeros(N, int), np.full(N, total), np.rint(spk / DT).astype(int), np.zeros(N, int),
                    np.full(N, len(spk)), delta=40, exclusive=True)
    assert np.array_equal(mf.coincidence_count, r["coinc"])
    assert np.array_equal(mf.spike_count, r["nspikes"])


@pytest.mark.parametrize("precision", [32, 64])
def test_reciprocal_division_falls_back_exactly(precision):
    """Divisions by run-constant divisors use reciprocal forms; dividends or
    quotients outside the range where those are exact (subnormal values,
    tiny quotients) make the kernel redo the block with IEEE division, zero
    dividends stay on the fast form, and zero / subnormal / infinite / NaN
    divisors send the whole simulation to IEEE division.  Every state must
    equal numpy's IEEE arithmetic bit for bit."""
    dtype = np.float32 if precision == 32 else np.float64
    tiny = 1e-36 if precision == 32 else 1e-300
    eqs = Equations("dV/dt = (a - V)/tau : 1\nI : 1\na : 1\ntau : 1", dummy=0.0)
    code = generate_model_code(eqs, "V > 1e30", "V = 0", DT, scalar="float" if precision == 32 else "double")
    assert code.update_fast and "bg_div_fast" in code.update_fast
    ns = 96
    rng = np.random.default_rng(8)
    V0 = np.concatenate([np.full(32, tiny), rng.uniform(-1, 1, 32), np.full(32, 0.25)])
    a = np.concatenate([np.zeros(32), rng.uniform(-1, 1, 32), np.full(32, 0.25)])   # a == V: zero dividends
    tau = np.concatenate([np.full(32, 1e-3), rng.uniform(1e-3, 1e-1, 32), np.full(32, 5e-3)])
    tau[[3, 40, 70]] = 0.0
    tau[[5, 41]] = 1e-40 if precision == 32 else 1e-320
    tau[[6, 42]] = np.inf
    tau[[7, 43]] = np.nan
    tau[44] = -0.0
    S0 = np.vstack([V0, a, tau])
    n = 3000
    c = dict(S0=S0, I=np.zeros(n), I_offset=np.zeros(ns, int), nsteps=np.full(ns, n),
             spiketimes=np.array([-10000, n + 10000]), spk_offset=np.zeros(ns, int), spk_end=np.full(ns, 2),
             delay=np.zeros(ns, int), refractory=np.zeros(ns, int))
    h = _device(code, c, precision, True)
    h.run(0, n)
    S = h.read(state=True)[2]
    m = of.ModelOracle(eqs, "V > 1e30", "V = 0", DT, dtype)
    with np.errstate(all="ignore"):
        r = of.simulate(m, S0, c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"], c["spk_end"])
    assert np.array_equal(S, r["state"], equal_nan=True)
    # the decaying tiny values did reach the subnormal range
    assert np.any((np.abs(r["state"][0, :32]) < np.finfo(dtype).tiny) & (r["state"][0, :32] != 0))


@pytest.mark.parametrize("slices,overlap", [(1, 0.0), (3, 5e-3), (4, 0.0)])
def test_time_slicing_matches_oracle(slices, overlap):
    """Time slicing (modelfitting.py:49-58, 126-163, 221-223): every slice
    of every candidate is simulated by the oracle from the input piece and
    the shifted target spikes the slicing rules give, counts are summed over
    the slices and gamma must equal the device's bit for bit."""
    from brian_b200.modelfitting import FittingProblem
    rng = np.random.default_rng(21)
    lens = [9001, 7003]                      # not multiples of the slice count
    inputs = [ou_current(n, DT, rng) for n in lens]
    data = [np.sort(rng.uniform(0, n * DT, 40)) for n in lens]
    pop = 16
    prob = FittingProblem(_eqs(), THRESHOLD, RESET, data, inputs, DT, pop, precision="double",
                          param_names=list(PARAMS), slices=slices, overlap=overlap)
    N = 2 * pop
    ov = int(overlap / DT) if slices > 1 else 0
    # the slicing rules restated: input pieces, offsets, steps and trains
    for j, (x, s) in enumerate(zip(inputs, data)):
        L = slices * (len(x) // slices)
        sl = L // slices
        piece = np.hstack((np.zeros(ov), x[:L]))
        base = prob.input_offsets[j]
        assert np.array_equal(prob.sim_input[base:base + len(piece)], piece)
        for k in range(slices):
            for p in range(pop):
                i = k * N + j * pop + p
                assert prob.sim_input_offsets[i] == base + k * sl
                assert prob.sim_nsteps[i] == (int((L * DT) / DT) if slices == 1 else sl + ov)
                inside = s[(s >= k * sl * DT) & (s < (k + 1) * sl * DT)]
                tr = np.hstack(([-1.0], inside - k * sl * DT + ov * DT, [overlap * (slices > 1) + L * DT / slices + 1.0]))
                got = prob.sim_trains[prob.sim_train_offsets[i]:prob.sim_train_ends[i]]
                assert np.array_equal(got, np.rint(tr / DT).astype(np.int32))
    X = sample_prior(N, rng)
    g = prob.evaluate(X)
    state = prob.code.state
    S0 = np.zeros((len(state), N * slices))
    for d, k in enumerate(PARAMS):
        S0[state.index(k)] = np.tile(X[d], slices)
    m = of.ModelOracle(_eqs(), THRESHOLD, RESET, DT, np.float64)
    r = of.simulate(m, S0, prob.sim_input, prob.sim_input_offsets, prob.sim_nsteps, prob.sim_trains,
                    prob.sim_train_offsets, prob.sim_train_ends, np.zeros(N * slices, dtype=int),
                    np.zeros(N * slices, dtype=int), delta=40, exclusive=True)
    nc = r["coinc"].reshape(slices, N).sum(axis=0)
    nm = r["nspikes"].reshape(slices, N).sum(axis=0)
    ref = of.gamma(nc, nm, prob.target_length, prob.target_rate, 4e-3)
    assert np.isfinite(ref).all() and nm.sum() > 100
    assert np.array_equal(g, ref)
    prob.handle.close()
