"""CPU checks of the fitting oracle, the model code generator and the NVRTC
build of the fitting kernel (no GPU needed)."""
import ctypes as ct
import os

import numpy as np
import pytest

from brian_b200 import Equations
from brian_b200.codegen import generate_model_code, CodegenError
from brian_b200.statistics import get_gamma_factor
from brian_b200.synthetic import ADAPTIVE_LIF, THRESHOLD, RESET, PARAMS, PRIOR, sample_prior, ou_current
from oracle import fitting as of

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def runsim_literal(model, S0, I, I_offset, nsteps, spk, spk_off, spk_end, delay, refr, delta, exclusive, onset):
    """Line-by-line transcription of the runsim template
    (gpu_modelfitting.py:39-156) for one simulation at a time, plain Python
    control flow; the model step comes from the oracle on 1-element arrays."""
    ns = S0.shape[1]
    out_c, out_n = [], []
    for i in range(ns):
        S = {v: np.array([S0[k, i]], dtype=model.dtype) for k, v in enumerate(model.state)}
        idx = int(spk_off[i])
        last_idx = int(spk_end[i]) - 1
        last_spike_time = int(spk[idx])
        next_spike_time = int(spk[idx + 1]) if idx < last_idx else 2 ** 31 - 1
        last_spike_allowed, next_spike_allowed = False, True
        ncoinc = nspikes = 0
        next_allowed_spiketime = -1
        for T in range(int(nsteps[i])):
            t = model.dtype(np.float64(T) * model.dt)
            Iv = np.array([I[I_offset[i] + T]], dtype=model.dtype)
            model.update(S, Iv, t)
            is_refractory = T <= next_allowed_spiketime
            has_spiked = bool(model.spiking(S, Iv, t)[0]) and not is_refractory
            nspikes += int(has_spiked and T >= onset)
            if has_spiked or is_refractory:
                model.apply_reset(S, Iv, t, np.array([True]))
            if has_spiked:
                next_allowed_spiketime = T + int(refr[i])
            Tspike = T + int(delay[i])
            if exclusive:
                near_last_spike = last_spike_time + delta >= Tspike
                near_next_spike = next_spike_time - delta <= Tspike
                near_last_spike = near_last_spike and has_spiked
                near_next_spike = near_next_spike and has_spiked
                ncoinc += int((near_last_spike and last_spike_allowed) or (near_next_spike and next_spike_allowed))
                near_both_allowed = (near_last_spike and last_spike_allowed) and (near_next_spike and
                                                                                  next_spike_allowed)
                last_spike_allowed = last_spike_allowed and not near_last_spike
                next_spike_allowed = (next_spike_allowed and not near_next_spike) or near_both_allowed
            else:
                ncoinc += int(has_spiked and ((last_spike_time + delta >= Tspike) or
                                              (next_spike_time - delta <= Tspike)))
            if Tspike >= next_spike_time:
                idx += 1
                last_spike_time = next_spike_time
                next_spike_time = int(spk[idx + 1]) if idx < last_idx else 2 ** 31 - 1
                if exclusive:
                    last_spike_allowed = next_spike_allowed
                    next_spike_allowed = True
        out_c.append(ncoinc)
        out_n.append(nspikes)
    return np.array(out_c), np.array(out_n)


def _adaptive(dtype, scheme="Euler"):
    eqs = Equations(ADAPTIVE_LIF, dummy=0.0)
    return of.ModelOracle(eqs, THRESHOLD, RESET, 1e-4, dtype, scheme=scheme)


def _random_case(model, ns, rng, maxlen=3000, minlen=500, with_delay=True, with_refr=True):
    P = sample_prior(ns, rng)
    S0 = np.zeros((len(model.state), ns))
    for d, k in enumerate(PARAMS):
        S0[model.state.index(k)] = P[d]
    S0[model.state.index("Vt")] = S0[model.state.index("Vt0")]
    nsteps = rng.integers(minlen, maxlen + 1, ns)
    I = np.concatenate([ou_current(int(n), 1e-4, rng) for n in nsteps])
    I_off = np.concatenate([[0], np.cumsum(nsteps)[:-1]])
    trains, offs, ends = [], [], []
    pos = 0
    for i in range(ns):
        k = rng.integers(0, 40)
        s = np.sort(rng.choice(int(nsteps[i]), size=k, replace=False))
        tr = np.concatenate([[-10000], s, [int(nsteps[i]) + 10000]])
        trains.append(tr)
        offs.append(pos)
        pos += len(tr)
        ends.append(pos)
    spk = np.concatenate(trains)
    delay = rng.integers(-30, 31, ns) if with_delay else np.zeros(ns, int)
    refr = rng.integers(0, 6, ns) if with_refr else np.zeros(ns, int)
    return dict(S0=S0, I=I, I_offset=I_off, nsteps=nsteps, spiketimes=spk, spk_offset=np.array(offs),
                spk_end=np.array(ends), delay=delay, refractory=refr)


@pytest.mark.parametrize("exclusive", [True, False])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_vectorised_oracle_matches_literal_transcription(exclusive, dtype):
    rng = np.random.default_rng(5)
    model = _adaptive(dtype)
    c = _random_case(model, 12, rng, maxlen=3000, minlen=1000)
    r = of.simulate(model, c["S0"], c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"],
                    c["spk_end"], c["delay"], c["refractory"], delta=40, exclusive=exclusive, onset=50)
    lc, ln = runsim_literal(model, c["S0"], c["I"], c["I_offset"], c["nsteps"], c["spiketimes"], c["spk_offset"],
                            c["spk_end"], c["delay"], c["refractory"], 40, exclusive, 50)
    assert np.array_equal(r["coinc"], lc)
    assert np.array_equal(r["nspikes"], ln)
    assert r["nspikes"].sum() > 30 and r["coinc"].sum() > 3


def _clock_model():
    # V grows by exactly 1/4 per step (dyadic arithmetic, no rounding) and
    # spikes when it exceeds 1: spikes at steps 4, 9, 14, ...
    eqs = Equations("dV/dt = I/tau : 1\nI : 1\ntau : 1", dummy=0.0)
    return of.ModelOracle(eqs, "V > 1", "V = 0", 0.25, np.float64)


def _clock_case(target_steps, nsteps=45, delay=0, refr=0):
    S0 = np.array([[0.0], [1.0]])          # V, tau
    spk = np.array([-10000] + list(target_steps) + [nsteps + 10000])
    return dict(S0=S0, I=np.ones(nsteps), I_offset=[0], nsteps=[nsteps], spiketimes=spk, spk_offset=[0],
                spk_end=[len(spk)], delay=[delay], refractory=[refr])


def test_coincidence_known_answers():
    m = _clock_model()
    # model spikes: 4 9 14 19 24 29 34 39 44
    c = _clock_case([6, 20, 21, 40])
    r = of.simulate(m, **c, delta=2, exclusive=True, record=True)
    assert r["rec"][0] == [4, 9, 14, 19, 24, 29, 34, 39, 44]
    # 4~6, 19~20 (21 left unmatched: 19 is spent), 39~40
    assert r["coinc"][0] == 3 and r["nspikes"][0] == 9
    r = of.simulate(m, **c, delta=2, exclusive=False)
    # inclusive: 4~6, 19~20/21, 39~40
    assert r["coinc"][0] == 3
    # two model spikes near one target: exclusive counts one, inclusive both
    c = _clock_case([7])
    assert of.simulate(m, **c, delta=3, exclusive=True)["coinc"][0] == 1
    assert of.simulate(m, **c, delta=3, exclusive=False)["coinc"][0] == 2
    # a spike delay of +2 moves every model spike to 6, 11, ...
    c = _clock_case([6, 11], delay=2)
    assert of.simulate(m, **c, delta=0, exclusive=True)["coinc"][0] == 2
    # refractory 3 steps: V held at 0 for 3 steps after each spike
    c = _clock_case([], refr=3)
    r = of.simulate(m, **c, delta=0, exclusive=True, record=True)
    assert r["rec"][0] == [4, 12, 20, 28, 36, 44]
    # onset: only spikes from step 10 on are counted
    c = _clock_case([])
    assert of.simulate(m, **c, delta=0, onset=10)["nspikes"][0] == 7


def test_online_exclusive_count_equals_offline_gamma_count():
    """With model and target spikes separated by more than 2 delta, the online
    exclusive count is the offline count of gamma_factor(normalize=False)
    (the comparison testinterface/test_monitor.py:272-419 sets up)."""
    rng = np.random.default_rng(11)
    eqs = Equations("dV/dt = I/tau : 1\nI : 1\ntau : 1", dummy=0.0)
    m = of.ModelOracle(eqs, "V > 1", "V = 0", 1.0, np.float64)
    delta = 5
    for trial in range(20):
        n = 4000
        # a model firing every `per` steps; targets jittered around a subset
        per = int(rng.integers(30, 60))
        model_spikes = np.arange(per - 1, n, per)
        keep = model_spikes[rng.random(len(model_spikes)) < 0.6]
        jit = rng.integers(-8, 9, len(keep))
        extra = rng.integers(0, n, 5)
        tgt = np.unique(np.clip(np.concatenate([keep + jit, extra]), 0, n - 1))
        tgt = tgt[np.concatenate([[True], np.diff(tgt) > 2 * delta])]
        S0 = np.array([[0.0], [float(per)]])
        spk = np.concatenate([[-10000], tgt, [n + 10000]])
        r = of.simulate(m, S0, np.ones(n), [0], [n], spk, [0], [len(spk)], delta=delta, exclusive=True, record=True)
        src = np.array(r["rec"][0])
        assert len(src) > 50 and np.all(np.diff(src) > 2 * delta)
        assert r["coinc"][0] == of.offline_coincidences(src, tgt, delta)


def test_gamma_matches_statistics():
    rng = np.random.default_rng(3)
    nc = rng.integers(0, 50, 100)
    nm = rng.integers(0, 80, 100)
    nt = rng.integers(2, 80, 100)
    r = rng.uniform(1, 40, 100)
    a = of.gamma(nc, nm, nt, r, 4e-3)
    b = get_gamma_factor(nc, nm, nt, r, 4e-3)
    assert np.array_equal(a, b)


def test_pso_reference_example_converges():
    """The reference's own example (particle_swarm.py:114-126): 5 groups of
    10 particles maximise exp(-0.7 |x|^2) in 5 dimensions."""
    rng = np.random.default_rng(0)
    X0 = 3 * rng.random((5, 50))
    Xg, fg, hist = of.pso_reference(X0, lambda x: np.exp(-.7 * np.sum(x ** 2, axis=0)), 150, [.8, 1.8, 1.8],
                                    -np.inf * np.ones(5), np.inf * np.ones(5), 10, seed=7)
    assert np.all(fg > 0.99)
    # group bests never decrease
    tr = np.array([h[3] for h in hist])
    assert np.all(np.diff(tr, axis=0) >= 0)


def test_philox_numpy_matches_c_oracle():
    lib = ct.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    f = lib.or_philox_uniform
    f.restype = ct.c_double
    f.argtypes = [ct.c_uint64, ct.c_int64, ct.c_int64]
    rng = np.random.default_rng(2)
    for seed in [0, 5, 2 ** 40 + 3]:
        st = rng.integers(0, 2 ** 40, 40)
        ix = rng.integers(0, 2 ** 40, 40)
        a = of.philox_uniform(seed, st, ix)
        b = np.array([f(seed, int(s), int(i)) for s, i in zip(st, ix)])
        assert np.array_equal(a, b)


def test_codegen_forms():
    eqs = Equations("dV/dt = (-V + a*V**2 + b*I**0.5 + c/I**-1)/tau : 1\nI : 1\ntau : 1",
                    a=0.1, b=2.0, c=3.0)
    code = generate_model_code(eqs, "V > 1", "V = 0", 1e-4, scalar="float")
    assert "(s_V * s_V)" in code.update
    assert "sqrtf(I_in)" in code.update
    assert "(0x1.99999a0000000p-4f)" in code.update   # 0.1 rounded to float, exact hex
    assert "((0x1.0000000000000p+0f) / I_in)" in code.update
    code = generate_model_code(eqs, "V > 1", "V = 0", 1e-4, scalar="double")
    assert "0x1.999999999999ap-4" in code.update
    with pytest.raises(CodegenError):
        generate_model_code(Equations("dV/dt = -V/unknown_name : 1", dummy=0.0), "V > 1", "V = 0", 1e-4)
    with pytest.raises(CodegenError):
        generate_model_code(eqs, "V > 1", "W = 0", 1e-4)


@pytest.mark.parametrize("scheme", ["Euler", "RK", "exponential_Euler"])
@pytest.mark.parametrize("precision", [32, 64])
def test_fit_kernel_compiles_for_sm100a(scheme, precision):
    from brian_b200._lib import fit_compile_check
    eqs = Equations(ADAPTIVE_LIF, dummy=0.0)
    code = generate_model_code(eqs, THRESHOLD, RESET, 1e-4, scalar="float" if precision == 32 else "double",
                               scheme=scheme)
    fit_compile_check(code, 1e-4, 40, True, precision)


def test_fit_kernel_compile_error_is_reported():
    from brian_b200._lib import fit_compile_check, EngineError

    class Bad(object):
        state = ["V"]
        update = "s_V = undefined_thing;"
        threshold = "s_V > 1.0"
        reset = ""
    with pytest.raises(EngineError, match="compilation failed"):
        fit_compile_check(Bad(), 1e-4, 40)
