"""Model fitting on the GPU: the reference's modelfitting API over the
batched fitting kernel.

* ``GPUModelFitting`` (library/modelfitting/gpu_modelfitting.py:202-401):
  one kernel over all candidates; ``reinit_vars``, ``launch``,
  ``coincidence_count``, ``spike_count``.
* ``modelfitting`` (library/modelfitting/modelfitting.py:232-518) with the
  data preparation of ``ModelFitting.prepare_data`` (modelfitting.py:117-173)
  and the fitness of ``ModelFitting.evaluate`` (modelfitting.py:175-227);
  the optimiser is the grouped particle swarm of tools/particle_swarm.py:
  6-111, run on the device (move, simulate, gamma, best updates per
  iteration, no host round trip).
* ``get_spikes`` and ``predict`` (modelfitting.py:523-608).

Extensions over the reference, for many targets of uneven length: ``input``
may be a list of arrays, one per target, each with its own duration.

Differences kept on purpose:

* the optimisers of the reference come from the external playdoh package,
  which is not in the reference tree: CMA-ES (the default, as in the
  reference) is restated from Hansen's tutorial (``cmaes.py``), the GA is a
  real-coded GA of published operators (``ga.py``), and PSO follows the
  reference's own ``particle_swarm``;
* a fixed ``refractory`` period is applied on the GPU (the reference's GPU
  path passes zeros unless the period is a fitted parameter,
  modelfitting.py:182-184);
* parameters named both in ``params`` and ``initial_values`` are rejected
  (the reference silently lets initial_values win).
"""
import numpy as np

from . import _lib
from .codegen import generate_model_code, SCHEMES
from .equations import Equations
from .statistics import firing_rate, gamma_factor

__all__ = ["GPUModelFitting", "modelfitting", "distributed_modelfitting", "get_spikes", "predict", "print_table",
           "PSO", "GA", "CMAES",
           "OptimizationResult", "euler_scheme", "rk2_scheme", "exp_euler_scheme", "MAXCPU", "MAXGPU"]

# integration scheme names (experimental/codegen/integration_schemes.py)
euler_scheme = "Euler"
rk2_scheme = "RK"
exp_euler_scheme = "exponential_Euler"
MAXCPU = -1
MAXGPU = -1


class PSO(object):
    """Particle swarm optimiser; optparams ``omega``, ``cl`` (cognitive) and
    ``cg`` (social) weights."""
    defaults = {"omega": 0.7298, "cl": 1.49618, "cg": 1.49618}


class GA(object):
    """Real-coded genetic algorithm (brian_b200/ga.py): binary tournament,
    BLX-alpha crossover, Gaussian mutation, elitism; optparams ``elite``,
    ``tournament``, ``crossover``, ``alpha``, ``mutation``, ``sigma`` (in the
    [-1, 1]-scaled space)."""
    defaults = {"elite": None, "tournament": 2, "crossover": 0.8, "alpha": 0.5, "mutation": None, "sigma": 0.1}


class CMAES(object):
    """Covariance matrix adaptation evolution strategy (brian_b200/cmaes.py);
    optparams ``sigma0`` (initial step in the [-1, 1]-scaled space)."""
    defaults = {"sigma0": 0.5}


_PRECISION = {"double": 64, "float": 32, 64: 64, 32: 32}


def _threshold_reset_of(G):
    th = getattr(G, "_threshold", None)
    rs = getattr(G, "_reset", None)
    if rs is None:
        rs = getattr(G, "_resetfun", None)
    return th, rs


class GPUModelFitting(object):
    """All candidates of a fit in one kernel (gpu_modelfitting.py:202-401).

    ``G`` gives the model, threshold, reset, clock and initial state (a
    NeuronGroup; it never runs on a network).  ``I``/``I_offset`` give each
    neuron's input trace, ``spiketimes``/``spiketimes_offset`` its target
    train (seconds, framed by a spike before 0 and one after the end).
    ``duration`` (here, optional) sets each neuron's own length; by default
    every neuron runs for the length passed to ``launch``."""

    def __init__(self, G, eqs, I, I_offset, spiketimes, spiketimes_offset, spikedelays, refractory, delta,
                 onset=0.0, coincidence_count_algorithm="exclusive", precision="double", scheme=euler_scheme,
                 device=0):
        if isinstance(eqs, str):
            eqs = Equations(eqs, level=1)
        self.G = G
        self.eqs = eqs
        self.N = N = len(G)
        self.dt = dt = float(G.clock.dt)
        self.delta = float(delta)
        self.onset = float(onset)
        self.precision = _PRECISION[precision]
        self.coincidence_count_algorithm = coincidence_count_algorithm
        if coincidence_count_algorithm not in ("exclusive", "inclusive"):
            raise ValueError("coincidence_count_algorithm must be 'exclusive' or 'inclusive'")
        th, rs = _threshold_reset_of(G)
        self.code = generate_model_code(eqs, th, rs, dt, scalar="float" if self.precision == 32 else "double",
                                        scheme=scheme)
        self.fit = _lib.FitHandle(self.code, dt, int(np.rint(self.delta / dt)),
                                  exclusive=coincidence_count_algorithm == "exclusive", precision=self.precision,
                                  device=device)
        self._launched_to = 0
        self.reinit_vars(I, I_offset, spiketimes, spiketimes_offset, spikedelays, refractory)

    def _state0(self):
        S = np.asarray(self.G._S_host if hasattr(self.G, "_S_host") else self.G._S, dtype=np.float64)
        names = list(getattr(self.G, "_names", self.eqs._diffeq_names))
        return np.array([S[names.index(v)] for v in self.code.state])

    def reinit_vars(self, I, I_offset, spiketimes, spiketimes_offset, spikedelays, refractory, nsteps=None):
        """Copies of the inputs, trains, delays and refractory periods; state
        from G (gpu_modelfitting.py:333-379)."""
        dt = self.dt
        I = np.asarray(I, dtype=np.float64)
        I_offset = np.asarray(I_offset, dtype=np.int64).reshape(-1)
        if len(I_offset) == 1 and self.N > 1:
            I_offset = np.repeat(I_offset, self.N)
        spk = np.asarray(np.rint(np.asarray(spiketimes, dtype=np.float64) / dt), dtype=np.int32)
        off = np.asarray(spiketimes_offset, dtype=np.int64).reshape(-1)
        # each train runs up to its trailing sentinel (the first entry after
        # the offset that lies past every input step)
        end = np.empty(self.N, dtype=np.int64)
        starts = np.unique(off)
        nxt = {}
        for s in starts:
            k = s + 1
            while k < len(spk) - 1 and spk[k] <= spk[k + 1]:
                k += 1
            nxt[s] = k + 1
        for i in range(self.N):
            end[i] = nxt[off[i]]
        if nsteps is None:
            nsteps = np.full(self.N, min(len(I) - int(I_offset.max()), 2 ** 31 - 1), dtype=np.int32)
        delays = np.asarray(np.rint(np.asarray(spikedelays, dtype=np.float64) * np.ones(self.N) / dt), dtype=np.int32)
        refr = np.asarray(np.rint(np.asarray(refractory, dtype=np.float64) * np.ones(self.N) / dt), dtype=np.int32)
        self.fit.set_input(I)
        self.fit.set_targets(spk)
        self.fit.set_sims(self._state0(), I_offset, nsteps, off, end, delays, refr,
                          int(np.rint(self.onset / dt)))
        self._launched_to = 0

    def launch(self, duration, stepsize=1.0):
        """Advance every neuron by `duration` (gpu_modelfitting.py:381-393);
        the stepsize only splits the launch."""
        total = int(duration / self.dt)
        if stepsize is None:
            chunks = [(0, total)]
        else:
            step = max(1, int(stepsize / self.dt))
            chunks = [(a, min(a + step, total)) for a in range(0, total, step)]
        for a, b in chunks:
            self.fit.run(self._launched_to + a, self._launched_to + b)
        self._launched_to += total

    def get_coincidence_count(self):
        return self.fit.read()[0]

    def get_spike_count(self):
        return self.fit.read()[1]

    coincidence_count = property(get_coincidence_count)
    spike_count = property(get_spike_count)


class OptimizationResult(object):
    """best_pos / best_fit / info per target group; ``r[key]`` gives the best
    value of parameter `key` (one value, or a list over groups), ``r[i]`` the
    result of group i."""

    def __init__(self, best_pos, best_fit, info):
        self.best_pos = best_pos
        self.best_fit = best_fit
        self.info = info

    def __getitem__(self, key):
        if isinstance(key, (int, np.integer)):
            if isinstance(self.best_pos, list):
                return OptimizationResult(self.best_pos[key], self.best_fit[key], self.info)
            if key == 0:
                return self
            raise IndexError(key)
        if isinstance(self.best_pos, list):
            return [p[key] for p in self.best_pos]
        return self.best_pos[key]

    def __repr__(self):
        return "OptimizationResult(best_fit=%r, best_pos=%r)" % (self.best_fit, self.best_pos)


def print_table(results, precision=4, colwidth=16):
    groups = results.best_pos if isinstance(results.best_pos, list) else [results.best_pos]
    fits = results.best_fit if isinstance(results.best_fit, (list, np.ndarray)) else [results.best_fit]
    keys = sorted(groups[0].keys())
    print("".join(("%s" % k).ljust(colwidth) for k in ["group"] + keys + ["best fit"]))
    for i, (g, f) in enumerate(zip(groups, fits)):
        row = [str(i)] + ["%.*g" % (precision, g[k]) for k in keys] + ["%.*g" % (precision, f)]
        print("".join(c.ljust(colwidth) for c in row))


class FittingProblem(object):
    """Device state of one fit: every candidate of every target group, with
    its input row, target train and gamma normalisation
    (ModelFitting.initialize/prepare_data, modelfitting.py:27-173).

    Time slicing (modelfitting.py:49-58, 126-163, 221-223): each input is cut
    to a multiple of `slices` steps; slice k of a candidate simulates its
    k-th piece preceded by `overlap` of the previous piece (zeros before the
    first), against the target spikes of that piece shifted into the
    slice's clock, and coincidences and spike counts are summed over the
    slices before gamma.  Simulations are slice-major (i = k * N + n, the
    reference's I_offset layout), every simulation runs the slice plus the
    overlap, and each gets its own candidate's parameters."""

    def __init__(self, model, threshold, reset, data, inputs, dt, popsize, delta=4e-3, refractory=0.0,
                 initial_values=None, precision="double", method="Euler", param_names=(), onset=0.0,
                 coincidence_count_algorithm="exclusive", input_var="I", device=0, record=0, slices=1,
                 overlap=0.0):
        if isinstance(model, str):
            model = Equations(model, level=2)
        self.eqs = model
        self.dt = dt = float(dt)
        if method not in SCHEMES:
            raise ValueError("The method can only be 'Euler', 'RK', or 'exponential_Euler'")
        self.precision = _PRECISION[precision]
        self.code = generate_model_code(model, threshold, reset, dt, input_var=input_var,
                                        scalar="float" if self.precision == 32 else "double", scheme=method)
        self.delta = float(delta)
        groups = len(inputs)
        self.groups = groups
        self.popsize = popsize = int(popsize)
        self.N = N = groups * popsize
        # inputs: one row per target group; each group's duration is its
        # input's (modelfitting.py:398, 44-49)
        self.slices = slices = int(slices)
        if slices < 1:
            raise ValueError("slices must be at least 1")
        if slices == 1:
            overlap = 0.0                        # no overlap without slicing (modelfitting.py:427-429)
        ov = int(float(overlap) / dt)
        self.overlap_steps = ov
        # per group: input cut to a multiple of `slices`, zeros of the overlap
        # in front, steps per slice (modelfitting.py:50-58)
        pieces, sliced, lens = [], [], []
        for x in inputs:
            x = np.asarray(x, dtype=np.float64)
            L = slices * (len(x) // slices)
            pieces.append(np.hstack((np.zeros(ov), x[:L])))
            sliced.append(L // slices)
            lens.append(L)
        # steps simulated: int(duration / dt) without slicing (the float round
        # trip of GPUModelFitting.launch, gpu_modelfitting.py:388), else the
        # slice plus the overlap (total_steps, modelfitting.py:54)
        self.nsteps_group = np.array([int((L * dt) / dt) if slices == 1 else s + ov for L, s in zip(lens, sliced)],
                                     dtype=np.int32)
        I = np.concatenate(pieces)
        ioff = np.concatenate([[0], np.cumsum([len(p) for p in pieces])[:-1]]).astype(np.int64)
        self.input_offsets = ioff
        # target trains with sentinels at -1 s and the slice's duration + 1 s
        # (modelfitting.py:139-163), lengths and rates of the whole train
        # (modelfitting.py:144-145); trains[k][j] is slice k of target j
        trains = [[None] * groups for _ in range(slices)]
        tlen, trate = [], []
        for j in range(groups):
            s = np.sort(np.asarray(data[j], dtype=np.float64))
            tlen.append(len(s))
            trate.append(firing_rate(s))
            duration = lens[j] * dt
            sliced_duration = float(overlap) + duration / slices
            for k in range(slices):
                inside = (s >= k * sliced[j] * dt) & (s < (k + 1) * sliced[j] * dt)
                local = s[inside] - k * sliced[j] * dt + ov * dt
                trains[k][j] = np.hstack(([-1.0], local, [sliced_duration + 1.0]))
        self.target_length = np.repeat(np.array(tlen, dtype=np.int32), popsize)
        self.target_rate = np.repeat(np.array(trate, dtype=np.float64), popsize)
        flat = [trains[k][j] for k in range(slices) for j in range(groups)]
        toff_kj = np.concatenate([[0], np.cumsum([len(t) for t in flat])[:-1]]).astype(np.int64).reshape(slices, groups)
        tend_kj = toff_kj + np.array([len(t) for t in flat], dtype=np.int64).reshape(slices, groups)
        spk = np.asarray(np.rint(np.concatenate(flat) / dt), dtype=np.int32)
        gidx = np.repeat(np.arange(groups), popsize)
        kidx = np.repeat(np.arange(slices), N)
        gall = np.tile(gidx, slices)
        sim_ioff = ioff[gall] + kidx * np.array(sliced, dtype=np.int64)[gall]
        sim_toff, sim_tend = toff_kj[kidx, gall], tend_kj[kidx, gall]
        NS = N * slices
        # the simulations as the device holds them (input offsets and steps,
        # target trains in steps and their [offset, end) per simulation)
        self.sim_input = I
        self.sim_input_offsets, self.sim_nsteps = sim_ioff, self.nsteps_group[gall]
        self.sim_trains, self.sim_train_offsets, self.sim_train_ends = spk, sim_toff, sim_tend
        # initial state: zeros (NeuronGroup.reinit), then initial_values
        S0 = np.zeros((len(self.code.state), NS))
        initial_values = initial_values or {}
        for k, v in initial_values.items():
            if k in param_names:
                raise ValueError("parameter %r is both fitted and given an initial value" % k)
            if k not in self.code.state:
                raise ValueError("initial value for unknown variable %r" % k)
            S0[self.code.index(k)] = v
        refr = np.full(NS, int(np.rint(float(refractory) / dt)), dtype=np.int32)
        self.handle = h = _lib.FitHandle(self.code, dt, int(np.rint(self.delta / dt)),
                                         exclusive=coincidence_count_algorithm == "exclusive",
                                         precision=self.precision, device=device)
        h.set_input(I)
        h.set_targets(spk)
        if record:
            h.set_record(record)
        h.set_sims(S0, sim_ioff, self.nsteps_group[gall], sim_toff, sim_tend, None, refr,
                   int(np.rint(float(onset) / dt)))
        h.set_gamma(N, slices, self.target_length, self.target_rate, self.delta)
        dim_var = []
        for p in param_names:
            if p == "delays":
                dim_var.append(-1)
            elif p == "refractory":
                dim_var.append(-2)
            elif p in self.code.state:
                dim_var.append(self.code.index(p))
            else:
                raise ValueError("Parameter %s must be defined as a parameter in the model" % p)
        self.param_names = list(param_names)
        h.set_params(dim_var)

    def evaluate(self, X):
        """Gamma factor of every candidate; X is [ndim][N]."""
        return self.handle.evaluate(X)

    def neuron_steps(self):
        return int(np.sum(self.nsteps_group.astype(np.int64)) * self.popsize * self.slices)


def _split_data(data):
    data = np.asarray(data, dtype=np.float64)
    if data.ndim == 1:
        data = np.column_stack((np.zeros(len(data)), data))
    groups = int(data[:, 0].max() + 1) if len(data) else 1
    return [data[data[:, 0] == j, 1] for j in range(groups)]


def _bounds(params):
    names, lo, hi, imin, imax = [], [], [], [], []
    for k, v in params.items():
        v = list(v)
        if len(v) == 2:
            lo_, a, b, hi_ = -np.inf, v[0], v[1], np.inf
        elif len(v) == 4:
            lo_, a, b, hi_ = v
        else:
            raise ValueError("parameter %s: give [min, max] or [bound_min, min, max, bound_max]" % k)
        names.append(k)
        lo.append(float(lo_))
        hi.append(float(hi_))
        imin.append(float(a))
        imax.append(float(b))
    return names, np.array(lo), np.array(hi), np.array(imin), np.array(imax)


def modelfitting(model=None, reset=None, threshold=None, refractory=0.0, data=None, input_var="I", input=None,
                 dt=None, popsize=1000, maxiter=10, delta=4e-3, slices=1, overlap=0.0, initial_values=None,
                 stepsize=0.1, unit_type=None, total_units=None, cpu=None, gpu=None, precision="double",
                 machines=(), allocation=None, returninfo=False, scaling=None, algorithm=CMAES, optparams=None,
                 method="Euler", seed=None, evaluate_initial=True, initial_positions=None, device=0, **params):
    """Fit a spiking neuron model to target spike trains (modelfitting.py:232-518).

    ``data``: spike times, or (target index, spike time) pairs; ``input``: one
    input trace shared by all targets, or a list with one trace per target
    (own durations).  ``params``: ``name=[min, max]`` or ``name=[bound_min,
    min, max, bound_max]``; ``delays`` and a list-valued ``refractory`` fit
    the spike delay and refractory period.  ``popsize`` candidates per target
    and ``maxiter`` iterations of ``algorithm``: CMAES (the default, as in the
    reference; one search per target, generations evaluated on the GPU), GA
    (one population per target, likewise) or PSO (the whole swarm on the
    GPU).

    ``initial_positions`` ([ndim][groups*popsize], optional) replaces the
    uniform initial draw, e.g. with proposals of a learned model;
    ``evaluate_initial`` scores the initial swarm before the first move.
    Returns an OptimizationResult; ``info`` holds the per-iteration group
    best fitness (``trace``) and GPU time (``iteration_ms``)."""
    if model is None or data is None or input is None:
        raise ValueError("model, data and input are required")
    if dt is None:
        raise Exception("dt (sampling frequency of the input) must be set")
    if algorithm not in (PSO, CMAES, GA):
        raise NotImplementedError("algorithm must be CMAES (the default), GA or PSO")
    if isinstance(model, str):
        model = Equations(model, level=1)
    trains = _split_data(data)
    groups = len(trains)
    if isinstance(input, (list, tuple)) and len(input) and np.ndim(input[0]) == 1:
        inputs = [np.asarray(x, dtype=np.float64) for x in input]
        if len(inputs) != groups:
            raise ValueError("one input per target train is needed (%d inputs, %d trains)" % (len(inputs), groups))
    else:
        inputs = [np.asarray(input, dtype=np.float64)] * groups
    params = dict(params)
    if isinstance(refractory, (list, tuple)):
        params["refractory"] = refractory
        refractory = 0.0
    for p in params:
        if p not in model._diffeq_names and p not in ("delays", "refractory"):
            raise Exception("Parameter %s must be defined as a parameter in the model" % p)
    names, lo, hi, imin, imax = _bounds(params)
    prob = FittingProblem(model, threshold, reset, trains, inputs, dt, popsize, delta=delta, refractory=refractory,
                          initial_values=initial_values, precision=precision, method=method, param_names=names,
                          input_var=input_var, device=device, slices=slices, overlap=overlap)
    M = prob.N
    rng = np.random.default_rng(seed)
    if algorithm is CMAES:
        return _fit_cmaes(prob, names, lo, hi, imin, imax, groups, popsize, maxiter, rng, optparams,
                          initial_positions)
    if algorithm is GA:
        return _fit_ga(prob, names, lo, hi, imin, imax, groups, popsize, maxiter, rng, optparams,
                       initial_positions)
    if initial_positions is None:
        X0 = imin.reshape(-1, 1) + (imax - imin).reshape(-1, 1) * rng.random((len(names), M))
    else:
        X0 = np.asarray(initial_positions, dtype=np.float64).reshape(len(names), M)
    opt = dict(PSO.defaults)
    opt.update(optparams or {})
    h = prob.handle
    h.pso_init(popsize, X0, lo, hi, opt["omega"], opt["cl"], opt["cg"],
               int(rng.integers(0, 2 ** 63 - 1)) if seed is None else int(seed))
    if evaluate_initial:
        h.pso_evaluate_initial()
    trace, ms = h.pso_run(int(maxiter))
    Xg, fg = h.pso_best()
    best_pos = [{k: float(Xg[d, j]) for d, k in enumerate(names)} for j in range(groups)]
    info = {"trace": trace, "iteration_ms": ms, "neuron_steps_per_iteration": prob.neuron_steps(),
            "groups": groups, "popsize": popsize}
    if groups == 1:
        return OptimizationResult(best_pos[0], float(fg[0]), info)
    return OptimizationResult(best_pos, list(map(float, fg)), info)


def _fit_cmaes(prob, names, lo, hi, imin, imax, groups, popsize, maxiter, rng, optparams, initial_positions):
    """CMA-ES per target group with mapminmax scaling (modelfitting.py:442-443):
    every generation's candidates of all groups in one device evaluation."""
    from .cmaes import CMAState
    opt = dict(CMAES.defaults)
    opt.update(optparams or {})
    n = len(names)
    span = (imax - imin)
    span = np.where(span > 0, span, 1.0)

    def to_params(xs):                       # scaled [-1, 1] -> parameter space
        return imin + (xs + 1.0) * 0.5 * span

    if initial_positions is None:
        mean = np.zeros((groups, n))
    else:
        X0 = np.asarray(initial_positions, dtype=np.float64).reshape(n, groups, popsize)
        mean = ((X0.mean(axis=2).T - imin) / (0.5 * span)) - 1.0
    st = CMAState(groups, n, popsize, mean, opt["sigma0"], rng)
    best_x = np.zeros((groups, n))
    best_f = np.full(groups, -np.inf)
    trace = np.zeros((int(maxiter), groups))
    ms = np.zeros(int(maxiter))
    for it in range(int(maxiter)):
        xs, y = st.ask()
        P = np.clip(to_params(xs), lo, hi)                  # [G][lam][n]
        X = np.ascontiguousarray(P.transpose(2, 0, 1).reshape(n, groups * popsize))
        f = prob.evaluate(X).reshape(groups, popsize)
        ms[it] = prob.handle.stats()["last_eval_ms"]
        fv = np.where(np.isnan(f), -np.inf, f)
        k = np.argmax(fv, axis=1)
        better = fv[np.arange(groups), k] > best_f
        best_f = np.where(better, fv[np.arange(groups), k], best_f)
        best_x[better] = P[np.arange(groups), k][better]
        trace[it] = best_f
        st.tell(y, f)
    best_pos = [{k_: float(best_x[j, d]) for d, k_ in enumerate(names)} for j in range(groups)]
    info = {"trace": trace, "iteration_ms": ms, "neuron_steps_per_iteration": prob.neuron_steps(),
            "groups": groups, "popsize": popsize, "algorithm": "CMAES"}
    if groups == 1:
        return OptimizationResult(best_pos[0], float(best_f[0]), info)
    return OptimizationResult(best_pos, list(map(float, best_f)), info)


def _fit_ga(prob, names, lo, hi, imin, imax, groups, popsize, maxiter, rng, optparams, initial_positions):
    """GA per target group in the mapminmax-scaled space: every generation's
    candidates of all groups in one device evaluation."""
    from .ga import GAState
    opt = dict(GA.defaults)
    opt.update(optparams or {})
    n = len(names)
    span = (imax - imin)
    span = np.where(span > 0, span, 1.0)
    slo = (np.asarray(lo) - imin) / (0.5 * span) - 1.0
    shi = (np.asarray(hi) - imin) / (0.5 * span) - 1.0
    if initial_positions is None:
        X0 = rng.uniform(-1.0, 1.0, (groups, popsize, n))
    else:
        P0 = np.asarray(initial_positions, dtype=np.float64).reshape(n, groups, popsize).transpose(1, 2, 0)
        X0 = (P0 - imin) / (0.5 * span) - 1.0
    st = GAState(groups, n, popsize, X0, rng, lo=slo, hi=shi, **opt)
    best_x = np.zeros((groups, n))
    best_f = np.full(groups, -np.inf)
    trace = np.zeros((int(maxiter), groups))
    ms = np.zeros(int(maxiter))
    for it in range(int(maxiter)):
        P = np.clip(imin + (st.ask() + 1.0) * 0.5 * span, lo, hi)     # [G][pop][n]
        X = np.ascontiguousarray(P.transpose(2, 0, 1).reshape(n, groups * popsize))
        f = prob.evaluate(X).reshape(groups, popsize)
        ms[it] = prob.handle.stats()["last_eval_ms"]
        fv = np.where(np.isnan(f), -np.inf, f)
        k = np.argmax(fv, axis=1)
        better = fv[np.arange(groups), k] > best_f
        best_f = np.where(better, fv[np.arange(groups), k], best_f)
        best_x[better] = P[np.arange(groups), k][better]
        trace[it] = best_f
        st.tell(f)
    best_pos = [{k_: float(best_x[j, d]) for d, k_ in enumerate(names)} for j in range(groups)]
    info = {"trace": trace, "iteration_ms": ms, "neuron_steps_per_iteration": prob.neuron_steps(),
            "groups": groups, "popsize": popsize, "algorithm": "GA"}
    if groups == 1:
        return OptimizationResult(best_pos[0], float(best_f[0]), info)
    return OptimizationResult(best_pos, list(map(float, best_f)), info)


def distributed_modelfitting(data=None, input=None, process_group=None, **kwargs):
    """modelfitting with the targets split over the ranks of a
    torch.distributed job, one GPU per rank (the reference spreads a fit
    over GPUs and machines through playdoh, modelfitting.py:446-518).

    Targets are independent groups of the search, so nothing is exchanged
    during the fit: rank r fits targets [r*G/W, (r+1)*G/W) on device
    LOCAL_RANK (unless ``device`` is given) with the same arguments, and
    the results are gathered (``all_gather_object``) into one
    OptimizationResult in target order on every rank; ``info["ranks"]``
    holds each rank's own info.  ``data`` is (target index, spike time)
    pairs; ``input`` one shared trace or one trace per target."""
    import os
    import torch.distributed as dist
    world = dist.get_world_size(process_group)
    rank = dist.get_rank(process_group)
    trains = _split_data(data)
    G = len(trains)
    lo, hi = rank * G // world, (rank + 1) * G // world
    per_target = isinstance(input, (list, tuple)) and len(input) and np.ndim(input[0]) == 1
    pos, fit, info = [], [], None
    if hi > lo:
        pairs = np.array([(k, t) for k, j in enumerate(range(lo, hi)) for t in trains[j]], dtype=np.float64)
        inp = list(input[lo:hi]) if per_target else input
        kw = dict(kwargs)
        kw.setdefault("device", int(os.environ.get("LOCAL_RANK", "0")))
        res = modelfitting(data=pairs, input=inp, **kw)
        pos = res.best_pos if isinstance(res.best_pos, list) else [res.best_pos]
        fit = res.best_fit if isinstance(res.best_fit, list) else [res.best_fit]
        info = res.info
    parts = [None] * world
    dist.all_gather_object(parts, (lo, pos, fit, info), group=process_group)
    parts.sort(key=lambda x: x[0])
    all_pos = [p for part in parts for p in part[1]]
    all_fit = [f for part in parts for f in part[2]]
    ginfo = {"ranks": [part[3] for part in parts], "world_size": world, "groups": G}
    if G == 1:
        return OptimizationResult(all_pos[0], all_fit[0], ginfo)
    return OptimizationResult(all_pos, all_fit, ginfo)


def get_spikes(model=None, reset=None, threshold=None, input=None, input_var="I", dt=None, initial_values=None,
               method="Euler", precision="double", max_spikes=None, **params):
    """Spikes (index, time) of the model with the given parameters, one
    neuron per parameter set (modelfitting.py:523-563), simulated by the
    fitting kernel."""
    if isinstance(model, str):
        model = Equations(model, level=1)
    vals = {k: np.atleast_1d(np.asarray(v, dtype=np.float64)) for k, v in params.items()
            if k not in ("delays", "fitness")}
    n = max([len(v) for v in vals.values()] + [1])
    if isinstance(input, (list, tuple)) and len(input) and np.ndim(input[0]) == 1:
        inputs = [np.asarray(x, dtype=np.float64) for x in input]
    else:
        inputs = [np.asarray(input, dtype=np.float64)] * n
    if max_spikes is None:
        max_spikes = max(len(x) for x in inputs) // 2 + 1
    dummy = [np.zeros(0)] * n
    prob = FittingProblem(model, threshold, reset, dummy, inputs, dt, 1, initial_values=initial_values,
                          precision=precision, method=method, param_names=list(vals), input_var=input_var,
                          record=int(max_spikes))
    X = np.array([np.broadcast_to(vals[k], (n,)) for k in vals]) if vals else np.zeros((0, n))
    prob.evaluate(X)
    counts, steps = prob.handle.read_spikes()
    out = []
    for i in range(n):
        c = min(int(counts[i]), prob.handle.rec_cap)
        out.extend((i, float(s) * float(dt)) for s in steps[i, :c])
    out.sort(key=lambda x: (x[1], x[0]))
    return out


def predict(model=None, reset=None, threshold=None, data=None, delta=4e-3, input=None, input_var="I", dt=None,
            **params):
    """Gamma factor of the fitted model against `data` for a new input
    (modelfitting.py:565-608)."""
    spikes = get_spikes(model=model, reset=reset, threshold=threshold, input=input, input_var=input_var, dt=dt,
                        **params)
    keys = [k for k in params if k not in ("delays", "fitness")]
    ngroups = len(np.atleast_1d(params[keys[0]])) if keys else 1
    gamma = np.zeros(ngroups)
    for i in range(ngroups):
        spk = [t for j, t in spikes if j == i]
        gamma[i] = gamma_factor(spk, data, delta, normalize=True, dt=dt)
    return gamma[0] if len(gamma) == 1 else gamma
