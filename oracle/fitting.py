"""CPU oracle for batched model fitting -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg
as the checker; nothing in the product path calls it.

A numpy restatement, vectorised over simulations, of:

* the reference GPU fitting kernel ``runsim`` and its coincidence algorithms
  (library/modelfitting/gpu_modelfitting.py:39-156): per step input read,
  state update, ``is_refractory = T <= next_allowed``, threshold, spike count
  from ``onset``, reset while spiking or refractory, ``next_allowed = T +
  refractory``, the exclusive / inclusive coincidence test on ``Tspike = T +
  delay`` and the target pointer move;
* the integration schemes euler / rk2 / exp_euler
  (experimental/codegen/integration_schemes.py:3-43), evaluating the model's
  equation strings with numpy in the scalar type (every constant rounded to
  that type, arithmetic in it);
* get_gamma_factor and firing_rate (tools/statistics.py:15-21, 236-240);
* the grouped particle swarm (tools/particle_swarm.py:6-111), with its
  uniform draws taken from Philox4x32-10 keyed (seed, 2*it [+1], d*M + p)
  instead of numpy's global generator;
* Philox4x32-10 (Random123) and the 53-bit uniform built from it.

Two deliberate differences from the reference kernel are restated too: each
simulation runs for its own number of steps, and the target pointer stops at
the train's final sentinel.
"""
import ast

import numpy as np

__all__ = ["philox_uniform", "ModelOracle", "simulate", "gamma", "firing_rate", "pso_reference",
           "offline_coincidences", "pso_move", "pso_best"]

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox_uniform(seed, step, idx):
    """53-bit uniform in [0, 1) from Philox4x32-10, counter (step lo, step hi,
    idx lo, idx hi), key (seed lo, seed hi); vectorised over step/idx."""
    step = np.asarray(step, dtype=np.int64).astype(np.uint64)
    idx = np.asarray(idx, dtype=np.int64).astype(np.uint64)
    step, idx = np.broadcast_arrays(step, idx)
    c0 = step & _MASK
    c1 = step >> np.uint64(32)
    c2 = idx & _MASK
    c3 = idx >> np.uint64(32)
    seed = int(seed) & ((1 << 64) - 1)
    k0 = np.uint64(seed & 0xFFFFFFFF)
    k1 = np.uint64(seed >> 32)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = _M0 * c0
            p1 = _M1 * c2
            hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
            hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
            n0 = hi1 ^ c1 ^ k0
            n2 = hi0 ^ c3 ^ k1
            c0, c1, c2, c3 = n0, lo1, n2, lo0
            k0 = (k0 + _W0) & _MASK
            k1 = (k1 + _W1) & _MASK
    a = c0 >> np.uint64(5)
    b = c1 >> np.uint64(6)
    return (a.astype(np.float64) * 67108864.0 + b.astype(np.float64)) * (1.0 / 9007199254740992.0)


class _Consts(ast.NodeTransformer):
    """Every numeric literal becomes a typed constant of the scalar type."""

    def __init__(self, table, base):
        self.table = table
        self.base = base

    def visit_Constant(self, node):
        if isinstance(node.value, (int, float)) and not isinstance(node.value, bool):
            name = "__c%d" % (self.base + len(self.table))
            self.table[name] = node.value
            return ast.copy_location(ast.Name(id=name, ctx=ast.Load()), node)
        return node


class ModelOracle(object):
    """A model (Equations, threshold, reset) evaluated with numpy in one
    scalar type (np.float32 or np.float64)."""

    _funcs = {"exp": np.exp, "log": np.log, "sqrt": np.sqrt, "sin": np.sin, "cos": np.cos, "tan": np.tan,
              "tanh": np.tanh, "sinh": np.sinh, "cosh": np.cosh, "arctan": np.arctan, "abs": np.abs,
              "log10": np.log10, "floor": np.floor, "ceil": np.ceil}

    def __init__(self, eqs, threshold, reset, dt, dtype, input_var="I", scheme="Euler", namespace=None):
        eqs.prepare()
        self.dtype = np.dtype(dtype).type
        self.dt = float(dt)
        self.input_var = input_var
        self.scheme = scheme
        self.state = [v for v in eqs._diffeq_names if v != input_var]
        self.dynamic = [v for v in eqs._diffeq_names_nonzero if v != input_var]
        ns = dict(eqs.namespace)
        if namespace:
            ns.update(namespace)
        self.consts = {}
        for k, v in ns.items():
            if isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, bool):
                self.consts[k] = self.dtype(v)
        self.consts.update(self._funcs)
        self.consts["dt"] = self.dtype(dt)
        self.rhs = {v: self._compile(eqs._string[v]) for v in self.state}
        self.threshold = self._compile(threshold, "eval")
        self.reset = []
        for raw in reset.replace(";", "\n").split("\n"):
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            st = ast.parse(line, mode="exec").body[0]
            if isinstance(st, ast.Assign):
                self.reset.append((st.targets[0].id, None, self._compile(ast.unparse(st.value))))
            else:
                op = {ast.Add: np.add, ast.Sub: np.subtract, ast.Mult: np.multiply, ast.Div: np.divide}[type(st.op)]
                self.reset.append((st.target.id, op, self._compile(ast.unparse(st.value))))

    def _compile(self, expr, mode="eval"):
        tree = ast.parse(expr.strip(), mode="eval")
        table = {}
        tree = ast.fix_missing_locations(_Consts(table, len(self.consts)).visit(tree))
        for k, v in table.items():
            self.consts[k] = self.dtype(v)
        return compile(tree, "<model>", "eval")

    def _env(self, S, I_in, t, override=None):
        env = dict(self.consts)
        env.update(S)
        env[self.input_var] = I_in
        env["t"] = t
        if override:
            env.update(override)
        return env

    def update(self, S, I_in, t):
        """One step of the scheme (integration_schemes.py:3-43); S maps
        names to arrays and is updated in place."""
        dt = self.consts["dt"]
        if self.scheme == "Euler":
            env = self._env(S, I_in, t)
            tmp = {v: eval(self.rhs[v], env) for v in self.dynamic}
            for v in self.dynamic:
                S[v] = S[v] + tmp[v] * dt
        elif self.scheme == "RK":
            env = self._env(S, I_in, t)
            half = {}
            buf = {}
            h = self.dtype(0.5) * dt
            for v in self.state:
                buf[v] = eval(self.rhs[v], env)
                half[v] = h * buf[v]
                half[v] = half[v] + S[v]
            env2 = self._env(S, I_in, t, half)
            for v in self.dynamic:
                buf[v] = eval(self.rhs[v], env2)
                S[v] = S[v] + dt * buf[v]
        elif self.scheme == "exponential_Euler":
            AB = {}
            for v in self.dynamic:
                B = eval(self.rhs[v], self._env(S, I_in, t, {v: self.dtype(0)}))
                A = eval(self.rhs[v], self._env(S, I_in, t, {v: self.dtype(1)}))
                A = A - B
                B = B / A
                A = A * dt
                AB[v] = (A, B)
            for v in self.dynamic:
                A, B = AB[v]
                S[v] = S[v] + B
                S[v] = S[v] * np.exp(A)
                S[v] = S[v] - B
        else:
            raise ValueError(self.scheme)
        for v in self.state:
            S[v] = np.asarray(S[v], dtype=self.dtype)

    def spiking(self, S, I_in, t):
        return np.asarray(eval(self.threshold, self._env(S, I_in, t)), dtype=bool)

    def apply_reset(self, S, I_in, t, mask):
        for tgt, op, code in self.reset:
            val = eval(code, self._env(S, I_in, t))
            new = val if op is None else op(S[tgt], val)
            S[tgt] = np.where(mask, np.asarray(new, dtype=self.dtype), S[tgt]).astype(self.dtype)


def simulate(model, S0, I, I_offset, nsteps, spiketimes, spk_offset, spk_end, delay=None, refractory=None,
             delta=40, exclusive=True, onset=0, Tstart=0, Tend=None, carry=None, record=False):
    """runsim (gpu_modelfitting.py:39-116) for every simulation.

    S0: [nstate][ns] initial state (doubles, converted to the scalar type);
    I: all inputs (converted); spiketimes: int steps with sentinels.
    Returns a dict with coinc, nspikes, state and the carried pointers; with
    record=True also the spike steps of every simulation."""
    dt_ = model.dtype
    ns = S0.shape[1]
    nsteps = np.asarray(nsteps, dtype=np.int64)
    I = np.asarray(I, dtype=np.float64).astype(dt_)
    I_offset = np.asarray(I_offset, dtype=np.int64)
    spk = np.asarray(spiketimes, dtype=np.int64)
    spk_end = np.asarray(spk_end, dtype=np.int64)
    delay = np.zeros(ns, dtype=np.int64) if delay is None else np.asarray(delay, dtype=np.int64)
    refractory = np.zeros(ns, dtype=np.int64) if refractory is None else np.asarray(refractory, dtype=np.int64)
    BIG = 2 ** 31 - 1
    if carry is None:
        S = {v: np.asarray(S0[k], dtype=np.float64).astype(dt_) for k, v in enumerate(model.state)}
        idx = np.asarray(spk_offset, dtype=np.int64).copy()
        last_allowed = np.zeros(ns, dtype=bool)
        next_allowed = np.ones(ns, dtype=bool)
        ncoinc = np.zeros(ns, dtype=np.int64)
        nspk = np.zeros(ns, dtype=np.int64)
        next_allowed_T = -np.ones(ns, dtype=np.int64)
        rec = [[] for _ in range(ns)]
    else:
        S = {v: carry["S"][v].copy() for v in model.state}
        idx = carry["idx"].copy()
        last_allowed = carry["last_allowed"].copy()
        next_allowed = carry["next_allowed"].copy()
        ncoinc = carry["ncoinc"].copy()
        nspk = carry["nspikes"].copy()
        next_allowed_T = carry["next_allowed_T"].copy()
        rec = [list(r) for r in carry["rec"]]
    last_idx = spk_end - 1
    last_spike = spk[idx]
    next_spike = np.where(idx < last_idx, spk[np.minimum(idx + 1, len(spk) - 1)], BIG)
    if Tend is None:
        Tend = int(nsteps.max()) if ns else 0
    Tend_i = np.minimum(Tend, nsteps)
    for T in range(Tstart, int(Tend_i.max()) if ns else Tstart):
        active = T < Tend_i
        if not active.any():
            break
        t = dt_(np.float64(T) * model.dt)
        I_in = I[np.where(active, I_offset + T, 0)]
        old = {v: S[v] for v in model.state}
        model.update(S, I_in, t)
        for v in model.state:
            S[v] = np.where(active, S[v], old[v]).astype(dt_)
        is_refr = T <= next_allowed_T
        has = model.spiking(S, I_in, t) & ~is_refr & active
        nspk += (has & (T >= onset)).astype(np.int64)
        model.apply_reset(S, I_in, t, (has | is_refr) & active)
        next_allowed_T = np.where(has, T + refractory, next_allowed_T)
        if record:
            for i in np.nonzero(has)[0]:
                rec[i].append(T)
        Tsp = T + delay
        if exclusive:
            near_last = has & (last_spike + delta >= Tsp)
            near_next = has & (next_spike - delta <= Tsp)
            ml = near_last & last_allowed
            mn = near_next & next_allowed
            ncoinc += (ml | mn).astype(np.int64)
            last_allowed = last_allowed & ~near_last
            next_allowed = (next_allowed & ~near_next) | (ml & mn)
        else:
            ncoinc += (has & ((last_spike + delta >= Tsp) | (next_spike - delta <= Tsp))).astype(np.int64)
        move = active & (Tsp >= next_spike)
        if move.any():
            idx = np.where(move, idx + 1, idx)
            last_spike = np.where(move, next_spike, last_spike)
            nxt = np.where(idx < last_idx, spk[np.minimum(idx + 1, len(spk) - 1)], BIG)
            next_spike = np.where(move, nxt, next_spike)
            if exclusive:
                last_allowed = np.where(move, next_allowed, last_allowed)
                next_allowed = np.where(move, True, next_allowed)
    return {"coinc": ncoinc, "nspikes": nspk, "S": S, "idx": idx, "last_allowed": last_allowed,
            "next_allowed": next_allowed, "ncoinc": ncoinc, "next_allowed_T": next_allowed_T, "rec": rec,
            "state": np.array([S[v].astype(np.float64) for v in model.state])}


def firing_rate(spikes):
    """(n - 1) / (t_last - t_first), NaN below two spikes (statistics.py:15-21)."""
    spikes = np.asarray(spikes, dtype=np.float64)
    if len(spikes) < 2:
        return np.nan
    return (len(spikes) - 1) / (spikes[-1] - spikes[0])


def gamma(coinc, nspikes, target_length, target_rate, delta):
    """get_gamma_factor (statistics.py:236-240) in numpy's evaluation order."""
    coinc = np.asarray(coinc, dtype=np.int64)
    model_length = np.asarray(nspikes, dtype=np.int64)
    target_length = np.asarray(target_length, dtype=np.int64)
    target_rates = np.asarray(target_rate, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        NCoincAvg = 2 * delta * target_length * target_rates
        norm = .5 * (1 - 2 * delta * target_rates)
        return (coinc - NCoincAvg) / (norm * (target_length + model_length))


def offline_coincidences(source, target, delta_steps):
    """Number of target spikes with a source spike within delta_steps of the
    nearest source spike (gamma_factor with normalize=False and dt given,
    statistics.py:261-314), on integer step trains."""
    source = np.asarray(source, dtype=np.int64)
    target = np.asarray(target, dtype=np.int64)
    if len(source) == 0 or len(target) == 0:
        return 0
    if len(source) > 1:
        bins = .5 * (source[1:] + source[:-1])
        indices = np.digitize(target, bins)
        return int(np.sum(np.abs(target - source[indices]) <= delta_steps))
    return int(sum(np.amin(np.abs(source - t)) <= delta_steps for t in target))


def pso_move(X, V, Xl, Xg, lo, hi, omega, c1, c2, seed, it, group_size):
    """One swarm move (particle_swarm.py:68-77) with Philox draws."""
    N, M = X.shape
    k = np.arange(N * M, dtype=np.int64).reshape(N, M)
    R1 = philox_uniform(seed, 2 * it, k)
    R2 = philox_uniform(seed, 2 * it + 1, k)
    G = M // group_size
    Xg2 = np.repeat(Xg, group_size, axis=1) if G else Xg
    V = omega * V + c1 * R1 * (Xl - X) + c2 * R2 * (Xg2 - X)
    X = X + V
    X = np.maximum(X, lo.reshape(-1, 1))
    X = np.minimum(X, hi.reshape(-1, 1))
    return X, V


def pso_best(X, fit, Xl, lfit, Xg, gfit, group_size):
    """Local and group best updates (particle_swarm.py:88-103); NaN never
    wins, the first particle holding a group's maximum is taken."""
    better = fit > lfit
    Xl = Xl.copy()
    lfit = lfit.copy()
    Xl[:, better] = X[:, better]
    lfit[better] = fit[better]
    Xg = Xg.copy()
    gfit = gfit.copy()
    G = len(gfit)
    for j in range(G):
        f = fit[j * group_size:(j + 1) * group_size]
        f = np.where(np.isnan(f), -np.inf, f)
        m = f.max()
        if m > gfit[j]:
            i = int(np.nonzero(f == m)[0][0])
            Xg[:, j] = X[:, j * group_size + i]
            gfit[j] = m
    return Xl, lfit, Xg, gfit


def pso_reference(X0, fun, iterations, pso_params, min_values, max_values, group_size, seed):
    """particle_swarm (particle_swarm.py:6-111) with Philox draws; fun maps an
    N x M matrix to M fitness values.  Returns (X_gbest, fitness_gbest,
    history of (X, V, fit) per iteration)."""
    N, M = X0.shape
    omega, c1, c2 = pso_params
    lo = np.asarray(min_values, dtype=np.float64)
    hi = np.asarray(max_values, dtype=np.float64)
    X = np.minimum(np.maximum(X0, lo.reshape(-1, 1)), hi.reshape(-1, 1))
    V = np.zeros((N, M))
    Xl = X.copy()
    lfit = -np.inf * np.ones(M)
    G = M // group_size
    Xg = X[:, np.arange(0, M, group_size)].copy()
    gfit = -np.inf * np.ones(G)
    hist = []
    for it in range(iterations):
        X, V = pso_move(X, V, Xl, Xg, lo, hi, omega, c1, c2, seed, it, group_size)
        fit = np.asarray(fun(X), dtype=np.float64)
        Xl, lfit, Xg, gfit = pso_best(X, fit, Xl, lfit, Xg, gfit, group_size)
        hist.append((X.copy(), V.copy(), fit.copy(), gfit.copy()))
    return Xg, gfit, hist
