"""Learned proposals for model fitting.

A network maps features of a target spike train and its input (log-ISI
histogram, firing rate, CV and spike-triggered average, computed on the
device from the train) to a diagonal Gaussian over the model's fitted
parameters, normalised to [-1, 1] on a log scale of the prior's ranges.  It is
trained only on (parameters, simulated train) pairs that the batched fitting
kernel generates from the prior, with hand-written tensor-core kernels for
every forward and backward product.  Its proposals are re-simulated and
scored by the gamma factor like any other candidate; the particle swarm then
refines from them, so the swarm stays the fallback for targets the network
places badly.

The reference has no counterpart: its optimisers start from uniform draws
(library/modelfitting/modelfitting.py:479-516, tools/particle_swarm.py:
51-57).
"""
import time

import numpy as np

from . import _lib
from .codegen import generate_model_code

__all__ = ["ProposalNetwork", "simulate_training_set", "target_features"]


class _TrainingSimulator(object):
    """One fitting handle that simulates chunks of prior draws over a pool of
    input traces and returns their features."""

    def __init__(self, model, threshold, reset, names, inputs, dt, chunk, precision="float", method="Euler",
                 initial_values=None, record=256, input_var="I", device=0, durations=None):
        self.code = generate_model_code(model, threshold, reset, dt, input_var=input_var,
                                        scalar="float" if precision == "float" else "double", scheme=method)
        self.h = h = _lib.FitHandle(self.code, dt, 40, exclusive=True, precision=32 if precision == "float" else 64,
                                    device=device)
        lens = np.array([len(x) for x in inputs], dtype=np.int64)
        I = np.concatenate([np.asarray(x, dtype=np.float64) for x in inputs])
        ioff = np.concatenate([[0], np.cumsum(lens)[:-1]])
        h.set_input(I)
        trains = np.concatenate([[-10000, int(n) + 10000] for n in lens]).astype(np.int32)
        h.set_targets(trains)
        h.set_record(record)
        k = np.arange(chunk) % len(inputs)
        S0 = np.zeros((len(self.code.state), chunk))
        for name, v in (initial_values or {}).items():
            S0[self.code.index(name)] = v
        nsteps = lens[k] if durations is None else np.minimum(lens[k], np.asarray(durations, dtype=np.int64))
        h.set_sims(S0, ioff[k], nsteps, 2 * k, 2 * k + 2)
        h.set_gamma(chunk, 1, np.zeros(chunk, np.int32), np.full(chunk, np.nan), 4e-3)
        h.set_params([self.code.index(n) for n in names])
        self.chunk = chunk

    def features(self, theta):
        """Features of the simulations of theta [ndim][chunk]."""
        self.h.evaluate(theta)
        return self.h.features()

    def close(self):
        self.h.close()


def sample_log_uniform(prior, names, n, rng):
    out = np.empty((len(names), n))
    for d, k in enumerate(names):
        lo, hi = prior[k]
        out[d] = np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * rng.random(n))
    return out


def simulate_training_set(model, threshold, reset, prior, inputs, dt, n, seed=0, chunk=131072, precision="float",
                          method="Euler", initial_values=None, record=1024, input_var="I", device=0,
                          duration_range=None):
    """n (features, parameters) pairs: parameters drawn log-uniform from
    `prior` (name -> (lo, hi)), simulation i driven by (the start of)
    inputs[i % len] for a duration drawn uniformly from `duration_range`
    seconds (default: the whole input), its features from the recorded
    train.  Returns (X [n][64] float32, theta [ndim][n], seconds)."""
    names = list(prior)
    rng = np.random.default_rng(seed)
    chunk = int(min(chunk, n))
    durations = None
    if duration_range is not None:
        durations = np.round(rng.uniform(duration_range[0], duration_range[1], chunk) / dt).astype(np.int64)
    sim = _TrainingSimulator(model, threshold, reset, names, inputs, dt, chunk, precision, method, initial_values,
                             record, input_var, device, durations)
    X = np.empty((n, 64), dtype=np.float32)
    theta = np.empty((len(names), n))
    t0 = time.time()
    for a in range(0, n, chunk):
        th = sample_log_uniform(prior, names, chunk, rng)
        F = sim.features(th)
        b = min(n, a + chunk)
        X[a:b] = F[:b - a]
        theta[:, a:b] = th[:, :b - a]
    el = time.time() - t0
    sim.close()
    return X, theta, el


def target_features(trains, inputs, dt, device=0):
    """Features of target trains (spike times in seconds) with their inputs."""
    steps = [np.asarray(np.rint(np.asarray(t, dtype=np.float64) / dt), dtype=np.int32) for t in trains]
    return _lib.spike_features(steps, inputs, dt, device=device)


class ProposalNetwork(object):
    """The proposal network for the parameters of `prior` (name -> (lo, hi),
    log scale).

    The network's Gaussian is diagonal in the coordinates u = basis . log(theta)
    (basis: an invertible ndim x ndim matrix, identity by default), each
    coordinate mapped to [-1, 1] over the prior box.  A basis aligned with a
    model's symmetries -- directions along which the spike train does not
    change -- lets a diagonal Gaussian describe the posterior's shape."""

    def __init__(self, prior, device=0, seed=0, basis=None):
        self.names = list(prior)
        self.ydim = len(self.names)
        self.log_lo = np.log(np.array([prior[k][0] for k in self.names], dtype=np.float64))
        self.log_hi = np.log(np.array([prior[k][1] for k in self.names], dtype=np.float64))
        self.basis = np.eye(self.ydim) if basis is None else np.asarray(basis, dtype=np.float64)
        self.inv_basis = np.linalg.inv(self.basis)
        # range of every coordinate over the corners of the prior box
        corners = np.array(np.meshgrid(*[[0, 1]] * self.ydim, indexing="ij")).reshape(self.ydim, -1)
        logs = self.log_lo.reshape(-1, 1) + (self.log_hi - self.log_lo).reshape(-1, 1) * corners
        u = self.basis @ logs
        self.u_lo = u.min(axis=1)
        self.u_hi = u.max(axis=1)
        self.net = _lib.MLPHandle(self.ydim, device=device)
        rng = np.random.default_rng(seed)
        for l in range(4):
            rows, cols = _lib.MLP_ROWS[l], _lib.MLP_COLS[l]
            W = rng.standard_normal((rows, cols)) * np.sqrt(2.0 / cols)
            if l == 3:
                W *= 0.05
                W[2 * self.ydim:] = 0.0
            self.net.set_params(l, W.astype(np.float32), np.zeros(rows, dtype=np.float32))
        self.mean = np.zeros(64, dtype=np.float32)
        self.std = np.ones(64, dtype=np.float32)
        self.last_ms = 0.0

    # ------------------------------------------------------------ scaling
    def encode(self, theta):
        """[ndim][n] parameters -> [n][ndim] network coordinates in [-1, 1]."""
        u = self.basis @ np.log(np.asarray(theta, dtype=np.float64))
        z = 2.0 * (u.T - self.u_lo) / (self.u_hi - self.u_lo) - 1.0
        return z.astype(np.float32)

    def decode(self, z):
        """[n][ndim] network coordinates -> [ndim][n] parameters."""
        u = self.u_lo + (np.asarray(z, dtype=np.float64) + 1.0) * 0.5 * (self.u_hi - self.u_lo)
        return np.exp(self.inv_basis @ u.T)

    def scale(self, X):
        return ((np.asarray(X, dtype=np.float32) - self.mean) / self.std).astype(np.float32)

    # ----------------------------------------------------------- training
    def train(self, X, theta, epochs=20, batch=4096, lr=1e-3, seed=0):
        """Fit on features X [n][64] and parameters theta [ndim][n]; returns
        (epoch losses, GPU milliseconds)."""
        X = np.asarray(X, dtype=np.float32)
        ok = np.all(np.isfinite(X), axis=1)
        X = X[ok]
        Z = self.encode(np.asarray(theta)[:, ok])
        self.mean = X.mean(axis=0)
        self.std = np.maximum(X.std(axis=0), 1e-6).astype(np.float32)
        n = (len(X) // batch) * batch
        self.net.set_data(self.scale(X[:n]), Z[:n])
        return self.net.train(epochs, batch, lr, seed)

    def predict(self, X):
        """Means and standard deviations in network coordinates; the device
        time of the pass is left in last_ms."""
        out = self.net.forward(self.scale(X))
        self.last_ms = self.net.last_forward_ms()
        mu = out[:, :self.ydim]
        sigma = np.exp(np.clip(out[:, self.ydim:2 * self.ydim], -7.0, 7.0))
        return mu, sigma

    def sample(self, X, n_per, rng, widen=1.0, clip=1.25):
        """n_per proposals per row of X: parameters [ndim][rows * n_per],
        target-major (row j's proposals are columns j*n_per .. ); the first
        proposal of every row is the predicted mean."""
        mu, sigma = self.predict(X)
        z = mu[:, None, :] + widen * sigma[:, None, :] * rng.standard_normal((len(mu), n_per, self.ydim))
        z[:, 0, :] = mu
        z = np.clip(z, -clip, clip).reshape(-1, self.ydim)
        return self.decode(z)


def _fraction_time(hits, frac):
    """Earliest time at which `frac` of the targets have a hit (inf if never)."""
    h = np.sort(np.asarray(hits, dtype=np.float64))
    k = int(np.ceil(frac * len(h))) - 1
    return float(h[max(k, 0)]) if len(h) else 0.0


def _swarm(prob, X0, box_lo, box_hi, pso, seed, goal, max_iter, t_start, chunk=5, inspect=None):
    """Swarm from X0 until every group's best reaches `goal` or max_iter;
    returns (per-group first time at goal in ms from t_start, final bests,
    iterations, GPU ms).  `inspect(fit_lbest)` sees the first evaluation."""
    h = prob.handle
    h.pso_init(prob.popsize, X0, box_lo, box_hi, pso[0], pso[1], pso[2], seed)
    h.pso_evaluate_initial()
    if inspect is not None:
        inspect(h.pso_state()[3])
    t = t_start + h.stats()["last_eval_ms"]
    best = h.pso_best()[1]
    hits = np.where(best >= goal, t, np.inf)
    it = 0
    while it < max_iter and np.any(~np.isfinite(hits)):
        n = min(chunk, max_iter - it)
        tr, ms = h.pso_run(n)
        for k in range(n):
            t += float(ms[k])
            newly = (~np.isfinite(hits)) & (tr[k] >= goal)
            hits[newly] = t
        it += n
    return hits, h.pso_best()[1], it, t - t_start


def race(model, threshold, reset, targets, inputs, dt, box, net=None, popsize=1024, n_prop=64, max_iter=50,
         goal=0.9, precision="float", seed=0, pso=(0.7298, 1.49618, 1.49618), method="Euler", initial_values=None,
         widen=1.25, device=0, arms=("plain", "learned"), refine_popsize=None):
    """GPU time until each target's fitted gamma reaches `goal`.

    Plain: the swarm from uniform draws over `box` (name -> (lo, hi)).
    Learned (when `net` is given): the network proposes n_prop parameter sets
    per target from the target's features; a swarm of refine_popsize
    particles per target (default popsize) starts from those proposals plus
    draws from the network's Gaussian widened by `widen`; its first
    evaluation re-simulates and scores the proposals, its iterations refine
    them.  Every time is device time from CUDA
    events, plus the network's own (timed on the host around synchronous
    calls).  Returns a dict per arm with per-target hit times (ms), final
    best gamma and summary times."""
    from .modelfitting import FittingProblem
    names = list(box)
    lo = np.array([box[k][0] for k in names], dtype=np.float64)
    hi = np.array([box[k][1] for k in names], dtype=np.float64)
    G = len(targets)
    rng = np.random.default_rng(seed)
    out = {}

    def summary(hits, best, gpu_ms, extra):
        d = {"hits_ms": hits.tolist(), "best_gamma": np.asarray(best).tolist(), "gpu_ms": gpu_ms,
             "t50_ms": _fraction_time(hits, 0.5), "t90_ms": _fraction_time(hits, 0.9),
             "t100_ms": _fraction_time(hits, 1.0), "reached": float(np.mean(np.isfinite(hits))),
             "median_best_gamma": float(np.median(best))}
        d.update(extra)
        return d

    # plain swarm
    if "plain" in arms:
        prob = FittingProblem(model, threshold, reset, targets, inputs, dt, popsize, precision=precision,
                              method=method, param_names=names, initial_values=initial_values, device=device)
        X0 = lo.reshape(-1, 1) + (hi - lo).reshape(-1, 1) * rng.random((len(names), prob.N))
        pfirst = {}

        def pinspect(lfit):
            f = np.where(np.isnan(lfit), -np.inf, lfit).reshape(G, popsize)
            pfirst["all"] = float(np.mean(f.max(axis=1) >= goal))

        hits, best, iters, ms = _swarm(prob, X0, lo, hi, pso, seed + 1, goal, max_iter, 0.0, inspect=pinspect)
        out["plain"] = summary(hits, best, ms, {"iterations": iters, "first_evaluation_reached": pfirst.get("all")})
        prob.handle.close()
    else:
        rng.random((len(names), G * popsize))      # same draws afterwards either way
    if net is None or "learned" not in arms:
        return out

    # learned: features of the targets (inputs already on the device), the
    # network, then one swarm whose first evaluation re-simulates the n_prop
    # proposals of every target together with popsize - n_prop further draws
    # from the network's Gaussian (widened); the swarm refines from there
    rp = int(refine_popsize or popsize)
    prob = FittingProblem(model, threshold, reset, targets, inputs, dt, rp, precision=precision, method=method,
                          param_names=names, initial_values=initial_values, device=device)
    t0 = time.perf_counter()
    steps = [np.asarray(np.rint(np.asarray(t, dtype=np.float64) / dt), dtype=np.int32) for t in targets]
    F, t_feat = prob.handle.train_features(steps, prob.input_offsets)
    P = net.sample(F, n_prop, rng, widen=1.0)
    t_net = t_feat + net.last_ms
    extra = net.sample(F, rp - n_prop, rng, widen=widen)
    wall_net = (time.perf_counter() - t0) * 1e3
    X0 = np.empty((len(names), G * rp))
    for j in range(G):
        X0[:, j * rp:j * rp + n_prop] = P[:, j * n_prop:(j + 1) * n_prop]
        X0[:, j * rp + n_prop:(j + 1) * rp] = extra[:, j * (rp - n_prop):(j + 1) * (rp - n_prop)]
    X0 = np.minimum(np.maximum(X0, lo.reshape(-1, 1)), hi.reshape(-1, 1))
    first = {}

    def inspect(lfit):
        f = np.where(np.isnan(lfit), -np.inf, lfit).reshape(G, rp)
        first["proposals"] = float(np.mean(f[:, :n_prop].max(axis=1) >= goal))
        first["all"] = float(np.mean(f.max(axis=1) >= goal))

    hits, best, iters, ms = _swarm(prob, X0, lo, hi, pso, seed + 2, goal, max_iter, t_net, inspect=inspect)
    prob.handle.close()
    out["learned"] = summary(hits, best, t_net + ms,
                             {"iterations": iters, "network_ms": t_net, "network_wall_ms": wall_net,
                              "refine_popsize": rp,
                              "first_evaluation_reached": first.get("all"),
                              "proposals_only_reached": first.get("proposals")})
    return out
