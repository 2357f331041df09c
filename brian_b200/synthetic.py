"""Seeded synthetic fitting workloads: Ornstein-Uhlenbeck input currents and
target spike trains of a hidden adaptive-threshold LIF.

The model (all values SI, as Brian holds them with units stripped):

    dV/dt  = (R*I - V) / tau
    dVt/dt = (Vt0 - Vt) / tau_t
    threshold V > Vt;  reset V = 0; Vt += alpha

Its five parameters are drawn log-uniform over PRIOR, whose ranges put the
firing rates of the OU-driven targets in 5-40 Hz.  The OU current uses the
exact discretisation I[k+1] = mu + (I[k] - mu) e^{-dt/tau} + sd sqrt(1 -
e^{-2 dt/tau}) N(0, 1) (the process of library/random_processes.py:13-38,
sampled exactly), from numpy's PCG64 generator.
"""
import numpy as np

__all__ = ["ADAPTIVE_LIF", "ADAPTIVE_LIF_BASIS", "THRESHOLD", "RESET", "PARAMS", "PRIOR", "ou_current", "sample_prior",
           "adaptive_lif_equations", "make_targets", "FitWorkload"]

ADAPTIVE_LIF = """
dV/dt = (R*I - V)/tau : 1
dVt/dt = (Vt0 - Vt)/tau_t : 1
I : 1
R : 1
tau : 1
Vt0 : 1
alpha : 1
tau_t : 1
"""
THRESHOLD = "V > Vt"
RESET = "V = 0\nVt += alpha"
PARAMS = ("R", "tau", "Vt0", "alpha", "tau_t")
# log-uniform ranges of the hidden parameters (ohm, s, V, V, s)
PRIOR = {"R": (2.5e7, 5e7), "tau": (5e-3, 2e-2), "Vt0": (1.5e-2, 2.5e-2), "alpha": (2e-3, 1e-2),
         "tau_t": (5e-2, 2e-1)}


# The adaptive LIF's spike train is unchanged when R, Vt0 and alpha are all
# scaled by one factor (V and Vt scale with it and both start at 0); in the
# coordinates (log R, log tau, log Vt0 - log R, log alpha - log R, log tau_t)
# only the first carries that freedom.
ADAPTIVE_LIF_BASIS = [[1, 0, 0, 0, 0],
                      [0, 1, 0, 0, 0],
                      [-1, 0, 1, 0, 0],
                      [-1, 0, 0, 1, 0],
                      [0, 0, 0, 0, 1]]


def adaptive_lif_equations():
    from .equations import Equations
    return Equations(ADAPTIVE_LIF, dummy=0.0)


def ou_current(n, dt, rng, tau=10e-3, mu=0.6e-9, sd=0.3e-9):
    """n samples of a stationary OU process with exact updates, x[0] drawn
    from the stationary law (the recursion runs as a first-order filter)."""
    from scipy.signal import lfilter
    a = np.exp(-dt / tau)
    b = sd * np.sqrt(1.0 - a * a)
    z = rng.standard_normal(n)
    drive = b * z
    drive[0] = sd * z[0]
    return mu + lfilter([1.0], [1.0, -a], drive)


def sample_prior(n, rng, prior=PRIOR):
    """[5][n] parameters, log-uniform per PARAMS."""
    out = np.empty((len(PARAMS), n))
    for d, k in enumerate(PARAMS):
        lo, hi = prior[k]
        out[d] = np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * rng.random(n))
    return out


def make_targets(inputs, params, dt, precision="double", method="Euler"):
    """Spike times (seconds) of the hidden model for each (input, parameter
    column) pair, simulated by the fitting kernel; list of arrays."""
    from .modelfitting import get_spikes
    kw = {k: params[d] for d, k in enumerate(PARAMS)}
    n = params.shape[1]
    spikes = get_spikes(model=adaptive_lif_equations(), reset=RESET, threshold=THRESHOLD, input=list(inputs),
                        dt=dt, method=method, precision=precision, **kw)
    out = [[] for _ in range(n)]
    for i, t in spikes:
        out[i].append(t)
    return [np.array(x) for x in out]


class FitWorkload(object):
    """`ntargets` targets with OU inputs of durations uniform in
    [dur_min, dur_max] seconds and hidden parameters from the prior."""

    def __init__(self, ntargets=64, dur_min=1.0, dur_max=20.0, dt=1e-4, seed=1234, prior=PRIOR):
        self.rng = np.random.default_rng(seed)
        self.dt = dt
        self.ntargets = ntargets
        self.durations = self.rng.uniform(dur_min, dur_max, ntargets)
        self.nsamples = np.maximum(1, np.round(self.durations / dt).astype(np.int64))
        self.inputs = [ou_current(int(n), dt, self.rng) for n in self.nsamples]
        self.prior = prior
        self.hidden = sample_prior(ntargets, self.rng, prior)
        self.targets = None

    def build_targets(self, precision="double", rate_range=(5.0, 40.0), max_rounds=20):
        """Target trains of the hidden parameters; targets whose rate falls
        outside `rate_range` get new hidden parameters (at most max_rounds
        redraws)."""
        self.targets = make_targets(self.inputs, self.hidden, self.dt, precision=precision)
        for _ in range(max_rounds):
            rates = np.array([len(t) / d for t, d in zip(self.targets, self.durations)])
            bad = np.nonzero((rates < rate_range[0]) | (rates > rate_range[1]))[0]
            if len(bad) == 0:
                break
            self.hidden[:, bad] = sample_prior(len(bad), self.rng, self.prior)
            redo = make_targets([self.inputs[j] for j in bad], self.hidden[:, bad], self.dt, precision=precision)
            for j, t in zip(bad, redo):
                self.targets[j] = t
        return self.targets

    def data(self):
        """(index, time) pairs for modelfitting()."""
        rows = [(j, t) for j, tr in enumerate(self.targets) for t in tr]
        return np.array(rows, dtype=np.float64).reshape(-1, 2)
