"""GA of modelfitting (brian_b200/ga.py), checked on the host: standard
test functions, independent groups, elitism, NaN fitness, and the
modelfitting plumbing around it with a stand-in evaluator."""
import importlib

import numpy as np

from brian_b200.ga import GAState, maximize_check

mf = importlib.import_module("brian_b200.modelfitting")


def test_sphere_and_rosenbrock():
    assert maximize_check(lambda x: float(np.sum(x ** 2)), 5, pop=60, iters=300, seed=1) < 1e-4
    rosen = lambda x: float(np.sum(100 * (x[1:] - x[:-1] ** 2) ** 2 + (1 - x[:-1]) ** 2))
    assert maximize_check(rosen, 3, pop=80, iters=400, seed=2, lo=-2.0, hi=2.0) < 1e-2


def test_groups_independent_elitism_and_nan():
    rng = np.random.default_rng(3)
    targets = np.array([[0.5, -0.2], [-0.7, 0.1], [0.0, 0.9]])
    st = GAState(3, 2, 40, rng.uniform(-1, 1, (3, 40, 2)), rng, lo=np.full(2, -1.0), hi=np.full(2, 1.0))
    prev = np.full(3, -np.inf)
    for it in range(120):
        X = st.ask()
        f = -np.sum((X - targets[:, None, :]) ** 2, axis=2)
        f[:, -1] = np.nan                     # never selected as an elite
        best = np.nanmax(f, axis=1)
        assert np.all(best >= prev)           # the elite carries the best forward
        prev = best
        st.tell(f)
    X = st.ask()
    dist = np.min(np.sum((X - targets[:, None, :]) ** 2, axis=2), axis=1)
    assert np.all(dist < 1e-4)
    assert np.all(np.abs(X) <= 1.0)


class _FakeHandle(object):
    def stats(self):
        return {"last_eval_ms": 0.0}


class _FakeProblem(object):
    """Fitness of each candidate column: minus its squared distance to the
    target of its group (candidates group-major)."""

    def __init__(self, targets, popsize):
        self.targets, self.popsize, self.handle = targets, popsize, _FakeHandle()

    def evaluate(self, X):
        G = len(self.targets)
        P = X.reshape(X.shape[0], G, self.popsize).transpose(1, 2, 0)
        return -np.sum((P - self.targets[:, None, :]) ** 2, axis=2).ravel()

    def neuron_steps(self):
        return 0


def test_fit_ga_plumbing():
    targets = np.array([[12e-3, 3.0], [18e-3, 7.5]])
    lo, hi = np.array([5e-3, 0.0]), np.array([30e-3, 10.0])
    imin, imax = np.array([8e-3, 1.0]), np.array([25e-3, 9.0])
    res = mf._fit_ga(_FakeProblem(targets, 60), ["tau", "R"], lo, hi, imin, imax, 2, 60, 150,
                     np.random.default_rng(5), None, None)
    assert res.info["algorithm"] == "GA" and res.info["trace"].shape == (150, 2)
    for j in range(2):
        got = np.array([res.best_pos[j]["tau"], res.best_pos[j]["R"]])
        assert np.allclose(got, targets[j], rtol=1e-3, atol=1e-4), (got, targets[j])
