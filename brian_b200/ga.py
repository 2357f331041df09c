"""Genetic algorithm for model fitting: one independent population per
target group.

The reference's ``modelfitting`` offers a GA (``algorithm=GA``) from the
external playdoh package, which is not part of the reference tree.  This is
a real-coded GA built from published operators, run on the host for every
group at once; the candidates of a generation, of all groups, are evaluated
together on the device by the caller:

* binary tournament selection (D. E. Goldberg and K. Deb, "A comparative
  analysis of selection schemes used in genetic algorithms", FOGA 1991);
* BLX-alpha crossover (L. J. Eshelman and J. D. Schaffer, "Real-coded
  genetic algorithms and interval-schemata", FOGA 1993): each child gene
  uniform in [min - alpha*d, max + alpha*d] of the parents' genes, d their
  distance;
* Gaussian mutation of each gene with probability ``mutation`` (default
  1/n) and standard deviation ``sigma``;
* elitism: the ``elite`` best individuals pass unchanged.

Genes live in the mapminmax-scaled space [-1, 1] of the initial range and
are clipped to the scaled parameter bounds; fitness is maximised, NaN is
the worst value.
"""
import numpy as np


class GAState(object):
    defaults = {"elite": None, "tournament": 2, "crossover": 0.8, "alpha": 0.5, "mutation": None, "sigma": 0.1}

    def __init__(self, G, n, pop, X0, rng, lo=None, hi=None, **opt):
        o = dict(self.defaults)
        o.update({k: v for k, v in opt.items() if k in self.defaults})
        self.G, self.n, self.pop = G, n, pop
        self.rng = rng
        self.elite = max(1, pop // 20) if o["elite"] is None else int(o["elite"])
        self.k = int(o["tournament"])
        self.pc, self.alpha = float(o["crossover"]), float(o["alpha"])
        self.pm = 1.0 / n if o["mutation"] is None else float(o["mutation"])
        self.sigma = float(o["sigma"])
        self.lo = np.full(n, -np.inf) if lo is None else np.asarray(lo, dtype=np.float64)
        self.hi = np.full(n, np.inf) if hi is None else np.asarray(hi, dtype=np.float64)
        self.X = np.clip(np.asarray(X0, dtype=np.float64).reshape(G, pop, n), self.lo, self.hi)

    def ask(self):
        """The current population [G][pop][n]."""
        return self.X

    def tell(self, fit):
        """Next generation from the fitness [G][pop] of the current one."""
        G, P, n, rng = self.G, self.pop, self.n, self.rng
        f = np.where(np.isnan(fit), -np.inf, np.asarray(fit, dtype=np.float64))
        order = np.argsort(-f, axis=1, kind="stable")
        gi = np.arange(G)[:, None]
        elite = self.X[gi, order[:, :self.elite]]
        nchild = P - self.elite

        def tournament(m):
            cand = rng.integers(0, P, size=(G, m, self.k))
            best = np.take_along_axis(cand, np.argmax(f[gi[:, :, None], cand], axis=2)[:, :, None], axis=2)[:, :, 0]
            return self.X[gi, best]                                   # [G][m][n]

        pa, pb = tournament(nchild), tournament(nchild)
        lo, hi = np.minimum(pa, pb), np.maximum(pa, pb)
        d = hi - lo
        blend = lo - self.alpha * d + rng.random((G, nchild, n)) * (1 + 2 * self.alpha) * d
        cross = rng.random((G, nchild, 1)) < self.pc
        child = np.where(cross, blend, pa)
        mut = rng.random((G, nchild, n)) < self.pm
        child = child + mut * rng.standard_normal((G, nchild, n)) * self.sigma
        self.X = np.clip(np.concatenate([elite, child], axis=1), self.lo, self.hi)


def maximize_check(fun, n, pop=50, iters=200, seed=0, lo=-5.0, hi=5.0):
    """One population maximising -fun(x) on a box (a host check)."""
    rng = np.random.default_rng(seed)
    X0 = lo + (hi - lo) * rng.random((1, pop, n))
    st = GAState(1, n, pop, X0, rng, lo=np.full(n, lo), hi=np.full(n, hi))
    best = np.inf
    for _ in range(iters):
        X = st.ask()
        fv = np.array([fun(x) for x in X[0]])
        best = min(best, fv.min())
        st.tell(-fv[None, :])
    return best
