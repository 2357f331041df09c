"""CMA-ES for model fitting: one independent search per target group.

The reference's `modelfitting` uses CMA-ES by default (modelfitting.py:256,
`algorithm=CMAES`, with `scaling='mapminmax'`, :442-443); its implementation
lives in the external playdoh package.  This is the published algorithm
(N. Hansen, "The CMA Evolution Strategy: A Tutorial", arXiv:1604.00772,
Table 1 defaults with positive recombination weights), run on the host for
every group at once; the candidates of a generation, of all groups, are
evaluated together on the device by the caller.

Search space: parameters mapped to [-1, 1] over their initial range
(mapminmax); candidates are clipped to the parameter bounds for evaluation
only, the distribution is updated with the unclipped samples.  Fitness is
maximised (gamma); NaN counts as the worst value.
"""
import numpy as np


class CMAState(object):
    """Distributions of G independent CMA-ES searches in n dimensions with
    population lam (Hansen 2016, Table 1 and the update of Fig. 7)."""

    def __init__(self, G, n, lam, mean, sigma, rng):
        self.G, self.n, self.lam = G, n, lam
        self.rng = rng
        mu = lam // 2
        w = np.log((lam + 1) / 2.0) - np.log(np.arange(1, mu + 1))
        self.w = w / w.sum()
        self.mu = mu
        self.mueff = 1.0 / np.sum(self.w ** 2)
        me = self.mueff
        self.cs = (me + 2) / (n + me + 5)
        self.ds = 1 + 2 * max(0.0, np.sqrt((me - 1) / (n + 1)) - 1) + self.cs
        self.cc = (4 + me / n) / (n + 4 + 2 * me / n)
        self.c1 = 2 / ((n + 1.3) ** 2 + me)
        self.cmu = min(1 - self.c1, 2 * (me - 2 + 1 / me) / ((n + 2) ** 2 + me))
        self.chi = np.sqrt(n) * (1 - 1 / (4 * n) + 1 / (21 * n * n))
        self.m = np.array(mean, dtype=np.float64).reshape(G, n)
        self.sigma = np.full(G, float(sigma))
        self.C = np.tile(np.eye(n), (G, 1, 1))
        self.B = np.tile(np.eye(n), (G, 1, 1))
        self.D = np.ones((G, n))
        self.ps = np.zeros((G, n))
        self.pc = np.zeros((G, n))
        self.gen = 0

    def ask(self):
        """Candidates [G][lam][n] and their steps y = B D z."""
        z = self.rng.standard_normal((self.G, self.lam, self.n))
        y = np.einsum("gij,gkj->gki", self.B, z * self.D[:, None, :])
        x = self.m[:, None, :] + self.sigma[:, None, None] * y
        return x, y

    def tell(self, y, fit):
        """Update with the steps y [G][lam][n] and fitness [G][lam] (larger is better)."""
        f = np.where(np.isnan(fit), -np.inf, fit)
        order = np.argsort(-f, axis=1, kind="stable")[:, :self.mu]
        ysel = np.take_along_axis(y, order[:, :, None], axis=1)           # [G][mu][n]
        yw = np.einsum("k,gkn->gn", self.w, ysel)
        self.m = self.m + self.sigma[:, None] * yw
        # C^{-1/2} yw = B D^{-1} B^T yw
        cinv = np.einsum("gij,gj,gkj,gk->gi", self.B, 1.0 / self.D, self.B, yw)
        self.ps = (1 - self.cs) * self.ps + np.sqrt(self.cs * (2 - self.cs) * self.mueff) * cinv
        nps = np.linalg.norm(self.ps, axis=1)
        self.gen += 1
        hs = (nps / np.sqrt(1 - (1 - self.cs) ** (2 * self.gen)) < (1.4 + 2 / (self.n + 1)) * self.chi)
        hs = hs.astype(np.float64)
        self.pc = (1 - self.cc) * self.pc + (hs * np.sqrt(self.cc * (2 - self.cc) * self.mueff))[:, None] * yw
        rank1 = np.einsum("gi,gj->gij", self.pc, self.pc)
        rankmu = np.einsum("k,gki,gkj->gij", self.w, ysel, ysel)
        decay = 1 - self.c1 - self.cmu + ((1 - hs) * self.c1 * self.cc * (2 - self.cc))
        self.C = decay[:, None, None] * self.C + self.c1 * rank1 + self.cmu * rankmu
        self.sigma = self.sigma * np.exp((self.cs / self.ds) * (nps / self.chi - 1))
        self.C = 0.5 * (self.C + np.transpose(self.C, (0, 2, 1)))
        evals, evecs = np.linalg.eigh(self.C)
        self.D = np.sqrt(np.maximum(evals, 1e-300))
        self.B = evecs


def minimize_like_check(fun, n, lam=16, iters=200, seed=0, x0=None, sigma=0.5):
    """One search maximising -fun(x) on R^n (a host check of the update)."""
    rng = np.random.default_rng(seed)
    st = CMAState(1, n, lam, np.zeros(n) if x0 is None else x0, sigma, rng)
    best = np.inf
    for _ in range(iters):
        x, y = st.ask()
        f = np.array([fun(v) for v in x[0]])
        best = min(best, f.min())
        st.tell(y, -f[None, :])
    return st.m[0], best
