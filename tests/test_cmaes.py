"""CMA-ES of modelfitting (brian_b200/cmaes.py): the update, restated from
Hansen's tutorial, solves the standard test functions on the host."""
import numpy as np

from brian_b200.cmaes import CMAState, minimize_like_check


def test_sphere_and_rosenbrock():
    _, best = minimize_like_check(lambda x: float(np.sum(x ** 2)), 5, lam=16, iters=150, seed=1,
                                  x0=np.full(5, 0.8))
    assert best < 1e-15
    rosen = lambda x: float(np.sum(100 * (x[1:] - x[:-1] ** 2) ** 2 + (1 - x[:-1]) ** 2))
    m, best = minimize_like_check(rosen, 4, lam=16, iters=500, seed=2, x0=np.zeros(4))
    assert best < 1e-12 and np.allclose(m, 1.0, atol=1e-5)


def test_groups_are_independent():
    """Vectorised over groups: each group's search equals a search run alone."""
    rng_all = np.random.default_rng(3)
    st = CMAState(3, 2, 8, np.zeros((3, 2)), 0.5, rng_all)
    targets = np.array([[0.5, -0.2], [-0.7, 0.1], [0.0, 0.9]])
    for _ in range(60):
        x, y = st.ask()
        f = -np.sum((x - targets[:, None, :]) ** 2, axis=2)
        st.tell(y, f)
    assert np.allclose(st.m, targets, atol=1e-4)
    # a NaN fitness never becomes a parent
    x, y = st.ask()
    f = np.full((3, 8), -1.0)
    f[:, 0] = np.nan
    m_before = st.m.copy()
    st.tell(y, f)
    assert np.all(np.isfinite(st.m)) and not np.allclose(st.m, m_before + st.sigma[:, None] * y[:, 0, :])
