"""distributed_modelfitting across two gloo ranks on the CPU.  Each rank fits
its own block of targets with a real fit -- the particle swarm of
particle_swarm.py:6-111 over the adaptive-threshold LIF's membrane time
constant, every candidate simulated by the fitting oracle and scored by the
gamma factor -- and every rank ends with all results in target order, equal
to fitting every target in one process."""
import importlib
import os
import socket
import sys
import tempfile

import numpy as np
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
DT, L, G = 1e-4, 3000, 5
TAUS = [6e-3, 9e-3, 12e-3, 15e-3, 18e-3]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    """Targets: the adaptive LIF with known tau on OU inputs (oracle
    simulation); returns (data pairs, inputs)."""
    sys.path.insert(0, os.path.dirname(HERE))
    from brian_b200.synthetic import adaptive_lif_equations, THRESHOLD, RESET, ou_current
    from oracle import fitting as of
    rng = np.random.default_rng(4)
    m = of.ModelOracle(adaptive_lif_equations(), THRESHOLD, RESET, DT, np.float64)
    data, inputs = [], []
    for j, tau in enumerate(TAUS):
        I = ou_current(L, DT, rng)
        S0 = np.zeros((7, 1))
        S0[2:7, 0] = [3.5e7, tau, 2e-2, 5e-3, 1e-1]
        S0[1] = S0[4]
        r = of.simulate(m, S0, I, [0], [L], np.array([-10000, 10 ** 7]), [0], [2], record=True)
        for st in r["rec"][0]:
            data.append((j, st * DT))
        inputs.append(I)
    return np.array(data), inputs


def oracle_fit(data=None, input=None, popsize=24, maxiter=6, **kw):
    """Fit tau of every target (the other parameters at their true values)
    with the oracle's particle swarm; the swarm's seed comes from the
    target's own spikes, so a target's result does not depend on which rank
    fits it."""
    from brian_b200.synthetic import adaptive_lif_equations, THRESHOLD, RESET
    from oracle import fitting as of
    mf = importlib.import_module("brian_b200.modelfitting")
    m = of.ModelOracle(adaptive_lif_equations(), THRESHOLD, RESET, DT, np.float64)
    pos, fit = [], []
    for t, I in zip(mf._split_data(data), input):
        steps = np.rint(np.asarray(t) / DT).astype(np.int64)
        tr = np.concatenate([[-10000], steps, [10 ** 7]])
        rate = (len(t) - 1) / (t[-1] - t[0])

        def fitness(X):
            P = X.shape[1]
            S0 = np.zeros((7, P))
            S0[2], S0[3], S0[4], S0[5], S0[6] = 3.5e7, X[0], 2e-2, 5e-3, 1e-1
            S0[1] = S0[4]
            r = of.simulate(m, S0, I, np.zeros(P, int), np.full(P, L), tr, np.zeros(P, int), np.full(P, len(tr)))
            return of.gamma(r["coinc"], r["nspikes"], len(t), rate, 40 * DT)

        seed = int(steps.sum()) % (1 << 31)
        X0 = 4e-3 + 16e-3 * of.philox_uniform(seed, 10 ** 6, np.arange(popsize)).reshape(1, -1)
        Xg, gfit, _ = of.pso_reference(X0, fitness, maxiter, (0.9, 1.9, 1.9), [4e-3], [2e-2], popsize, seed)
        pos.append({"tau": float(Xg[0, 0])})
        fit.append(float(gfit[0]))
    if len(pos) == 1:
        return mf.OptimizationResult(pos[0], fit[0], {"targets": 1})
    return mf.OptimizationResult(pos, fit, {"targets": len(pos)})


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, os.path.dirname(HERE))
    sys.path.insert(0, HERE)
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    mf = importlib.import_module("brian_b200.modelfitting")
    calls = []

    def fit(data=None, input=None, **kw):
        calls.append((len(mf._split_data(data)), kw.get("device"), kw.get("popsize")))
        return oracle_fit(data=data, input=input, popsize=kw["popsize"], maxiter=kw["maxiter"])

    mf.modelfitting = fit
    data, inputs = _problem()
    res = mf.distributed_modelfitting(data=data, input=inputs, popsize=24, maxiter=6)
    np.save(os.path.join(out_dir, "r%d.npy" % rank), np.array([[p["tau"], f] for p, f in zip(res.best_pos,
                                                                                          res.best_fit)]))
    np.save(os.path.join(out_dir, "c%d.npy" % rank), np.array(calls))
    dist.destroy_process_group()


def test_two_ranks_fit_and_gather_in_target_order():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d), nprocs=world, join=True, start_method="spawn")
        data, inputs = _problem()
        whole = oracle_fit(data=data, input=inputs, popsize=24, maxiter=6)
        want = np.array([[p["tau"], f] for p, f in zip(whole.best_pos, whole.best_fit)])
        for r in range(world):
            assert np.array_equal(np.load(os.path.join(d, "r%d.npy" % r)), want)
        c0, c1 = np.load(os.path.join(d, "c0.npy")), np.load(os.path.join(d, "c1.npy"))
        # rank 0: targets 0-1 on device 0; rank 1: targets 2-4 (device from LOCAL_RANK, 0 when unset)
        assert c0.tolist() == [[2, 0, 24]] and c1.tolist() == [[3, 0, 24]]
    # the fits find the hidden time constants
    taus = want[:, 0]
    assert np.all(np.abs(taus - np.array(TAUS)) / np.array(TAUS) < 0.25), taus
    assert np.all(want[:, 1] > 0.5), want[:, 1]
