"""GPU checks of the tensor-core (tcgen05) network kernels: the BF16 GEMM
against a PyTorch FP32 product of the same BF16 values, the forward pass and
every gradient against the FP64 oracle (oracle/mlp.py), training progress,
and the spike-train features against their numpy restatement."""
import numpy as np
import pytest

from brian_b200 import _lib
from oracle import mlp as om

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 200, 128), (4096, 512, 512), (64, 512, 4096),
                                   (512, 64, 4096), (1000, 16, 192)])
def test_gemm_matches_torch_fp32(M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda", dtype=torch.float32)
    t = _lib.product_table()
    t.check(t.gemm_bf16(M, N, K, A.data_ptr(), B.data_ptr(), C.data_ptr(), None), "gemm_bf16")
    ref = A.float() @ B.float().T
    # products of bf16 values are exact in fp32: only the summation order differs
    assert torch.allclose(C, ref, rtol=1e-5, atol=1e-5 * K)


def _net(seed=0):
    rng = np.random.default_rng(seed)
    P = om.init_params(rng)
    for l in range(4):
        P[l] = (P[l][0], (0.1 * rng.standard_normal(om.ROWS[l])).astype(np.float32))
    P[3][1][10:] = 0
    h = _lib.MLPHandle(5)
    for l in range(4):
        h.set_params(l, *P[l])
    return h, P, rng


def test_forward_matches_oracle():
    h, P, rng = _net(1)
    X = rng.standard_normal((300, 64)).astype(np.float32)
    out = h.forward(X)
    _, ref = om.forward(P, X)
    ref = ref[:, :10]
    err = np.abs(out - ref)
    assert np.max(err) < 2e-2 * max(1.0, np.max(np.abs(ref)))
    assert np.median(err) < 2e-3 * max(1.0, np.max(np.abs(ref)))


def test_gradients_match_oracle():
    h, P, rng = _net(2)
    n = 1024
    X = rng.standard_normal((n, 64)).astype(np.float32)
    Y = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
    h.set_data(X, Y)
    loss, dW, db = h.gradients(n)
    rloss, rdW, rdb, _ = om.gradients(P, X, Y, 5)
    assert abs(loss - rloss) <= 1e-3 * abs(rloss)
    for l in range(4):
        eW = np.linalg.norm(dW[l] - rdW[l]) / max(np.linalg.norm(rdW[l]), 1e-30)
        eb = np.linalg.norm(db[l] - rdb[l]) / max(np.linalg.norm(rdb[l]), 1e-30)
        assert eW < 2e-2, (l, eW)
        assert eb < 2e-2, (l, eb)
    # the padded output rows carry no gradient
    assert np.all(dW[3][10:] == 0) and np.all(db[3][10:] == 0)


def test_training_reduces_nll():
    h, P, rng = _net(3)
    n = 32768
    X = rng.standard_normal((n, 64)).astype(np.float32)
    A = rng.standard_normal((64, 5)) / 8
    Y = np.tanh(X @ A).astype(np.float32) + 0.05 * rng.standard_normal((n, 5)).astype(np.float32)
    h.set_data(X, Y)
    loss, ms = h.train(8, 2048, 1e-3, 11)
    assert np.all(np.isfinite(loss))
    assert loss[-1] < loss[0] - 1.0
    assert ms > 0
    # the trained network predicts the targets of training rows
    out = h.forward(X[:2048])
    assert np.mean((out[:, :5] - Y[:2048]) ** 2) < 0.25 * np.mean(Y[:2048] ** 2)


def test_features_match_oracle():
    from brian_b200.codegen import generate_model_code
    from brian_b200.synthetic import adaptive_lif_equations, THRESHOLD, RESET, PARAMS, sample_prior, ou_current
    rng = np.random.default_rng(4)
    ns, L, dt = 64, 8000, 1e-4
    P = sample_prior(ns, rng)
    S0 = np.zeros((7, ns))
    S0[2:7] = P
    S0[1] = P[2]
    I = np.concatenate([ou_current(L, dt, rng) for _ in range(ns)])
    code = generate_model_code(adaptive_lif_equations(), THRESHOLD, RESET, dt, scalar="double")
    h = _lib.FitHandle(code, dt, 40)
    h.set_input(I)
    h.set_targets(np.array([-10000, L + 10000] * ns))
    h.set_record(512)
    h.set_sims(S0, np.arange(ns) * L, np.full(ns, L), np.arange(ns) * 2, np.arange(ns) * 2 + 2)
    h.run(0, L)
    F = h.features()
    cnt, steps = h.read_spikes()
    assert cnt.sum() > 200
    for i in range(ns):
        ref = om.features(steps[i, :cnt[i]], I[i * L:(i + 1) * L], dt)
        assert np.allclose(F[i], ref, rtol=1e-5, atol=1e-6), i


def test_learned_proposals_beat_plain_swarm():
    """What the trained network gains: on fresh targets, the swarm seeded by
    the network's proposals reaches gamma >= 0.9 for more targets sooner
    than the swarm started from uniform draws (same kernel, same budget)."""
    from brian_b200.synthetic import (FitWorkload, adaptive_lif_equations, THRESHOLD, RESET, PARAMS, PRIOR,
                                      ADAPTIVE_LIF_BASIS, ou_current)
    from brian_b200.proposal import ProposalNetwork, simulate_training_set, race
    rng = np.random.default_rng(0)
    dt = 1e-4
    eqs = adaptive_lif_equations()
    prior = {k: PRIOR[k] for k in PARAMS}
    pool = [ou_current(50000, dt, rng) for _ in range(64)]
    X, th, _ = simulate_training_set(eqs, THRESHOLD, RESET, prior, pool, dt, 1 << 18, seed=1,
                                     duration_range=(1.0, 5.0))
    net = ProposalNetwork(prior, seed=2, basis=ADAPTIVE_LIF_BASIS)
    loss, _ = net.train(X, th, epochs=10, batch=4096, lr=1e-3, seed=3)
    assert loss[-1] < loss[0]
    w = FitWorkload(ntargets=16, dur_min=1.0, dur_max=5.0, seed=77)
    w.build_targets()
    box = {k: (PRIOR[k][0] / 2, PRIOR[k][1] * 2) for k in PARAMS}
    res = race(eqs, THRESHOLD, RESET, w.targets, w.inputs, dt, box, net=net, popsize=512, n_prop=64, max_iter=10,
               goal=0.9, seed=5)
    p, l = res["plain"], res["learned"]
    assert l["first_evaluation_reached"] > p["first_evaluation_reached"]
    assert l["t50_ms"] < p["t50_ms"]
    assert l["reached"] >= p["reached"]


def test_step_gradients_match_gradients():
    """The flat gradient of one training step (the data-parallel path: the
    weight partials and the bias gradients summed on the device) over a set
    that is exactly one batch equals the gradients of the same rows taken in
    another order, segment by segment (W0, b0, W1, b1, ...)."""
    import torch
    h, P, rng = _net(3)
    n = 4096
    X = rng.standard_normal((n, 64)).astype(np.float32)
    Y = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
    h.set_data(X, Y)
    loss, dW, db = h.gradients(n)
    h.epoch_order(5, 0)
    loss2, g = h.step_gradients(n, 0)
    flat = g.torch().cpu().numpy()
    assert abs(loss - loss2) <= 1e-4 * abs(loss)
    o = 0
    for l in range(4):
        for want in (dW[l].ravel(), db[l]):
            got = flat[o:o + want.size]
            o += want.size
            err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30)
            assert err < 1e-3, (l, want.size, err)
    assert o == flat.size
    h.close()
