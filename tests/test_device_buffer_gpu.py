"""Borrowed device buffers (bg_import_device_ptr + bg_group_use_buffer): a
group's state kept in a torch tensor the caller owns.  The run is the same
bit for bit as with engine-owned state; the tensor shows the state after each
run, and values written into it between runs are what the next run uses."""
import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms, mV
from brian_b200.connections import fixed_indegree_csr


def _net(N=5000):
    eqs = b.Equations("dv/dt=(ge+gi-(v-El))/taum : volt\ndge/dt=-ge/taue : volt\ndgi/dt=-gi/taui : volt",
                      taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    P = b.NeuronGroup(N, model=eqs, threshold=-50 * mV, reset=-60 * mV)
    ne = int(0.8 * N)
    rng = np.random.Generator(np.random.PCG64(6))
    objs = [P]
    for src, n, k, w, var, sd in ((P.subgroup(ne), ne, 80, 0.162e-2, "ge", 1), (P.subgroup(N - ne), N - ne, 20,
                                                                               -0.9e-2, "gi", 2)):
        rowptr, cols = fixed_indegree_csr(n, N, k, seed=sd)
        C = b.DelayConnection(src, P, var, max_delay=5 * ms)
        C.connect_csr(rowptr, cols, w, delay_steps=rng.integers(1, 51, size=len(cols)).astype(np.uint8))
        objs.append(C)
    P.v = -60 * mV + rng.random(N) * 10 * mV
    objs.append(b.StateMonitor(P, "v", record=[0, 1]))
    return b.Network(*objs), P


@pytest.mark.gpu
@pytest.mark.parametrize("persistent", [True, False])
def test_group_state_in_torch_tensor(gpu_table, persistent):
    prev = b.get_global_preference("persistent")
    b.set_global_preferences(persistent=persistent)
    try:
        _state_in_tensor(persistent)
    finally:
        b.set_global_preferences(persistent=prev)


def _state_in_tensor(persistent):
    import torch
    N = 5000
    b.clear()
    ref, Pr = _net(N)
    ref.run(400 * 0.1 * ms)
    b.clear()
    net, P = _net(N)
    buf = torch.zeros((3, P.padded_size()), dtype=torch.float64, device="cuda")
    P.use_device_buffer(buf)
    net.run(400 * 0.1 * ms)
    torch.cuda.synchronize()
    host = buf.cpu().numpy()
    for k, v in enumerate(("v", "ge", "gi")):
        assert np.array_equal(np.asarray(getattr(P, v)), np.asarray(getattr(Pr, v)))
        assert np.array_equal(host[k, :N], np.asarray(getattr(Pr, v)))
    assert net.stats()["persistent_threads"] == (512 if persistent else 0)
    # written between runs through the tensor, through the API on the other
    vnew = -60 * mV + np.random.default_rng(2).random(N) * 10 * mV
    buf[0, :N] = torch.from_numpy(vnew).cuda()
    torch.cuda.synchronize()
    Pr.v = vnew
    net.run(300 * 0.1 * ms)
    ref.run(300 * 0.1 * ms)
    torch.cuda.synchronize()
    for k, v in enumerate(("v", "ge", "gi")):
        assert np.array_equal(buf[k, :N].cpu().numpy(), np.asarray(getattr(Pr, v)))
    net._invalidate()
    ref._invalidate()


@pytest.mark.gpu
def test_device_buffer_checked(gpu_table):
    import torch
    from brian_b200._lib import EngineError
    b.clear()
    net, P = _net(3000)
    P.use_device_buffer(torch.zeros((3, 512), dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        net.run(10 * 0.1 * ms)
    b.clear()
    net, P = _net(3000)
    P.use_device_buffer(torch.zeros((3, P.padded_size()), dtype=torch.float32, device="cuda"))
    with pytest.raises(ValueError):
        net.run(10 * 0.1 * ms)
