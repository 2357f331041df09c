"""The allocation-free entry point bg_delay_group_run_noalloc.

Callers that cannot allocate device memory -- code living inside another
framework's caching allocator, which owns the device memory, or a process
that reserved all device memory up front -- pass their own device buffers
and get the engine's result without any cudaMalloc: the scratch lives in a
fixed array compiled into the library.

This test checks it against the network entry points (bg_net_*, through the
public API) on two calls in a row: the second call starts from the first
call's output and must not see anything the first call left in the shared
scratch.  Results must agree bit for bit, as in every GPU parity test here.
"""
import ctypes as ct

import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms, mV
from brian_b200.connections import fixed_indegree_csr
from brian_b200.equations import linear_propagator

N = 20000
INDEG = 100
TAUS = dict(taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)


def _connectivity():
    ne = int(0.8 * N)
    rng = np.random.Generator(np.random.PCG64(11))
    exc = fixed_indegree_csr(ne, N, 80, seed=21)
    inh = fixed_indegree_csr(N - ne, N, 20, seed=22)
    d_exc = rng.integers(1, 51, size=len(exc[1])).astype(np.uint8)
    d_inh = rng.integers(1, 51, size=len(inh[1])).astype(np.uint8)
    S0 = np.stack([-60 * mV + rng.random(N) * 10 * mV, np.zeros(N), np.zeros(N)])
    return ne, exc, inh, d_exc, d_inh, S0


def _engine_run(S_init, nsteps, conn):
    """Reference result: the network entry points via the public API."""
    ne, exc, inh, d_exc, d_inh, _ = conn
    b.clear()
    b.reinit_default_clock()
    eqs = b.Equations("dv/dt=(ge+gi-(v-El))/taum : volt\ndge/dt=-ge/taue : volt\ndgi/dt=-gi/taui : volt", **TAUS)
    P = b.NeuronGroup(N, model=eqs, threshold=-50 * mV, reset=-60 * mV)
    Ce = b.DelayConnection(P.subgroup(ne), P, "ge", max_delay=5 * ms)
    Ce.connect_csr(exc[0], exc[1], 0.162e-2, delay_steps=d_exc)
    Ci = b.DelayConnection(P.subgroup(N - ne), P, "gi", max_delay=5 * ms)
    Ci.connect_csr(inh[0], inh[1], -0.9e-2, delay_steps=d_inh)
    P.v, P.ge, P.gi = S_init[0], S_init[1], S_init[2]
    net = b.Network(P, Ce, Ci)
    net.run(nsteps * 0.1 * ms)
    spikes = int(net._binding.rt.counters(1, 2)[0][0])
    out = np.stack([np.array(P.v), np.array(P.ge), np.array(P.gi)])
    A, C = linear_propagator(eqs, 0.1 * ms)
    net._invalidate()
    return out, spikes, A, C


def _noalloc_run(lib, dev, S_init, nsteps, A, C, expect=0):
    import torch
    S = torch.from_numpy(np.ascontiguousarray(S_init)).to("cuda")
    torch.cuda.synchronize()
    A = np.ascontiguousarray(A, dtype=np.float64)
    C = np.ascontiguousarray(C, dtype=np.float64)
    i64 = lambda xs: (ct.c_int64 * len(xs))(*xs)
    ptrs = lambda ts: (ct.c_void_p * len(ts))(*[t.data_ptr() for t in ts])
    spikes = ct.c_int64(0)
    st = lib.bg_delay_group_run_noalloc(
        N, 3, ct.c_void_p(S.data_ptr()), A.ctypes.data_as(ct.c_void_p), C.ctypes.data_as(ct.c_void_p),
        0, -50 * mV, 0, -60 * mV, 2, i64([0, dev["ne"]]), i64([dev["ne"], N - dev["ne"]]), (ct.c_int * 2)(1, 2),
        ptrs(dev["rowptr"]), ptrs(dev["cols"]), ptrs(dev["delays"]), (ct.c_double * 2)(0.162e-2, -0.9e-2),
        (ct.c_int32 * 2)(51, 51), nsteps, None, ct.byref(spikes))
    if st != expect:
        buf = ct.create_string_buffer(512)
        lib.bg_last_error(buf, 512)
        raise AssertionError("bg_delay_group_run_noalloc returned %d: %s" % (st, buf.value.decode()))
    return S.cpu().numpy(), spikes.value


def _bind(lib):
    lib.bg_delay_group_run_noalloc.restype = ct.c_int
    lib.bg_delay_group_run_noalloc.argtypes = [
        ct.c_int64, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_double, ct.c_int, ct.c_double,
        ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
        ct.c_void_p, ct.c_int64, ct.c_void_p, ct.POINTER(ct.c_int64)]


@pytest.mark.gpu
def test_noalloc_matches_network_engine_twice(gpu_table):
    import torch
    lib = gpu_table.lib
    _bind(lib)
    conn = _connectivity()
    ne, exc, inh, d_exc, d_inh, S0 = conn
    dev = {"ne": ne,
           "rowptr": [torch.from_numpy(exc[0]).cuda(), torch.from_numpy(inh[0]).cuda()],
           "cols": [torch.from_numpy(exc[1]).cuda(), torch.from_numpy(inh[1]).cuda()],
           "delays": [torch.from_numpy(d_exc).cuda(), torch.from_numpy(d_inh).cuda()]}
    # call 1: from S0
    ref1, spk_ref1, A, C = _engine_run(S0, 600, conn)
    out1, spk1 = _noalloc_run(lib, dev, S0, 600, A, C)
    assert spk_ref1 > 100
    assert spk1 == spk_ref1
    assert np.array_equal(out1, ref1)
    # call 2: continue from call 1's output, fresh rings; the scratch still
    # holds call 1's rings and history and must be cleared by the call
    ref2, spk_ref2, _, _ = _engine_run(out1, 350, conn)
    out2, spk2 = _noalloc_run(lib, dev, out1, 350, A, C)
    assert spk2 == spk_ref2
    assert np.array_equal(out2, ref2)


@pytest.mark.gpu
def test_noalloc_refuses_malformed_rows(gpu_table):
    """A decreasing or negative rowptr, a target beyond the group or a delay
    at the ring depth is refused with BG_EINVAL by the device checks that
    run before the step loop; the state is untouched."""
    import torch
    lib = gpu_table.lib
    _bind(lib)
    ne, exc, inh, d_exc, d_inh, S0 = _connectivity()
    A = np.eye(3)
    for bad in ("decreasing", "negative", "target", "delay"):
        rp, cl, dl = exc[0].copy(), exc[1].copy(), d_exc.copy()
        if bad == "decreasing":
            rp[5], rp[6] = rp[6], rp[5]
        elif bad == "negative":
            rp[0] = -1
        elif bad == "target":
            cl[1000] = N                    # one target beyond the group
        else:
            dl[1000] = 51                   # ring depth 51: delays 0..50
        dev = {"ne": ne,
               "rowptr": [torch.from_numpy(rp).cuda(), torch.from_numpy(inh[0]).cuda()],
               "cols": [torch.from_numpy(cl).cuda(), torch.from_numpy(inh[1]).cuda()],
               "delays": [torch.from_numpy(dl).cuda(), torch.from_numpy(d_inh).cuda()]}
        out, _ = _noalloc_run(lib, dev, S0, 10, A, np.zeros(3), expect=-1)
        assert np.array_equal(out, S0)
