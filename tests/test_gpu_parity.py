"""CUDA engine vs the CPU oracle on identical seeded networks.

FP64: spikes (step, index) identical and every state variable, trace and
weight equal bit for bit (+0 == -0), which is stronger than the 1e-12
relative bound the FP64 path promises."""
import numpy as np
import pytest

import scenarios
import brian_b200 as b
from brian_b200.network import engine


def _both(fn, oracle_table, **kw):
    out = []
    for tab in (oracle_table, None):
        b.clear()
        b.reinit_default_clock()
        np.random.seed(1234)
        if tab is None:
            out.append(fn(**kw))
        else:
            with engine(tab):
                out.append(fn(**kw))
    return out


def _pop_threads(*outs):
    return [o.pop("persistent_threads") for o in outs]


@pytest.mark.gpu
def test_cuba4000_bit_exact(oracle_table, gpu_table):
    """Zero-delay Connections, a SpikeMonitor and a StateMonitor of v: the
    persistent kernel (4 blocks of 1024 neurons)."""
    ref, gpu = _both(scenarios.cuba, oracle_table, steps=10000)
    assert _pop_threads(ref, gpu)[1] == 512
    assert len(ref["spk0.idx"]) > 10000
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("persistent", [True, False])
def test_cuba4000_split_runs_statemonitor_period(oracle_table, gpu_table, persistent):
    """Three run() calls, recorded neurons in several blocks and out of
    order, every third step: the persistent and the stepped path."""
    ref, gpu = _both(scenarios.cuba, oracle_table, steps=2400, runs=3, timestep=3,
                     record=[3999, 0, 1500, 1024, 2047, 7], persistent=persistent)
    assert _pop_threads(ref, gpu)[1] == (512 if persistent else 0)
    assert len(ref["st0.steps"]) == 800
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
def test_cuba4000_refractory_bit_exact(oracle_table, gpu_table):
    ref, gpu = _both(scenarios.cuba, oracle_table, steps=3000, refractory=5 * b.ms)
    assert _pop_threads(ref, gpu)[1] == 0            # refractoriness: the stepped path
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("wdtype", [np.float32, np.float64])
def test_delay_ring_bit_exact(oracle_table, gpu_table, wdtype):
    ref, gpu = _both(scenarios.cuba_delay, oracle_table, wdtype=wdtype)
    assert len(ref["spk0.idx"]) > 500
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("dmin,runs", [(1, 1), (1, 3), (0, 2)])
def test_persistent_path_bit_exact(oracle_table, gpu_table, dmin, runs):
    """No monitors: single group with shared-weight DelayConnections runs in
    the persistent cooperative kernel (lag-2 wait; lag-1 when a delay is 0)."""
    ref, gpu = _both(scenarios.cuba_delay, oracle_table, monitors=False, dmin=dmin, runs=runs, N=6000,
                     steps=3000)
    assert ref["spikes"][0] > 1000
    ref.pop("launches"), ref.pop("persistent_threads")
    launches, th = gpu.pop("launches"), gpu.pop("persistent_threads")
    scenarios.compare(ref, gpu)
    assert th == 512                        # 6 blocks of 1024 neurons
    import brian_b200 as bb
    assert bb.network._magic_cache is not None
    assert launches == runs                 # one cooperative launch per run


@pytest.mark.gpu
@pytest.mark.parametrize("burst", [False, True])
def test_persistent_spike_monitors_bit_exact(oracle_table, gpu_table, burst):
    """Spike monitors (the whole group, and the inhibitory subgroup whose
    range starts and ends inside a 32-neuron word at N=6010) on
    the persistent path: the kernel's per-step spike words become the same
    (step, index) records as the reference's SpikeMonitor, across launches
    of at most 1024 steps and across runs."""
    ref, gpu = _both(scenarios.cuba_delay, oracle_table, monitors="spikes", N=6010, steps=3000, runs=2,
                     burst=burst)
    assert len(ref["spk0.idx"]) > 1000 and len(ref["spk1.idx"]) > 100
    ref.pop("launches"), ref.pop("persistent_threads")
    launches, th = gpu.pop("launches"), gpu.pop("persistent_threads")
    scenarios.compare(ref, gpu)
    # per run: two launches of <= 1024 steps, each followed by 3 monitor kernels per monitor
    assert th == 512 and launches == 2 * 2 * (1 + 3 * 2)


@pytest.mark.gpu
def test_persistent_burst_bit_exact(oracle_table, gpu_table):
    """Synchronous firing: blocks push hundreds of spikes in one step, in
    several batches of the persistent kernel's push."""
    ref, gpu = _both(scenarios.cuba_delay, oracle_table, monitors=False, N=6000, steps=1500, burst=True)
    assert ref["spikes"][0] > 10000       # all 6000 fire at step 0, then a second wave
    ref.pop("launches"), ref.pop("persistent_threads")
    launches, th = gpu.pop("launches"), gpu.pop("persistent_threads")
    scenarios.compare(ref, gpu)
    assert launches == 1 and th == 512


@pytest.mark.gpu
def test_persistent_general_matrix_bit_exact(oracle_table, gpu_table):
    """A linear update outside the specialised pattern (gi driven by ge)
    takes the persistent kernel's general update."""
    ref, gpu = _both(scenarios.cuba_delay, oracle_table, monitors=False, N=6000, steps=2000, coupled=True)
    assert ref["spikes"][0] > 1000
    ref.pop("launches"), ref.pop("persistent_threads")
    launches, th = gpu.pop("launches"), gpu.pop("persistent_threads")
    scenarios.compare(ref, gpu)
    assert launches == 1 and th == 512


@pytest.mark.gpu
@pytest.mark.parametrize("threads", [256, 512])
def test_persistent_block_sizes_bit_exact(oracle_table, gpu_table, threads):
    """Both shapes of the persistent kernel (ragged last block at N=7000)
    give the oracle's results bit for bit."""
    ref, gpu = _both(scenarios.cuba_delay, oracle_table, monitors=False, N=7000, steps=2000, runs=2,
                     persistent=threads)
    assert ref["spikes"][0] > 1000
    ref.pop("launches"), ref.pop("persistent_threads")
    launches, th = gpu.pop("launches"), gpu.pop("persistent_threads")
    scenarios.compare(ref, gpu)
    assert launches == 2 and th == threads


@pytest.mark.gpu
def test_delay_ring_general_weights_ordered(oracle_table, gpu_table):
    ref, gpu = _both(scenarios.cuba_delay, oracle_table, hetero_weights=True, steps=1000)
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("dense", [True, False])
def test_stdp_bit_exact(oracle_table, gpu_table, dense):
    ref, gpu = _both(scenarios.stdp, oracle_table, dense=dense)
    assert len(ref["spk0.idx"]) > 0
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("wdtype,interactions,runs", [(np.float64, "all", 1), (np.float32, "all", 1),
                                                      (np.float64, "nearest", 2), (np.float64, "nearest_pre", 1)])
def test_stdp_delay_bit_exact(oracle_table, gpu_table, wdtype, interactions, runs):
    """ExponentialSTDP on a DelayConnection: weights, traces and spikes."""
    ref, gpu = _both(scenarios.stdp_delay, oracle_table, wdtype=wdtype, interactions=interactions, runs=runs)
    assert len(ref["spk0.idx"]) > 20
    assert not np.array_equal(ref["w0"], ref["w_init"])
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("dense,update", [(True, "multiplicative"), (False, "multiplicative"), (True, "mixed"),
                                          (False, "mixed")])
def test_stdp_update_forms_bit_exact(oracle_table, gpu_table, dense, update):
    """ExponentialSTDP update='multiplicative' / 'mixed' (FP64 weights)."""
    ref, gpu = _both(scenarios.stdp, oracle_table, dense=dense, wdtype=np.float64, update=update)
    assert len(ref["spk0.idx"]) > 0
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("update", ["multiplicative", "mixed"])
def test_stdp_delay_update_forms_bit_exact(oracle_table, gpu_table, update):
    ref, gpu = _both(scenarios.stdp_delay, oracle_table, update=update)
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
def test_stdp_delay_large_bit_exact(oracle_table, gpu_table):
    """More sources than one block's words, several spikes per step."""
    ref, gpu = _both(scenarios.stdp_delay, oracle_table, Nin=5000, Nout=300, p=0.1, steps=1500)
    assert len(ref["spk0.idx"]) > 100
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
def test_cuba_large_persistent_bit_exact(oracle_table, gpu_table):
    """The benchmark's construction at 200 000 neurons and in-degree 1000
    (200 M synapses; 196 persistent blocks of 1024 neurons, more than one
    per SM, so the cross-block waits run over the whole grid): spikes and
    final states of the persistent path equal the oracle's over 400 steps,
    split into two runs."""
    ref, gpu = _both(scenarios.cuba_large, oracle_table, N=200000, steps=400, runs=2)
    assert ref["spikes"][0] > 5000 and ref["events"].sum() > 5_000_000
    ref.pop("launches"), ref.pop("persistent_threads")
    launches, th = gpu.pop("launches"), gpu.pop("persistent_threads")
    assert th > 0                           # the persistent kernel ran
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
def test_kitchen_sink_bit_exact(oracle_table, gpu_table):
    ref, gpu = _both(scenarios.kitchen_sink, oracle_table)
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
def test_run_split_equals_single_run(gpu_table):
    """run(T1) + run(T2) == run(T1+T2): chunking, graph replay and the fused
    tail of the last step leave no trace in the results."""
    b.clear(); b.reinit_default_clock(); np.random.seed(1)
    one = scenarios.cuba(N=2000, steps=1234)
    b.clear(); b.reinit_default_clock(); np.random.seed(1)
    two = scenarios.cuba(N=2000, steps=1234, runs=2)
    assert one["spk0.idx"].size > 0
    scenarios.compare(one, two)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(method="RK"), dict(string_threshold=False, string_reset=False),
                                dict(delays=False), dict(empirical=True), dict(linear=True)],
                         ids=["euler-strings", "rk2", "euler-builtin-thr-reset", "no-delays", "empirical",
                              "linear-strings"])
def test_generated_model_bit_exact(oracle_table, gpu_table, kw):
    """Nonlinear (conductance-based) groups and string thresholds/resets:
    the group kernel compiled by NVRTC around the generated model gives the
    oracle's spikes and states bit for bit (polynomial model, FP64)."""
    ref, gpu = _both(scenarios.coba, oracle_table, **kw)
    assert len(ref["spk0.idx"]) > 1000
    scenarios.compare(ref, gpu)


@pytest.mark.gpu
def test_generated_exponential_euler_close(oracle_table, gpu_table):
    """Exponential Euler calls exp (CUDA's against the C library's): the
    first 300 steps agree in spikes and to 1e-12 in states."""
    ref, gpu = _both(scenarios.coba, oracle_table, implicit=True, steps=300)
    assert len(ref["spk0.idx"]) > 100
    for k in ("spk0.idx", "spk0.steps"):
        assert np.array_equal(ref[k], gpu[k])
    for k in ("g0.v", "g0.ge", "g0.gi"):
        assert np.allclose(ref[k], gpu[k], rtol=1e-12, atol=1e-15)


def _fp32_and_oracle(fn, oracle_table, **kw):
    """fn on the FP64 oracle and on the GPU engine at precision 32."""
    b.clear(); b.reinit_default_clock(); np.random.seed(1234)
    with engine(oracle_table):
        ref = fn(**kw)
    prev = b.get_global_preference("precision")
    b.set_global_preferences(precision=32)
    try:
        b.clear(); b.reinit_default_clock(); np.random.seed(1234)
        gpu = fn(**kw)
    finally:
        b.set_global_preferences(precision=prev)
    return ref, gpu


def _spike_total(r):
    return int(r["spikes"][0]) if "spikes" in r else len(r["spk0.idx"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cuba", "persistent", "generated", "stdp"])
def test_fp32_network_close_to_fp64_oracle(oracle_table, gpu_table, case):
    """The FP32 engine (state and ring values in float) against the FP64
    oracle: states after 20 steps agree to float precision, and over 2000
    steps the spike counts stay within 3 %."""
    fn, kw = {"cuba": (scenarios.cuba, dict(N=4000)),
              "persistent": (scenarios.cuba_delay, dict(monitors=False, N=6000)),
              "generated": (scenarios.coba, dict()),
              "stdp": (scenarios.stdp, dict(Nin=400, Nout=64))}[case]
    ref, gpu = _fp32_and_oracle(fn, oracle_table, steps=20, **kw)
    for k in ref:
        if k.startswith("g0.") or k == "w0":
            scale = max(1e-3, float(np.max(np.abs(ref[k]))))
            assert np.max(np.abs(np.asarray(gpu[k], dtype=np.float64) - ref[k])) <= 1e-4 * scale, k
    ref, gpu = _fp32_and_oracle(fn, oracle_table, steps=2000, **kw)
    n_ref, n_gpu = _spike_total(ref), _spike_total(gpu)
    assert n_ref > 500
    assert abs(n_gpu - n_ref) <= 0.03 * n_ref, (n_gpu, n_ref)
