"""precision_agreement: the FP32-vs-FP64 report over two spike records."""
import numpy as np

from brian_b200.statistics import precision_agreement, spike_trains


def _record(rng, n, steps, rate_steps):
    s, i = np.nonzero(rng.random((steps, n)) < 1.0 / rate_steps)
    return s.astype(np.int64), i.astype(np.int32)


def test_identical_records_agree_fully():
    rng = np.random.default_rng(1)
    rec = _record(rng, 50, 20000, 500)
    v = rng.standard_normal((20000, 3))
    r = precision_agreement(rec, rec, 50, 2.0, v, v)
    assert abs(r["gamma_mean"] - 1) < 1e-12 and abs(r["gamma_min"] - 1) < 1e-12 and r["spike_match_frac"] == 1.0
    assert r["rate_rel_err"] == 0.0 and r["v_rms_err_mV"] == 0.0 and r["first_differing_step"] is None
    assert all(abs(g - 1) < 1e-12 for g in r["gamma_mean_by_window_ms"].values() if g is not None)


def test_shifted_and_independent_records():
    rng = np.random.default_rng(2)
    rec = _record(rng, 40, 20000, 400)
    # every spike one step later: within delta, so gamma stays high; a spike
    # repeats exactly only where a neuron fired on two consecutive steps;
    # the first difference is the first spike
    shifted = (rec[0] + 1, rec[1])
    r = precision_agreement(rec, shifted, 40, 2.0)
    assert r["gamma_mean"] > 0.9 and r["spike_match_frac"] < 0.01
    assert r["first_differing_step"] == int(rec[0].min())
    # an independent record of the same rate: gamma near chance
    other = _record(np.random.default_rng(3), 40, 20000, 400)
    r = precision_agreement(rec, other, 40, 2.0)
    assert abs(r["gamma_mean"]) < 0.2 and r["rate_rel_err"] < 0.1


def test_spike_trains_split():
    tr = spike_trains(np.array([5, 1, 3, 3]), np.array([2, 0, 2, 1]), 4, 0.5)
    assert [list(t) for t in tr] == [[0.5], [1.5], [2.5, 1.5], []]
