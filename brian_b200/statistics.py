"""Spike-train statistics (tools/statistics.py of Brian 1.4.4), FP64 on the host.

firing_rate (statistics.py:15-21), CV (23-30), spike_triggered_average
(125-153), get_gamma_factor (236-240) and gamma_factor (261-314); and, with
no counterpart in the reference, spike_trains (a SpikeMonitor record split
per neuron) and precision_agreement (how closely a run with FP32 state
follows the FP64 run of the same network).
"""
import numpy as np

__all__ = ["firing_rate", "CV", "gamma_factor", "get_gamma_factor", "spike_triggered_average", "spike_trains",
           "precision_agreement"]


def firing_rate(spikes):
    """(n-1) / (t_last - t_first); NaN for fewer than two spikes."""
    spikes = np.asarray(spikes, dtype=float)
    if len(spikes) < 2:
        return np.nan
    return (len(spikes) - 1) / (spikes[-1] - spikes[0])


def CV(spikes):
    spikes = np.asarray(spikes, dtype=float)
    if len(spikes) == 0:
        return np.nan
    isi = np.diff(spikes)
    return np.std(isi) / np.mean(isi)


def get_gamma_factor(coincidence_count, model_length, target_length, target_rates, delta):
    """gamma = (Nc - 2 delta Nt r) / (0.5 (1 - 2 delta r) (Nt + Nm))."""
    NCoincAvg = 2 * delta * target_length * target_rates
    norm = .5 * (1 - 2 * delta * target_rates)
    return (coincidence_count - NCoincAvg) / (norm * (target_length + model_length))


def gamma_factor(source, target, delta, normalize=True, dt=None):
    """Offline coincidence count between two spike trains (statistics.py:261-314)."""
    source = np.asarray(source, dtype=float)
    target = np.asarray(target, dtype=float)
    target_rate = firing_rate(target)
    if dt is None:
        delta_diff = delta
    else:
        source = np.array(np.rint(source / dt), dtype=int)
        target = np.array(np.rint(target / dt), dtype=int)
        delta_diff = int(np.rint(delta / dt))
    ns, nt = len(source), len(target)
    if nt == 0 or ns == 0:
        return 0
    if ns > 1:
        bins = .5 * (source[1:] + source[:-1])
        indices = np.digitize(target, bins)
        diff = np.abs(target - source[indices])
        coincidences = int(np.sum(diff <= delta_diff))
    else:
        coincidences = int(sum(np.amin(np.abs(source - target[i])) <= delta_diff for i in range(nt)))
    gamma = get_gamma_factor(coincidences, ns, nt, target_rate, delta)
    return gamma if normalize else coincidences


def spike_triggered_average(spikes, stimulus, max_interval, dt, onset=None, display=False):
    """Average of the stimulus over `max_interval` before each spike after
    `onset`, most recent sample first (statistics.py:125-153)."""
    stimulus = np.asarray(stimulus).flatten()
    if onset is None or onset < max_interval:
        onset = max_interval
    nspikes = len(spikes)
    L = int(max_interval / dt)
    ens = np.zeros((nspikes, L))
    for k, s in enumerate(spikes):
        if s > onset:
            i = int(s / dt)
            ens[k, :] = stimulus[i - L:i]
    return np.sum(ens, axis=0)[::-1] / (nspikes - 1), np.linspace(0, max_interval, L)


def spike_trains(steps, idx, n, dt):
    """Per-neuron spike times (s) of a SpikeMonitor record."""
    steps = np.asarray(steps)
    idx = np.asarray(idx)
    order = np.argsort(idx, kind="stable")
    cuts = np.searchsorted(idx[order], np.arange(n + 1))
    t = steps[order] * dt
    return [t[cuts[i]:cuts[i + 1]] for i in range(n)]


def precision_agreement(rec64, rec32, n, duration, v64=None, v32=None, delta=4e-3, dt=1e-4):
    """Agreement of an FP32-state run with the FP64 run of the same network:
    gamma factor (delta 4 ms, tools/statistics.py:261-314) of each neuron's
    FP32 train against its FP64 train, over neurons with at least two FP64
    spikes and 2 delta r < 1 (gamma is undefined at higher rates); firing
    rates and their relative error; the fraction of FP64 spikes (step,
    index) the FP32 run repeats exactly; the RMS difference of the recorded
    v traces."""
    t64 = spike_trains(rec64[0], rec64[1], n, dt)
    t32 = spike_trains(rec32[0], rec32[1], n, dt)
    g, skipped = [], 0
    for a, b_ in zip(t32, t64):
        if len(b_) < 2:
            continue
        r = (len(b_) - 1) / (b_[-1] - b_[0]) if b_[-1] > b_[0] else np.inf
        if not 2 * delta * r < 1:
            skipped += 1
            continue
        g.append(float(gamma_factor(a, b_, delta, dt=dt)))
    # the windows [0, T) over which the FP32 run still tracks the FP64 one
    windows = {}
    for T in (0.01, 0.02, 0.05, 0.1, 0.2, 0.5, 1.0, 2.0, 5.0, 10.0):
        if T > duration + 1e-12:
            break
        gw = []
        for a, b_ in zip(t32, t64):
            b_ = b_[b_ < T]
            if len(b_) < 2 or b_[-1] <= b_[0]:
                continue
            r = (len(b_) - 1) / (b_[-1] - b_[0])
            if 2 * delta * r < 1:
                gw.append(float(gamma_factor(a[a < T], b_, delta, dt=dt)))
        windows["%g" % (T * 1e3)] = float(np.mean(gw)) if gw else None
    key64 = np.asarray(rec64[0], dtype=np.int64) * n + np.asarray(rec64[1], dtype=np.int64)
    key32 = np.asarray(rec32[0], dtype=np.int64) * n + np.asarray(rec32[1], dtype=np.int64)
    match = len(np.intersect1d(key64, key32)) / max(1, len(key64))
    r64 = len(key64) / (n * duration)
    r32 = len(key32) / (n * duration)
    out = {"neurons": n, "duration_s": duration, "delta_ms": delta * 1e3,
           "gamma_mean": float(np.mean(g)) if g else None, "gamma_median": float(np.median(g)) if g else None,
           "gamma_min": float(np.min(g)) if g else None,
           "gamma_frac_ge_0.95": float(np.mean(np.asarray(g) >= 0.95)) if g else None,
           "gamma_neurons": len(g), "gamma_skipped_rate": skipped,
           "rate_fp64_hz": r64, "rate_fp32_hz": r32, "rate_rel_err": abs(r32 - r64) / r64 if r64 > 0 else None,
           "spikes_fp64": int(len(key64)), "spikes_fp32": int(len(key32)), "spike_match_frac": float(match),
           "gamma_mean_by_window_ms": windows}
    diff = np.setxor1d(key64, key32)
    out["first_differing_step"] = int(diff.min() // n) if len(diff) else None
    if v64 is not None and v32 is not None:
        d = np.asarray(v32, dtype=np.float64) - np.asarray(v64, dtype=np.float64)
        out["v_rms_err_mV"] = float(np.sqrt(np.mean(d * d)) * 1e3)
    return out
