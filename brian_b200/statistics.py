"""Spike-train statistics (tools/statistics.py of Brian 1.4.4), FP64 on the host.

firing_rate (statistics.py:15-21), CV (23-30), spike_triggered_average
(125-153), get_gamma_factor (236-240) and gamma_factor (261-314).
"""
import numpy as np

__all__ = ["firing_rate", "CV", "gamma_factor", "get_gamma_factor", "spike_triggered_average"]


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
