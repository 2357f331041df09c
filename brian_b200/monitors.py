"""Monitors (monitor.py of Brian 1.4.4).

SpikeMonitor records (index, time) pairs in the connections slot
(monitor.py:156-166); StateMonitor records a state variable after the resets
(when='end', monitor.py:824-842).  Records accumulate in device buffers and
are drained to host memory by the engine between chunks of steps.
SpikeCounter, PopulationSpikeCounter and PopulationRateMonitor are views of
a spike record.  CoincidenceCounter (monitor.py:1229-1376) is computed from
the recorded spikes with the reference's online algorithm.
"""
import numpy as np

from ._lib import EngineBound
from .clock import guess_clock

__all__ = ["SpikeMonitor", "StateMonitor", "SpikeCounter", "PopulationSpikeCounter",
           "PopulationRateMonitor", "CoincidenceCounter", "MultiStateMonitor", "RecentStateMonitor",
           "ISIHistogramMonitor"]


class SpikeMonitor(EngineBound):
    def __init__(self, source, record=True, delay=0, function=None):
        if function is not None:
            raise NotImplementedError("per-step Python callbacks are not supported on the engine")
        self.source = source
        self.record = record
        self.delay = int(float(delay) / source.clock.dt) if delay else 0
        self._binding = None
        self._mid = None
        self._steps = np.zeros(0, dtype=np.int64)
        self._idx = np.zeros(0, dtype=np.int32)
        self._archived = (np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int32))

    def _lower(self, rt, gids):
        return rt.spikemon_add(gids[self.source._owner], self.source._origin, len(self.source), self.delay)

    def _record(self):
        if self._binding is not None:
            s, i = self._binding.read_spikes(self)
            return (np.concatenate([self._archived[0], s]), np.concatenate([self._archived[1], i]))
        return self._archived

    def _archive(self):
        self._archived = self._record()

    def _host_state(self, d):
        d["_archived"] = self._record()

    def reinit(self):
        self._archived = (np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int32))
        if self._binding is not None:
            self._binding.clear_monitor(self)

    @property
    def nspikes(self):
        return len(self._record()[1])

    @property
    def it(self):
        s, i = self._record()
        return i.astype(int), s * self.source.clock.dt

    @property
    def spikes(self):
        i, t = self.it
        return list(zip(i.tolist(), t.tolist()))

    @property
    def spiketimes(self):
        i, t = self.it
        return {k: t[i == k] for k in range(len(self.source))}

    def __getitem__(self, k):
        i, t = self.it
        return t[i == k]

    getspiketimes = spiketimes


class SpikeCounter(SpikeMonitor):
    """Spike count per neuron (monitor.py:297-333)."""

    def __init__(self, source):
        SpikeMonitor.__init__(self, source)

    @property
    def count(self):
        return np.bincount(self._record()[1], minlength=len(self.source))

    def __getitem__(self, k):
        return self.count[k]


class PopulationSpikeCounter(SpikeMonitor):
    """Total spike count (monitor.py:267-294)."""

    def __init__(self, source, delay=0):
        SpikeMonitor.__init__(self, source, delay=delay)


class PopulationRateMonitor(SpikeMonitor):
    """Population rate in bins of `bin` seconds (monitor.py:590-680)."""

    def __init__(self, source, bin=None):
        SpikeMonitor.__init__(self, source)
        self.bin = bin

    def _rates(self):
        s, _ = self._record()
        dt = self.source.clock.dt
        binsteps = 1 if self.bin is None else max(1, int(round(self.bin / dt)))
        if len(s) == 0:
            return np.zeros(0), np.zeros(0)
        s0 = 0
        nb = int((s.max() - s0) // binsteps) + 1
        counts = np.bincount((s - s0) // binsteps, minlength=nb)
        times = (np.arange(nb) * binsteps + s0) * dt
        return times, counts / (len(self.source) * binsteps * dt)

    @property
    def times(self):
        return self._rates()[0]

    @property
    def rate(self):
        return self._rates()[1]

    def smooth_rate(self, width=1e-3, filter="gaussian"):
        times, rate = self._rates()
        dt = self.source.clock.dt * (1 if self.bin is None else max(1, int(round(self.bin / self.source.clock.dt))))
        w = width / dt
        if filter == "gaussian":
            k = np.exp(-np.arange(-int(3 * w), int(3 * w) + 1) ** 2 / (2 * w * w))
        else:
            k = np.ones(max(1, int(2 * w) + 1))
        k /= k.sum()
        return np.convolve(rate, k, mode="same")


class StateMonitor(EngineBound):
    """Records S[varname] at `record` (True, index, list) every `timestep`
    steps at the end of each step (monitor.py:683-989).  ``record=False``
    keeps the running mean and variance of every neuron."""

    def __init__(self, P, varname, clock=None, record=False, timestep=1, when="end"):
        if when not in ("end", "start"):
            raise NotImplementedError("StateMonitor when=%r is not supported (use 'end')" % when)
        self.P = P
        self.varname = varname
        self.clock = guess_clock(clock)
        self.record = record
        self.timestep = int(timestep)
        self.when = when
        self._binding = None
        self._mid = None
        if record is True or record is False:
            self._indices = np.arange(len(P), dtype=np.int32)
        elif isinstance(record, (int, np.integer)):
            self._indices = np.array([int(record)], dtype=np.int32)
        else:
            self._indices = np.asarray(list(record), dtype=np.int32)
        self._archived = (np.zeros(0, dtype=np.int64), np.zeros((0, len(self._indices))))

    def _lower(self, rt, gids):
        owner = self.P._owner
        var = owner.get_var_index(self.varname)
        return rt.statemon_add(gids[owner], var, self._indices + self.P._origin, self.timestep)

    def _record(self):
        if self._binding is not None:
            s, v = self._binding.read_states(self)
            return (np.concatenate([self._archived[0], s]), np.vstack([self._archived[1], v]))
        return self._archived

    def _archive(self):
        self._archived = self._record()

    def _host_state(self, d):
        d["_archived"] = self._record()

    def reinit(self):
        self._archived = (np.zeros(0, dtype=np.int64), np.zeros((0, len(self._indices))))
        if self._binding is not None:
            self._binding.clear_monitor(self)

    @property
    def times(self):
        s, _ = self._record()
        return s * self.clock.dt

    times_ = times

    @property
    def values(self):
        _, v = self._record()
        return v.T.copy()

    values_ = values

    def get_record_indices(self):
        if self.record is False:
            return []
        return self._indices

    def __getitem__(self, i):
        if self.record is False:
            raise IndexError("Neuron %d was not recorded." % i)
        pos = np.nonzero(self._indices == i)[0]
        if len(pos) == 0:
            raise IndexError("Neuron %d was not recorded." % i)
        return self.values[pos[0]]

    @property
    def N(self):
        return len(self._record()[0])

    @property
    def mean(self):
        return self._record()[1].mean(axis=0)

    @property
    def var(self):
        v = self._record()[1]
        return v.var(axis=0, ddof=1)

    @property
    def std(self):
        return self.var ** 0.5


class MultiStateMonitor(object):
    def __init__(self, G, vars=None, **kwds):
        vars = vars if vars is not None else [n for n in G._owner._names]
        self.monitors = {v: StateMonitor(G, v, **kwds) for v in vars}
        self.contained_objects = list(self.monitors.values())

    def __getitem__(self, v):
        return self.monitors[v]


class CoincidenceCounter(SpikeMonitor):
    """Coincidences between model spikes and target trains (monitor.py:
    1229-1376).  The model spikes are recorded on the device; the online
    counting runs on the host over the recorded spikes, in the order the
    reference processes them step by step."""

    def __init__(self, source, data, spiketimes_offset=None, spikedelays=None,
                 coincidence_count_algorithm="exclusive", onset=None, delta=4e-3):
        SpikeMonitor.__init__(self, source)
        self.data = np.asarray(data, dtype=float)
        N = len(source)
        self.spiketimes_offset = np.zeros(N, dtype=int) if spiketimes_offset is None else np.asarray(spiketimes_offset)
        self.spikedelays = np.zeros(N) if spikedelays is None else np.asarray(spikedelays, dtype=float)
        self.onset = 0.0 if onset is None else float(onset)
        self.algorithm = coincidence_count_algorithm
        dt = source.clock.dt
        self.delta = int(np.rint(delta / dt))

    def _count(self):
        steps, idx = self._record()
        dt = self.source.clock.dt
        N = len(self.source)
        model_length = np.zeros(N, dtype=int)
        target_length = np.zeros(N, dtype=int)
        coinc = np.zeros(N, dtype=int)
        sti = self.spiketimes_offset.copy()
        last = np.rint(self.data[sti] / dt).astype(int)
        nxt = np.rint(self.data[sti + 1] / dt).astype(int)
        last_ok = np.ones(N, bool)
        next_ok = np.ones(N, bool)
        order = np.lexsort((idx, steps))
        steps, idx = steps[order], idx[order]
        bounds = np.flatnonzero(np.diff(steps)) + 1
        for sl in np.split(np.arange(len(steps)), bounds):
            if len(sl) == 0:
                continue
            t = steps[sl[0]] * dt
            spk = idx[sl].astype(int)
            if t >= self.onset:
                model_length[spk] += 1
            T = np.rint((t + self.spikedelays[spk]) / dt).astype(int)
            rem, remT = spk, T
            while True:
                r = np.nonzero(remT > nxt[rem])[0]
                if not len(r):
                    break
                ii = rem[r]
                target_length[ii] += 1
                sti[ii] += 1
                last[ii] = nxt[ii]
                nxt[ii] = np.rint(self.data[sti[ii] + 1] / dt).astype(int)
                if self.algorithm == "exclusive":
                    last_ok[ii] = next_ok[ii]
                    next_ok[ii] = True
                rem, remT = rem[r], remT[r]
            near_last = last[spk] + self.delta >= T
            near_next = nxt[spk] - self.delta <= T
            lo, no = last_ok[spk], next_ok[spk]
            hit = (near_last & lo) | (near_next & no)
            if t >= self.onset:
                coinc[spk[hit]] += 1
            if self.algorithm == "exclusive":
                both = (near_last & lo) & (near_next & no)
                last_ok[spk] = lo & ~near_last
                next_ok[spk] = (no & ~near_next) | both
        return coinc, model_length, target_length

    @property
    def coincidences(self):
        return self._count()[0]

    @property
    def model_length(self):
        return self._count()[1]

    @property
    def target_length(self):
        return self._count()[2]


class RecentStateMonitor(StateMonitor):
    """StateMonitor of the most recent ``duration`` (monitor.py:991-1141).

    Records like StateMonitor (``record`` defaults to True); the reference's
    ring of ``num_duration = int(duration / (timestep*dt)) + 1`` slots, where
    record r sits in slot r mod num_duration, is a view over the records.
    ``values``/``times`` are sorted by time (values [time][neuron], as in the
    reference); ``unsorted_values``/``unsorted_times`` are the ring itself;
    ``get_past_values`` reads the slot ``(current_time_index - 1 -
    int((1/dt) * times)) mod num_duration`` (monitor.py:1078-1096)."""

    def __init__(self, P, varname, duration=5e-3, clock=None, record=True, timestep=1, when="end"):
        StateMonitor.__init__(self, P, varname, clock=clock, record=record, timestep=timestep, when=when)
        self.duration = float(duration)
        self.num_duration = int(self.duration / (self.timestep * self.clock.dt)) + 1
        self._invtargetdt = 1.0 / self.clock.dt

    def _ring(self):
        s, v = self._record()
        M, R = self.num_duration, len(s)
        vals = np.zeros((M, v.shape[1]))
        times = np.zeros(M)
        k = np.arange(max(0, R - M), R)
        vals[k % M] = v[k]
        times[k % M] = s[k] * self.clock.dt
        return vals, times, R % M, R >= M

    @property
    def current_time_index(self):
        return self._ring()[2]

    @property
    def has_looped(self):
        return self._ring()[3]

    def sorted_times_indices(self):
        _, times, cur, looped = self._ring()
        if not looped:
            return np.arange(cur)
        return np.argsort(times)

    @property
    def unsorted_values(self):
        return self._ring()[0]

    unsorted_values_ = unsorted_values

    def getvalues(self):
        return self._ring()[0]

    getvalues_ = getvalues

    @property
    def unsorted_times(self):
        return self._ring()[1]

    unsorted_times_ = unsorted_times

    def get_sorted_times(self):
        return self._ring()[1][self.sorted_times_indices()]

    def get_sorted_values(self):
        return self._ring()[0][self.sorted_times_indices(), :]

    times = property(get_sorted_times)
    times_ = times
    values = property(get_sorted_values)
    values_ = values

    def __getitem__(self, i):
        if self.record is False:
            raise IndexError("Neuron %d was not recorded." % i)
        pos = np.nonzero(self._indices == i)[0]
        if len(pos) == 0:
            raise IndexError("Neuron %d was not recorded." % i)
        return self.get_sorted_values()[:, pos[0]]

    def get_past_values(self, times):
        vals, _, cur, _ = self._ring()
        idx = (cur - 1 - np.array(self._invtargetdt * np.asarray(times), dtype=int)) % self.num_duration
        return vals[idx, np.arange(vals.shape[1])]

    def get_past_values_sequence(self, times_seq):
        if len(times_seq) == 0:
            return []
        vals, _, cur, _ = self._ring()
        out = []
        for times in times_seq:
            idx = (cur - 1 - np.array(self._invtargetdt * np.asarray(times), dtype=int)) % self.num_duration
            out.append(vals[idx, np.arange(vals.shape[1])])
        return out


class ISIHistogramMonitor(SpikeMonitor):
    """Interspike-interval histogram of a group (monitor.py:430-504),
    computed from the recorded spikes.

    ``bins`` are the lower bounds of the bins, the last one open-ended.  As
    in the reference, each neuron's previous spike time starts at 1000 s,
    so a neuron's first spike gives a negative interval; intervals inside
    [bins[0], bins[-1]] are counted with numpy's histogram over the bin
    edges, every other interval (the first spikes among them) in the last
    bin.  The reference passes ``delay`` on as SpikeMonitor's ``record``
    argument, so it never delays the spikes; it is ignored here too."""

    def __init__(self, source, bins, delay=0):
        SpikeMonitor.__init__(self, source, record=True, delay=0)
        self.bins = np.array(bins, dtype=np.float64)

    @property
    def count(self):
        steps, idx = self._record()
        t = np.asarray(steps, dtype=np.float64) * self.source.clock.dt
        idx = np.asarray(idx, dtype=np.int64)
        last = np.full(len(self.source), 1000.0)
        isi = np.empty(len(idx))
        for k in range(len(idx)):           # chronological order, as the updates run
            isi[k] = t[k] - last[idx[k]]
            last[idx[k]] = t[k]
        out = np.zeros(len(self.bins))
        if len(self.bins) > 1:
            h, _ = np.histogram(isi, self.bins)
            out[:-1] += h
            out[-1] += len(isi) - h.sum()
        else:
            out[-1] += len(isi)
        return out
