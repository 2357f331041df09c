"""TimedArray and TimedArraySetter (timedarray.py of Brian 1.4.4).

A ``TimedArray`` is an array whose first index is time: values on a clock
grid (a clock, or ``start`` and ``dt``; by default the default clock) or at
explicit ``times``.  Calling it with a time gives the value of the nearest
grid point, ``x[rint((t - t_init) / dt)]`` clamped to the array
(timedarray.py:209-235).

``TimedArraySetter(group, var, arr)`` -- or ``group.var = arr`` with a
TimedArray, or ``set_group_var_by_array`` -- sets the variable at the start
of every step, before the group's state update (timedarray.py:238-303): on a
clock grid to ``arr(t)``; on explicit (ascending) times to the last value
whose time is <= t.  A 1-D array gives every neuron of the group the same
value; a 2-D array (T, N) one value per neuron.  On the engine the setter
runs inside the group's update kernel: the row is computed from the clock
step as the reference computes it from ``clock._t`` (rint of an IEEE double
quotient), so the values are exact.

Setters run on the group's clock.  A TimedArray on another clock object must
have the group's dt; such a setter first runs at the first step whose time
is >= that clock's start.  (The reference schedules a separate clock of the
same dt before or after the group's by the order of a Python set; here the
setter is always before the update.)
"""
import math

import numpy as np

from .clock import Clock, guess_clock

__all__ = ["TimedArray", "TimedArraySetter", "set_group_var_by_array"]


class TimedArray(np.ndarray):
    def __new__(cls, arr, times=None, clock=None, start=None, dt=None):
        return np.asarray(arr).view(cls)

    def __init__(self, arr, times=None, clock=None, start=None, dt=None):
        if start is not None or dt is not None:
            if start is None:
                start = 0.0
            if clock is not None:
                raise ValueError("Specify start and dt or clock, but not both.")
            clock = Clock(t=float(start), dt=float(dt))
        if times is not None and clock is not None:
            raise ValueError("Specify times or clock but not both.")
        self.guessed_clock = times is None and clock is None
        if self.guessed_clock:
            clock = guess_clock(None)
        self.clock = clock
        if clock is not None:
            self._t_init = int(clock._t / clock._dt) * clock._dt
            self._dt = clock._dt
            times = clock._t + np.arange(len(self)) * clock._dt
        else:
            self._t_init = None
            self._dt = None
        self.times = np.asarray(times, dtype=np.float64)

    def __array_finalize__(self, orig):
        for k in ("times", "clock", "_t_init", "_dt", "guessed_clock"):
            if hasattr(orig, k):
                setattr(self, k, getattr(orig, k))

    def __reduce__(self):
        base = list(np.ndarray.__reduce__(self))
        extra = (self.times, self.clock, self.guessed_clock, self._t_init, self._dt)
        return (base[0], base[1], (base[2], extra))

    def __setstate__(self, state):
        nd, extra = state
        np.ndarray.__setstate__(self, nd)
        self.times, self.clock, self.guessed_clock, self._t_init, self._dt = extra

    def _with_times(self, values, item0):
        times = self.times[item0]
        if isinstance(item0, slice) and self.clock is not None and np.ndim(times) == 1 and len(times) > 1:
            step = times[1] - times[0]
            return TimedArray(values, clock=Clock(t=float(times[0]), dt=float(step)))
        return TimedArray(values, times=np.atleast_1d(times))

    def __getitem__(self, item):
        # slices on the time index keep a clock; other indexing keeps the times
        x = np.ndarray.__getitem__(np.asarray(self), item)
        if isinstance(item, tuple):
            return self._with_times(x, item[0])
        if isinstance(item, (int, np.integer)):
            return TimedArray(x, times=self.times[item:item + 1])
        return self._with_times(x, item)

    def __call__(self, t):
        if self.clock is None:
            raise ValueError("Can only call timed arrays if they are based on a clock.")
        if isinstance(t, (list, tuple)):
            t = np.array(t)
        if isinstance(t, np.ndarray) and t.ndim > 0:
            if self.ndim > 2:
                raise ValueError("Calling TimedArray with array valued t only supported for 1D or 2D TimedArray.")
            if self.ndim == 2 and len(t) != self.shape[1]:
                raise ValueError("Calling TimedArray with array valued t on 2D TimedArray requires len(t)=arr.shape[1]")
            k = np.array(np.rint((t - self._t_init) / self._dt), dtype=int)
            k[k < 0] = 0
            k[k >= len(self.times)] = len(self.times) - 1
            if self.ndim == 1:
                return np.asarray(self)[k]
            return np.asarray(self)[k, np.arange(len(k))]
        k = int(np.rint((float(t) - self._t_init) / self._dt))
        k = min(max(k, 0), len(self.times) - 1)
        return np.asarray(self)[k]


class TimedArraySetter(object):
    """Sets `var` of `group` from `arr` at the start of every step."""

    def __init__(self, group, var, arr, times=None, clock=None, start=None, dt=None, when="start"):
        if when != "start":
            raise NotImplementedError("TimedArraySetter runs in the 'start' slot on the engine")
        if clock is None:
            clock = arr.clock if isinstance(arr, TimedArray) and arr.clock is not None else group.clock
        self.clock = clock
        self.when = when
        self.group = group
        self.var = var
        if not isinstance(arr, TimedArray):
            arr = TimedArray(arr, times=times, clock=clock, start=start, dt=dt)
        self.arr = arr

    def reinit(self):
        pass

    def _lower(self, rt, gid, owner, dt):
        """Register on the engine: group `gid` (the owner of self.group)."""
        grp = self.group
        var = grp.get_var_index(self.var)
        vals = np.asarray(self.arr, dtype=np.float64)
        if vals.ndim == 1:
            vals = vals.reshape(-1, 1)
        elif vals.ndim != 2 or vals.shape[1] != len(grp):
            raise ValueError("a TimedArray for a group of %d neurons is (T,) or (T, %d)" % (len(grp), len(grp)))
        if len(vals) == 0:
            raise ValueError("empty TimedArray")
        if abs(self.clock.dt - dt) > 1e-12 * dt:
            raise NotImplementedError("a TimedArraySetter on a clock with another dt than its group's")
        # a setter on its own clock first runs when that clock has started
        first = 0 if self.clock is owner.clock else int(math.ceil(self.clock._t / dt - 1e-9))
        a = self.arr
        if a.clock is not None:
            rt.group_set_timed_array(gid, var, grp._origin, len(grp), vals, 0, a._t_init, a._dt, first, None)
        else:
            times = np.asarray(a.times, dtype=np.float64)
            if np.any(np.diff(times) < 0):
                raise ValueError("TimedArray times must be ascending")
            # breakpoint of row i >= 1: the first clock step s with s*dt >= times[i]
            bp = np.empty(max(0, len(times) - 1), dtype=np.int64)
            for i in range(1, len(times)):
                s = max(0, int(math.ceil(times[i] / dt)))
                while s > 0 and (s - 1) * dt >= times[i]:
                    s -= 1
                while s * dt < times[i]:
                    s += 1
                bp[i - 1] = s
            rt.group_set_timed_array(gid, var, grp._origin, len(grp), vals, 1, 0.0, 0.0, first, bp)


def set_group_var_by_array(group, var, arr, times=None, clock=None, start=None, dt=None):
    """TimedArraySetter for `group.var`, carried by the group into every
    network that contains it (timedarray.py:296-303)."""
    setter = TimedArraySetter(group, var, arr, times=times, clock=clock, start=start, dt=dt)
    group._owner._setters.append(setter)
    binding = group._owner.__dict__.get("_binding")
    if binding is not None:
        binding.net._invalidate()          # the engine is rebuilt with the setter by the next run
    return setter
