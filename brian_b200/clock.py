"""Integer-tick clock (clock.py:52-224 of Brian 1.4.4).

Time is ``t = n*dt`` with an integer step counter ``n``; ``set_duration``
schedules ``ceil(duration/dt)`` steps (clock.py:204-206).
"""
import math

__all__ = ["Clock", "defaultclock", "reinit_default_clock", "guess_clock", "define_default_clock"]


class Clock(object):
    def __init__(self, dt=0.1e-3, t=0.0, order=0, makedefaultclock=False):
        self._dt = float(dt)
        self._n = int(float(t) / self._dt)
        self._end = self._n
        self.order = order
        if makedefaultclock:
            global defaultclock
            defaultclock = self

    # -- properties mirroring the reference attribute names
    @property
    def dt(self):
        return self._dt

    @dt.setter
    def dt(self, value):
        self._dt = float(value)

    @property
    def t(self):
        return self._n * self._dt

    @t.setter
    def t(self, value):
        self._n = int(float(value) / self._dt)

    _t = property(lambda self: self._n * self._dt)

    @property
    def step(self):
        """Current integer step."""
        return self._n

    def tick(self):
        self._n += 1

    def reinit(self, t=0.0):
        self._n = int(float(t) / self._dt)

    def set_duration(self, duration):
        """Number of steps a run of `duration` takes (clock.py:204-206)."""
        self._end = self._n + int(math.ceil(float(duration) / self._dt))
        return self._end - self._n

    def still_running(self):
        return self._n < self._end

    def __repr__(self):
        return "Clock(dt=%r, t=%r)" % (self._dt, self.t)


defaultclock = Clock()


def reinit_default_clock(t=0.0):
    defaultclock.reinit(t)


def define_default_clock(dt=0.1e-3, t=0.0):
    global defaultclock
    defaultclock.dt = dt
    defaultclock.reinit(t)
    return defaultclock


def guess_clock(clock=None):
    return clock if clock is not None else defaultclock
