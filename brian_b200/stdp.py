"""Spike-timing-dependent plasticity on a Connection.

ExponentialSTDP (stdp.py:452-539 of Brian 1.4.4) builds the trace equations
``dA_pre/dt = -A_pre/taup``, ``dA_post/dt = -A_post/taum`` and the rules
pre: ``A_pre += Ap; w += A_post``, post: ``A_post += Am; w += A_pre`` (with
``Ap, Am`` scaled by ``wmax`` for additive updates), clipped to
``[wmin, wmax]`` after each update.  The reference separates the traces
into two NeuronGroups with 1x1 linear updaters (stdp.py:282-293) and runs
the pre/post code as SpikeMonitors in the connections slot (stdp.py:31-54,
370-414); the engine keeps the traces on the device and fuses the
presynaptic update into the connection's propagation kernel.
"""
import numpy as np

from .equations import Equations, linear_propagator

__all__ = ["ExponentialSTDP", "STDP"]

_INTER = {"all": 0, "nearest": 1, "nearest_pre": 2, "nearest_post": 3}


def _code_bound(x):
    """The reference inserts the bounds into generated code with '%e'
    (stdp.py:403-407), i.e. rounded to 7 significant digits."""
    return float("%e" % x)


class ExponentialSTDP(object):
    def __init__(self, C, taup, taum, Ap, Am, interactions="all", wmin=0, wmax=None, update="additive",
                 delay_pre=None, delay_post=None, clock=None):
        if wmax is None:
            raise AttributeError("You must specify the maximum synaptic weight")
        if interactions not in _INTER:
            raise AttributeError("Unknown interaction type " + interactions)
        if update != "additive":
            raise NotImplementedError("only additive ExponentialSTDP runs on the engine")
        wmax = float(wmax)
        self.C = C
        self.taup, self.taum = float(taup), float(taum)
        self.Ap, self.Am = float(Ap) * wmax, float(Am) * wmax
        self.wmin, self.wmax = _code_bound(float(wmin)), _code_bound(wmax)
        self.interactions = _INTER[interactions]
        self.clock = clock if clock is not None else C.source.clock
        dt = self.clock.dt
        eqs = Equations("dA_pre/dt=-A_pre/taup : 1\ndA_post/dt=-A_post/taum : 1", taup=self.taup,
                        taum=self.taum)
        # each trace is a separate 1x1 linear group in the reference
        a_pre, c_pre = linear_propagator(Equations("dA_pre/dt=-A_pre/taup : 1", taup=self.taup), dt)
        a_post, c_post = linear_propagator(Equations("dA_post/dt=-A_post/taum : 1", taup=self.taup,
                                                     taum=self.taum), dt)
        self.decay = np.array([a_pre[0, 0], c_pre[0], a_post[0, 0], c_post[0]], dtype=np.float64)
        self.eqs = eqs
        conn_delay = getattr(C, "delay", 0) if isinstance(getattr(C, "delay", 0), int) else 0
        if delay_pre is None and delay_post is None:
            self.pre_delay, self.post_delay = conn_delay, 0
        elif delay_pre is None:
            self.post_delay = int(float(delay_post) / dt)
            self.pre_delay = conn_delay - self.post_delay
        elif delay_post is None:
            self.pre_delay = int(float(delay_pre) / dt)
            self.post_delay = conn_delay - self.pre_delay
        else:
            self.pre_delay, self.post_delay = int(float(delay_pre) / dt), int(float(delay_post) / dt)
        if self.pre_delay < 0 or self.post_delay < 0:
            raise AttributeError("STDP delay larger than the connection delay")
        self._binding = None
        self._sid = None
        self._A_pre = np.zeros(len(C.source))
        self._A_post = np.zeros(len(C.target))
        self.contained_objects = []

    def _lower(self, rt, cid):
        return rt.stdp_add(cid, self.decay, self.Ap, self.Am, self.wmin, self.wmax, self.interactions,
                           self.pre_delay, self.post_delay)

    def _traces(self):
        if self._binding is not None:
            self._A_pre, self._A_post = self._binding.read_traces(self)
        return self._A_pre, self._A_post

    @property
    def A_pre(self):
        return self._traces()[0]

    @property
    def A_post(self):
        return self._traces()[1]


def STDP(C, eqs, pre, post, wmin=0, wmax=np.inf, level=0, clock=None, delay_pre=None, delay_post=None):
    """General STDP rules are generated code in the reference (stdp.py:92-449);
    the engine runs the exponential additive family through ExponentialSTDP."""
    raise NotImplementedError("use ExponentialSTDP: general STDP code strings are not compiled by the engine")
