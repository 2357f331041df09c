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

On a DelayConnection (stdp.py:296-368) the presynaptic code splits into an
immediate part (``A_pre += Ap`` at the spike) and a delayed part run for the
spikes of max_delay ago, whose ``w += A_post`` reads A_post as it was when
the spike reached each target; the postsynaptic ``w += A_pre`` reads A_pre
as it was when each source's spike left.  The reference gets those past
values from two RecentStateMonitors (monitor.py:991-1099); the engine keeps
the same ring of recorded traces on the device and looks each synapse up by
a lag computed here with the reference's float arithmetic.
"""
import numpy as np

import re

from ._lib import EngineBound
from .equations import Equations, linear_propagator, _caller_namespace, _identifiers

__all__ = ["ExponentialSTDP", "STDP"]

_INTER = {"all": 0, "nearest": 1, "nearest_pre": 2, "nearest_post": 3}


def _code_bound(x):
    """The reference inserts the bounds into generated code with '%e'
    (stdp.py:403-407), i.e. rounded to 7 significant digits."""
    return float("%e" % x)


def _lines(code):
    """Statements of a code string: lines, or ';'-separated on one line
    (stdp.py:205-214)."""
    if "\n" in code:
        parts = code.split("\n")
    else:
        parts = code.split(";")
    return [p.split("#", 1)[0].strip() for p in parts if p.split("#", 1)[0].strip()]


def _modified(lines):
    """Variables assigned by the statements (modified_variables)."""
    out = set()
    for ln in lines:
        m = re.match(r"^(\w+)\s*[-+*/]?=(?!=)", ln)
        if m:
            out.add(m.group(1))
    return out


class STDP(EngineBound):
    """Spike-timing-dependent plasticity from equations and code strings
    (stdp.py:92-449).

    The reference separates the equations into a presynaptic and a
    postsynaptic group and runs the code strings in SpikeMonitors.  The
    engine runs the family ExponentialSTDP generates: one linear trace
    equation per side, a presynaptic code of ``x_pre += c`` (or ``= c``) and
    a w line in ``x_post``, a postsynaptic code of ``x_post += c`` (or
    ``= c``) and a w line in ``x_pre``, each w line one of ``w += x``,
    ``w *= (1+x)``, ``w += (wmax-w)*x`` (the last two on FP64 weights);
    weights clipped to [wmin, wmax] after each update.  Other code raises
    NotImplementedError.  Constants in the code are looked up
    in the caller's namespace (``level`` frames up), as the reference does."""

    def __init__(self, C, eqs, pre, post, wmin=0, wmax=np.inf, level=0, clock=None, delay_pre=None,
                 delay_post=None):
        ns = _caller_namespace(level + 1)
        eqs_obj = eqs if isinstance(eqs, Equations) else Equations(eqs, level=level + 1)
        ns_eq = dict(eqs_obj._namespace)
        pre_lines, post_lines = _lines(pre), _lines(post)
        names = list(eqs_obj._diffeq_names)
        vars_pre = [v for v in names if v in _modified(pre_lines)]
        vars_post = [v for v in names if v in _modified(post_lines)]
        if len(names) != 2 or len(vars_pre) != 1 or len(vars_post) != 1 or vars_pre == vars_post:
            raise NotImplementedError("the engine runs STDP with one presynaptic and one postsynaptic trace")
        xp, xq = vars_pre[0], vars_post[0]
        Ap, pre_set, pre_mode, wx_pre = self._trace_rule(pre_lines, xp, xq, ns)
        Am, post_set, post_mode, wx_post = self._trace_rule(post_lines, xq, xp, ns)
        if wx_pre is not None and wx_post is not None and wx_pre != wx_post:
            raise NotImplementedError("two different maxima in the soft-bound updates")
        inter = {(False, False): 0, (True, True): 1, (False, True): 3}.get((pre_set, post_set))
        if inter is None:
            raise NotImplementedError("presynaptic '=' with postsynaptic '+=' rule")
        clock = clock if clock is not None else C.source.clock
        decay = []
        for v in (xp, xq):
            # each trace is a separate 1x1 linear group (stdp.py:282-293)
            one = Equations("d%s/dt=%s : %s" % (v, eqs_obj._string[v], eqs_obj._units[v] or "1"), **ns_eq) \
                if ns_eq else Equations("d%s/dt=%s : %s" % (v, eqs_obj._string[v], eqs_obj._units[v] or "1"),
                                        level=level + 1)
            if set(_identifiers(eqs_obj._string[v])) & (set(names) - {v}):
                raise NotImplementedError("coupled trace equations")
            a, c = linear_propagator(one, clock.dt)
            decay += [a[0, 0], c[0]]
        self.eqs = eqs_obj
        self._setup(C, np.array(decay, dtype=np.float64), Ap, Am, wmin, wmax, inter, clock, delay_pre, delay_post)
        self.pre_mode, self.post_mode = pre_mode, post_mode
        self.wx = wx_pre if wx_pre is not None else (wx_post if wx_post is not None else 0.0)

    @staticmethod
    def _w_line(line, other, ns):
        """(mode, exact maximum or None) of a w line: 'w += other' (0),
        'w *= (1+other)' (1), 'w += (wmax-w)*other' (2) (stdp.py:510-533)."""
        t = line.replace(" ", "")
        if t == "w+=%s" % other:
            return 0, None
        if t in ("w*=(1+%s)" % other, "w*=1+%s" % other):
            return 1, None
        m = re.match(r"^w\+=\((.+)-w\)\*%s$" % re.escape(other), t)
        if m and not (_identifiers(m.group(1)) & {"w", other}):
            return 2, float(eval(m.group(1), {"__builtins__": {}}, ns))
        return None

    @classmethod
    def _trace_rule(cls, lines, own, other, ns):
        """(constant, '=' instead of '+=', w-line mode, exact maximum) of
        'own (+)= c' next to a w line."""
        if len(lines) != 2:
            raise NotImplementedError("STDP code other than a trace update and a w update: %r" % (lines,))
        rule, wl = None, None
        for ln in lines:
            w = cls._w_line(ln, other, ns) if ln.lstrip().startswith("w") else None
            if w is not None:
                wl = w
                continue
            m = re.match(r"^(\w+)\s*(\+=|=)\s*(.+)$", ln)
            if m and m.group(1) == own and not (_identifiers(m.group(3)) & {own, other, "w"}):
                rule = (float(eval(m.group(3), {"__builtins__": {}}, ns)), m.group(2) == "=")
            else:
                raise NotImplementedError("STDP statement: %r" % ln)
        if rule is None or wl is None:
            raise NotImplementedError("STDP code other than a trace update and a w update: %r" % (lines,))
        return rule[0], rule[1], wl[0], wl[1]

    def _setup(self, C, decay, Ap, Am, wmin, wmax, inter, clock, delay_pre, delay_post):
        self.C = C
        self.Ap, self.Am = float(Ap), float(Am)
        self.wmin, self.wmax = _code_bound(float(wmin)), _code_bound(float(wmax))
        self.interactions = inter
        self.clock = clock
        from .connections import DelayConnection
        self.delayed = isinstance(C, DelayConnection)
        if self.delayed and (delay_pre is not None or delay_post is not None):
            raise ValueError("Must use delay_pre=delay_post=None for the moment.")
        dt = self.clock.dt
        self.decay = decay
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
        self.pre_mode = self.post_mode = 0
        self.wx = 0.0
        self._binding = None
        self._sid = None
        self._A_pre = np.zeros(len(C.source))
        self._A_post = np.zeros(len(C.target))
        self.contained_objects = []

    def _delayed_schedule(self):
        """(pre_delay bins, history length, lag_pre, lag_post) of the delayed
        updaters, per synapse in the connection's CSR order.

        max_delay = C._max_delay * dt (stdp.py:297); the delayed presynaptic
        updater is a SpikeMonitor delayed by int(max_delay / dt) bins
        (monitor.py:142); the trace monitors keep int((C._max_delay+1)*dt / dt)
        + 1 records (monitor.py:1024-1026) and look a synapse of delay d up
        int((1/dt) * times) records before the last one (monitor.py:1092),
        times = max_delay - d before a presynaptic update and d before a
        postsynaptic one (stdp.py:335-336).  The expression 'max_delay-d' gets
        max_delay substituted as text by str(float(max_delay)), which keeps 12
        significant digits (stdp.py:78)."""
        C = self.C
        dt_t, dt_s, dt = float(C.target.clock.dt), float(C.source.clock.dt), float(self.clock.dt)
        max_delay = C._md * dt_t
        pre_delay = int(max_delay / dt_s)
        hist_len = int(((C._md + 1) * dt_t) / (1 * dt)) + 1
        if hist_len > 256:
            raise NotImplementedError("STDP on a DelayConnection with max_delay beyond 254 steps")
        maxd = float("%.12g" % max_delay)
        inv = 1.0 / dt
        d = C._delay_seconds()
        lag_pre = np.array(inv * (maxd - d), dtype=np.int64) % hist_len
        lag_post = np.array(inv * d, dtype=np.int64) % hist_len
        return pre_delay, hist_len, lag_pre.astype(np.uint8), lag_post.astype(np.uint8)

    def _lower(self, rt, cid):
        if self.delayed:
            pre_delay, hist_len, lag_pre, lag_post = self._delayed_schedule()
            sid = rt.stdp_add_delayed(cid, self.decay, self.Ap, self.Am, self.wmin, self.wmax, self.interactions,
                                      pre_delay, hist_len, lag_pre, lag_post)
        else:
            sid = rt.stdp_add(cid, self.decay, self.Ap, self.Am, self.wmin, self.wmax, self.interactions,
                              self.pre_delay, self.post_delay)
        if self.pre_mode or self.post_mode:
            rt.stdp_set_update(sid, self.pre_mode, self.post_mode, self.wx)
        return sid

    def _host_state(self, d):
        d["_A_pre"], d["_A_post"] = self._binding.read_traces(self)

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


class ExponentialSTDP(STDP):
    """Exponential STDP (stdp.py:452-539): the trace equations and code
    strings of the reference's ExponentialSTDP, run through STDP; additive,
    multiplicative and mixed updates (the last two on FP64 weights)."""

    def __init__(self, C, taup, taum, Ap, Am, interactions="all", wmin=0, wmax=None, update="additive",
                 delay_pre=None, delay_post=None, clock=None):
        if wmax is None:
            raise AttributeError("You must specify the maximum synaptic weight")
        wmax = float(wmax)
        eqs = Equations("dA_pre/dt=-A_pre/taup : 1\ndA_post/dt=-A_post/taum : 1", taup=float(taup),
                        taum=float(taum), wmax=wmax)
        if interactions == "all":
            pre, post = "A_pre+=Ap", "A_post+=Am"
        elif interactions == "nearest":
            pre, post = "A_pre=Ap", "A_post=Am"
        elif interactions == "nearest_pre":
            pre, post = "A_pre=Ap", "A_post=+Am"
        elif interactions == "nearest_post":
            pre, post = "A_pre+=Ap", "A_post=Am"
        else:
            raise AttributeError("Unknown interaction type " + interactions)
        Ap, Am = float(Ap), float(Am)
        if update == "additive":
            Ap *= wmax
            Am *= wmax
            pre += "\nw+=A_post"
            post += "\nw+=A_pre"
        elif update == "multiplicative":
            pre += "\nw*=(1+A_post)" if Am < 0 else "\nw+=(wmax-w)*A_post"
            post += "\nw*=(1+A_pre)" if Ap < 0 else "\nw+=(wmax-w)*A_pre"
        elif update == "mixed":
            if Am < 0 and Ap > 0:
                Ap *= wmax
                pre += "\nw*=(1+A_post)"
                post += "\nw+=A_pre"
            elif Am > 0 and Ap < 0:
                Am *= wmax
                post += "\nw*=(1+A_pre)"
                pre += "\nw+=A_post"
            elif Am > 0:
                raise AttributeError("There is no depression in STDP rule")
            else:
                raise AttributeError("There is no potentiation in STDP rule")
        else:
            raise AttributeError("Unknown update type " + update)
        self.taup, self.taum = float(taup), float(taum)
        STDP.__init__(self, C, eqs=eqs, pre=pre, post=post, wmin=wmin, wmax=wmax, delay_pre=delay_pre,
                      delay_post=delay_post, clock=clock)
        # the reference's interaction names (nearest_pre runs as nearest)
        self.interactions = _INTER[interactions]
