"""Neuron groups, thresholds and resets (host side).

NeuronGroup (neurongroup.py:258-599), the threshold classes of threshold.py
(Threshold 129-200, VariableThreshold 337-406, PoissonThreshold 461-479) and
the reset classes of reset.py (Reset 115-152, VariableReset 220-257,
Refractoriness 288-335).  A group keeps its state matrix on the host until a
Network binds it to an engine handle; from then on state reads and writes go
to device memory.
"""
import itertools
import re

import numpy as np

from .clock import guess_clock
from ._lib import EngineBound
from .equations import Equations, linear_propagator, _identifiers, _picklable_namespace

__all__ = ["NeuronGroup", "PoissonGroup", "SpikeGeneratorGroup", "Threshold", "VariableThreshold",
           "PoissonThreshold", "NoThreshold", "StringThreshold", "Reset", "VariableReset", "StringReset",
           "NoReset", "Refractoriness", "LazyStateUpdater", "EmpiricalThreshold"]

_counter = itertools.count()


# ---------------------------------------------------------------- thresholds
class Threshold(object):
    """S[state] > threshold (threshold.py:129-200)."""

    def __init__(self, threshold=1e-3, state=0):
        self.threshold = float(threshold)
        self.state = state


class VariableThreshold(Threshold):
    """S[state] > S[threshold_state] (threshold.py:337-406)."""

    def __init__(self, threshold_state=1, state=0):
        self.threshold_state = threshold_state
        self.state = state


class PoissonThreshold(Threshold):
    """Spike with probability S[state]*dt (threshold.py:461-479); the uniform
    draw is a Philox4x32-10 function of (seed, step, index)."""

    def __init__(self, state=0, seed=None):
        self.state = state
        self.seed = seed


class NoThreshold(Threshold):
    def __init__(self):
        pass


class EmpiricalThreshold(Threshold):
    """S[state] > threshold for neurons that did not spike in the last
    `refractory` (threshold.py:409-457), for models such as Hodgkin-Huxley
    that return to rest by their own dynamics (use with no reset)."""

    def __init__(self, threshold=1e-3, refractory=1e-3, state=0, clock=None):
        self.threshold = float(threshold)
        self.state = state
        dt = guess_clock(clock).dt
        self.refractory = int(float(refractory) / dt)
        # a whole number of steps is taken one step shorter (threshold.py:444-447)
        if self.refractory > 0 and _approx_equal(self.refractory * dt, float(refractory)):
            self.refractory -= 1


def _approx_equal(x, y):
    """is_approx_equal (utils/approximatecomparisons.py:96-98): within
    10000 machine epsilons relative to x."""
    return x == y or abs(x - y) < abs(x) * (np.finfo(np.float64).eps * 10000)


class StringThreshold(Threshold):
    """Threshold given as a string: any condition on the state variables
    (and t), compiled into the group's kernel."""

    def __init__(self, expr, level=0, namespace=None):
        self.expr = expr
        self.namespace = namespace or {}

    def __getstate__(self):
        return dict(self.__dict__, namespace=_picklable_namespace(self.namespace))


class LazyStateUpdater(object):
    """State variables that do not evolve (stateupdater.py LazyStateUpdater)."""

    def __init__(self, numstatevariables=1):
        self.nvar = numstatevariables


# -------------------------------------------------------------------- resets
class Reset(object):
    """S[state] = resetvalue for the neurons that just spiked (reset.py:115-152)."""

    def __init__(self, resetvalue=0.0, state=0):
        self.resetvalue = float(resetvalue)
        self.state = state


class VariableReset(Reset):
    """S[state] = S[resetvaluestate] (reset.py:220-257)."""

    def __init__(self, resetvaluestate=1, state=0):
        self.resetvaluestate = resetvaluestate
        self.state = state


class StringReset(Reset):
    """Reset given as a string; ``x = <constant>`` and ``x = y`` are
    supported on the network path."""

    def __init__(self, expr, level=0, namespace=None):
        self.expr = expr
        self.namespace = namespace or {}

    def __getstate__(self):
        return dict(self.__dict__, namespace=_picklable_namespace(self.namespace))


class NoReset(Reset):
    def __init__(self):
        pass


class Refractoriness(Reset):
    """Hold S[state] at resetvalue for `period` after a spike (reset.py:288-335)."""

    def __init__(self, resetvalue=0.0, period=5e-3, state=0):
        self.resetvalue = float(resetvalue)
        self.period = float(period)
        self.state = state


def _is_timed_array(value):
    from .timedarray import TimedArray
    return isinstance(value, TimedArray)


# ------------------------------------------------------------ state arrays
class StateArray(np.ndarray):
    """Array returned by ``G.v``: item assignment writes through to the group."""

    def __setitem__(self, key, value):
        super(StateArray, self).__setitem__(key, value)
        sink = getattr(self, "_sink", None)
        if sink is not None:
            grp, var = sink
            grp._write_var(var, np.asarray(self).view(np.ndarray))

    def __array_finalize__(self, obj):
        self._sink = None


class _GroupBase(EngineBound):
    def __len__(self):
        return self._n

    # owner-relative access
    def _owner_range(self):
        return self._origin, self._origin + self._n

    def get_var_index(self, name):
        owner = self._owner
        if isinstance(name, (int, np.integer)):
            return int(name)
        try:
            return owner.var_index[name]
        except KeyError:
            raise AttributeError("No state variable %r" % name)

    def state_(self, name):
        var = self.get_var_index(name)
        owner = self._owner
        full = owner._read_full(var)
        a, b = self._owner_range()
        arr = np.array(full[a:b]).view(StateArray)
        arr._sink = (self, var)
        return arr

    state = state_

    def _write_var(self, var, values):
        owner = self._owner
        full = owner._read_full(var).copy()
        a, b = self._owner_range()
        full[a:b] = values
        owner._write_full(var, full)

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        owner = self.__dict__.get("_owner")
        if owner is not None and name in owner.__dict__.get("var_index", {}):
            return self.state_(name)
        if owner is not None and name.endswith("_") and name[:-1] in owner.__dict__.get("var_index", {}):
            return self.state_(name[:-1])
        raise AttributeError(name)

    def __setattr__(self, name, value):
        owner = self.__dict__.get("_owner")
        if owner is not None and not name.startswith("_"):
            key = name[:-1] if name.endswith("_") else name
            if key in owner.__dict__.get("var_index", {}) and _is_timed_array(value):
                # G.x = TimedArray(...): a setter (neurongroup.py:645-652)
                self.set_var_by_array(key, value)
                return
            if key in owner.__dict__.get("var_index", {}):
                var = owner.var_index[key]
                vals = np.broadcast_to(np.asarray(value, dtype=np.float64), (self._n,))
                self._write_var(var, vals)
                return
        object.__setattr__(self, name, value)

    def set_var_by_array(self, var, arr, times=None, clock=None, start=None, dt=None):
        """Set `var` from a TimedArray at the start of every step
        (neurongroup.py:731-735)."""
        from .timedarray import set_group_var_by_array
        return set_group_var_by_array(self, var, arr, times=times, clock=clock, start=start, dt=dt)

    def subgroup(self, N):
        if self._next_subgroup + N > self._n:
            raise IndexError("Subgroup is too large.")
        P = self[self._next_subgroup:self._next_subgroup + N]
        self._next_subgroup += N
        return P

    def __getitem__(self, key):
        if isinstance(key, slice):
            a, b, st = key.indices(self._n)
            if st != 1:
                raise IndexError("subgroups need a unit stride")
            return Subgroup(self._owner, self._origin + a, b - a)
        raise TypeError("groups can be sliced only")

    @property
    def origin(self):
        return self._origin


class NeuronGroup(_GroupBase):
    """Group of neurons sharing one model (neurongroup.py:258-456).

    The state updater follows magic_state_updater (stateupdater.py:70-172):
    linear equations get the exact propagator; nonlinear ones (or an explicit
    `method`) are integrated by Euler, second-order Runge-Kutta (order=2 or
    method='RK') or exponential Euler (implicit=True or
    method='exponential_Euler'), generated as C and compiled into the group's
    kernel.  Thresholds: scalar, Threshold, VariableThreshold,
    EmpiricalThreshold, PoissonThreshold, or any condition string; resets:
    scalar, Reset, VariableReset, or statement strings; refractory period >
    0.9*dt selects Refractoriness as in the reference."""

    def __init__(self, N, model=None, threshold=None, reset=None, init=None, refractory=0.0, level=0,
                 clock=None, order=1, implicit=False, unit_checking=True, max_delay=0.0, compile=False,
                 freeze=False, method=None, max_refractory=None, **kw):
        object.__setattr__(self, "_owner", None)
        self._id = next(_counter)
        self.clock = guess_clock(clock)
        self._n = int(N)
        self._origin = 0
        self._next_subgroup = 0
        self.method = method
        # ---- model
        if isinstance(model, LazyStateUpdater):
            self.eqs = None
            names = ["S%d" % k for k in range(model.nvar)]
        elif model is None:
            self.eqs = None
            names = []
        else:
            if isinstance(model, str):
                model = Equations(model, level=level + 1)
            self.eqs = model
            self.eqs.prepare()
            names = list(self.eqs._diffeq_names)
        self.var_index = {nm: k for k, nm in enumerate(names)}
        for k in range(len(names)):
            self.var_index[k] = k
        self._names = names
        self._S = np.zeros((len(names), self._n))
        if init is not None:
            for k, v in enumerate(init):
                self._S[k, :] = v
        self._S_init = self._S.copy()
        self._linear = None
        # A group the network engine cannot run (numerically integrated or
        # nonlinear model, general string threshold/reset) can still be built:
        # GPUModelFitting takes its model.  Lowering it onto a network raises.
        self._fitting_only = None
        self._setters = []                 # TimedArraySetters carried by the group
        self._level = level
        # integration scheme of a generated update (None: exact linear)
        self._scheme = None
        if self.eqs is not None:
            if method not in (None, "linear", "Euler", "RK", "exponential_Euler"):
                raise NotImplementedError("integration method %r is not supported" % method)
            if method in ("Euler", "RK", "exponential_Euler"):
                self._scheme = method
            elif not self.eqs.is_linear():
                if method == "linear":
                    raise TypeError("method='linear' given for nonlinear equations")
                self._scheme = "exponential_Euler" if implicit else ("RK" if order == 2 else "Euler")
        # ---- threshold
        self._threshold = self._select_threshold(threshold, level + 1)
        # ---- reset / refractoriness (neurongroup.py:369-429)
        dt = self.clock.dt
        self._refractory = float(refractory)
        self._reset = self._select_reset(reset, level + 1)
        self._period = 0
        # spike filter next_allowed <= t, next_allowed = t + T - dt/2
        # (neurongroup.py:424-429, 506-515): on unless T < 0.9*dt
        self._refractory_time = float(refractory) - 0.5 * dt
        self._use_refractory_filter = not (float(refractory) < 0.9 * dt)
        if isinstance(self._reset, Refractoriness):
            self._period = int(self._reset.period / dt) + 1
        elif float(refractory) > 0.9 * dt and type(self._reset) is Reset:
            # a constant reset with a refractory period becomes Refractoriness
            self._reset = Refractoriness(self._reset.resetvalue, float(refractory), self._reset.state)
            self._period = int(float(refractory) / dt) + 1
        self._binding = None   # (Network runtime holder, gid)
        self._owner = self

    # ------------------------------------------------------------------
    def _var(self, ref):
        if isinstance(ref, (int, np.integer)):
            return int(ref)
        if ref not in self.var_index:
            raise ValueError("unknown state variable %r" % ref)
        return self.var_index[ref]

    def _ns(self, level):
        from .equations import _caller_namespace
        ns = {}
        if self.eqs is not None:
            ns.update(self.eqs.namespace)
        ns.update(_caller_namespace(level + 1))
        return ns

    def _select_threshold(self, threshold, level):
        if threshold is None:
            return NoThreshold()
        if isinstance(threshold, (int, float, np.floating, np.integer)) and not isinstance(threshold, bool):
            return Threshold(float(threshold), state=0)
        if isinstance(threshold, str):
            m = re.match(r"^\s*(\w+)\s*>\s*(.+?)\s*$", threshold)
            rhs = m.group(2) if m else ""
            if not m or m.group(1) not in self.var_index or (
                    rhs not in self.var_index and _identifiers(rhs) & (set(self._names) | {"t"})):
                # a general condition: compiled into the group's kernel
                return StringThreshold(threshold, namespace=self._ns(level + 1))
            if rhs in self.var_index:
                return VariableThreshold(rhs, m.group(1))
            ns = self._ns(level + 1)
            return Threshold(float(eval(rhs, ns)), m.group(1))
        if isinstance(threshold, Threshold):
            return threshold
        raise TypeError("unsupported threshold %r" % (threshold,))

    def _select_reset(self, reset, level):
        if reset is None:
            return NoReset()
        if isinstance(reset, (int, float, np.floating, np.integer)) and not isinstance(reset, bool):
            return Reset(float(reset), state=0)
        if isinstance(reset, str):
            stmts = [s.strip() for s in re.split(r"[;\n]", reset) if s.strip()]
            m = re.match(r"^(\w+)\s*=\s*(.+)$", stmts[0]) if len(stmts) == 1 else None
            rhs = m.group(2).strip() if m else ""
            if not m or m.group(1) not in self.var_index or (
                    rhs not in self.var_index and _identifiers(rhs) & (set(self._names) | {"t"})):
                # general statements: compiled into the group's kernel
                return StringReset(reset, namespace=self._ns(level + 1))
            if rhs in self.var_index:
                return VariableReset(rhs, m.group(1))
            return Reset(float(eval(rhs, self._ns(level + 1))), m.group(1))
        if isinstance(reset, Reset):
            return reset
        raise TypeError("unsupported reset %r" % (reset,))

    # ------------------------------------------------------------- state I/O
    def _read_full(self, var):
        if self._binding is not None:
            return self._binding.read_state(self, var)
        return self._S[var]

    def _write_full(self, var, values):
        if self._binding is not None:
            self._binding.write_state(self, var, values)
        else:
            self._S[var, :] = values

    def _host_state(self, d):
        d["_S"] = self._S_host

    def padded_size(self):
        """Rows of the engine's state layout: a multiple of 1024 >= len(self)."""
        return max(1024, (self._n + 1023) // 1024 * 1024)

    def use_device_buffer(self, tensor):
        """Keep this group's state in `tensor`, a contiguous CUDA tensor of
        shape (number of state variables, padded_size()) and the network's
        precision, on the network's device.  No copy: after each run the
        tensor holds the state (column i = neuron i; columns past len(self)
        are scratch), and values written into it between runs are what the
        next run starts from.  Set before the network's first run; the
        caller keeps ownership of the memory (bg_import_device_ptr)."""
        if self.__dict__.get("_binding") is not None:
            raise RuntimeError("set the device buffer before the network's first run")
        self._device_state = tensor

    def __getstate__(self):
        d = _GroupBase.__getstate__(self)
        d.pop("_device_state", None)      # device memory of this process does not pickle
        return d

    @property
    def _S_host(self):
        if self._binding is not None:
            return np.vstack([self._binding.read_state(self, k) for k in range(len(self._names))]) \
                if self._names else np.zeros((0, self._n))
        return self._S

    def num_states(self):
        return len(self._names)

    def reinit(self):
        for k in range(len(self._names)):
            self._write_full(k, self._S_init[k])

    # --------------------------------------------------------------- lowering
    def _lower(self, rt, dt):
        """Register this group on a runtime; returns the group id."""
        if self._fitting_only:
            raise NotImplementedError(self._fitting_only)
        S0 = self._S_host if self._names else np.zeros((0, self._n))
        gid = rt.group_add(S0)
        dev = self.__dict__.get("_device_state")
        if dev is not None:
            npad = rt.group_padded_size(gid)
            want = (len(self._names), npad)
            if tuple(dev.shape) != want:
                raise ValueError("device state buffer must have shape %s" % (want,))
            import torch
            if dev.dtype != (torch.float64 if rt.precision == 64 else torch.float32) or not dev.is_contiguous():
                raise ValueError("device state buffer must be a contiguous float%d tensor" % rt.precision)
            bid = rt.import_device_ptr(dev.data_ptr(), dev.numel() * dev.element_size(), rt.precision)
            rt.group_use_buffer(gid, bid)
        if self.eqs is not None and self._names and self._scheme is None:
            A, C = linear_propagator(self.eqs, dt)
            rt.group_set_linear(gid, A, C)
        for setter in self.__dict__.get("_setters", ()):
            setter._lower(rt, gid, self, dt)
        th = self._threshold
        gen_thr = isinstance(th, StringThreshold)
        gen_reset = isinstance(self._reset, StringReset)
        if self._scheme is not None or gen_thr or gen_reset:
            from .codegen import generate_model_code
            if self.eqs is None:
                raise NotImplementedError("string thresholds and resets need a model with equations")
            ns = {}
            for obj in (th, self._reset):
                ns.update(getattr(obj, "namespace", None) or {})
            code = generate_model_code(self.eqs, th.expr if gen_thr else 0.0,
                                       self._reset.expr if gen_reset else None, dt, input_var=None,
                                       scalar="float" if rt.precision == 32 else "double",
                                       scheme=self._scheme or "Euler", namespace=ns)
            if list(code.state) != list(self._names):
                raise NotImplementedError("generated model variables %s differ from the group's %s"
                                          % (code.state, self._names))
            rt.group_set_model(gid, code, update=self._scheme is not None, threshold=gen_thr, reset=gen_reset)
        if isinstance(th, EmpiricalThreshold):
            rt.group_set_threshold(gid, 1, self._var(th.state), th.threshold, 0)
            if th.refractory > 0:
                rt.group_set_empirical(gid, th.refractory)
            th = None
        if isinstance(th, PoissonThreshold):
            seed = th.seed if th.seed is not None else int(np.random.randint(0, 2 ** 31 - 1))
            th.seed = seed
            rt.group_set_poisson(gid, self._var(th.state), seed)
        elif isinstance(th, _GeneratorThreshold):
            rt.group_set_generator(gid, th.steps, th.idx)
        elif isinstance(th, VariableThreshold):
            rt.group_set_threshold(gid, 2, self._var(th.state), 0.0, self._var(th.threshold_state))
        elif th is None or isinstance(th, (NoThreshold, StringThreshold)):
            pass
        elif isinstance(th, Threshold):
            rt.group_set_threshold(gid, 1, self._var(th.state), th.threshold, 0)
        rs = self._reset
        filt = self._refractory_time if self._use_refractory_filter else -1.0
        if isinstance(rs, Refractoriness):
            rt.group_set_reset(gid, 1, self._var(rs.state), rs.resetvalue, 0)
            rt.group_set_refractory(gid, filt, self._period, self._var(rs.state), rs.resetvalue)
        elif self._use_refractory_filter:
            rt.group_set_refractory(gid, filt, 0, 0, 0.0)
        if isinstance(rs, Refractoriness):
            pass
        elif isinstance(rs, VariableReset):
            rt.group_set_reset(gid, 2, self._var(rs.state), 0.0, self._var(rs.resetvaluestate))
        elif isinstance(rs, (NoReset, StringReset)):
            pass
        elif isinstance(rs, Reset):
            rt.group_set_reset(gid, 1, self._var(rs.state), rs.resetvalue, 0)
        return gid

    def __repr__(self):
        return "NeuronGroup(%d, vars=%s)" % (self._n, self._names)


class Subgroup(_GroupBase):
    """A contiguous slice of a NeuronGroup (neurongroup.py:551-599)."""

    def __init__(self, owner, origin, n):
        object.__setattr__(self, "_owner", None)
        self._n = int(n)
        self._origin = int(origin)
        self._next_subgroup = 0
        self.clock = owner.clock
        self._owner = owner

    def __repr__(self):
        return "Subgroup(%r, origin=%d, n=%d)" % (self._owner, self._origin, self._n)


class PoissonGroup(NeuronGroup):
    """Independent Poisson spike sources (directcontrol.py:406-447).

    `rates` (Hz, scalar or array) is state variable 0 ('rate').  `seed`
    keys the counter-based uniform stream."""

    def __init__(self, N, rates=0.0, clock=None, seed=None):
        NeuronGroup.__init__(self, N, model=None, threshold=None, clock=clock)
        self._names = ["rate"]
        self.var_index = {"rate": 0, 0: 0}
        self._S = np.zeros((1, self._n))
        if callable(rates):
            raise NotImplementedError("time-varying Poisson rates are not supported")
        self._S[0, :] = rates
        self._S_init = self._S.copy()
        self._threshold = PoissonThreshold(state=0, seed=seed)


class _GeneratorThreshold(Threshold):
    def __init__(self, steps, idx):
        self.steps = steps
        self.idx = idx


class SpikeGeneratorGroup(NeuronGroup):
    """Emits given spikes (directcontrol.py:63-268): spike (i, t) fires at
    step ceil(t/dt); spikes are sorted by (step, index)."""

    def __init__(self, N, spiketimes, clock=None, period=None, sort=True, gather=None):
        NeuronGroup.__init__(self, N, model=None, threshold=None, clock=clock)
        if period is not None:
            raise NotImplementedError("periodic SpikeGeneratorGroup is not supported")
        if isinstance(spiketimes, tuple):
            idx, times = np.asarray(spiketimes[0]), np.asarray(spiketimes[1], dtype=float)
        elif isinstance(spiketimes, np.ndarray):
            idx, times = spiketimes[:, 0], spiketimes[:, 1]
        else:
            pairs = list(spiketimes)
            idx = np.array([p[0] for p in pairs], dtype=np.int64)
            times = np.array([float(p[1]) for p in pairs], dtype=float)
        steps = np.ceil(times / self.clock.dt).astype(np.int64)
        idx = np.asarray(idx).astype(np.int64)
        order = np.lexsort((idx, steps))
        steps, idx = steps[order], idx[order]
        if len(steps):
            keep = np.ones(len(steps), bool)
            keep[1:] = (steps[1:] != steps[:-1]) | (idx[1:] != idx[:-1])
            steps, idx = steps[keep], idx[keep]
        self._threshold = _GeneratorThreshold(steps, idx.astype(np.int32))
