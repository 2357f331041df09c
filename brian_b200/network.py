"""Network container, schedule and run loop (network.py of Brian 1.4.4).

A Network collects groups, connections, STDP rules and monitors
(network.py:62-311), lowers them onto one engine handle at the first run
(the reference's ``prepare``, network.py:313-363) and advances the integer
clock by ``ceil(duration/dt)`` steps per ``run`` (network.py:541-586).

Schedule of every step (update_schedule_standard, network.py:365-380):
groups update -> connections slot (connections, spike monitors and STDP
updaters in the order they were added) -> after_connections (delayed
delivery) -> resets -> end (state monitors).  The reference groups
connections by (source, delay) in a hash-ordered dict (network.py:331-343);
here the order is the insertion order, contained objects right after their
owner.

`engine(table)` is the plugin boundary: it selects the function table the
next networks bind to.  The default is the CUDA engine; nothing in this
package selects another one.
"""
import contextlib
import inspect
import math

import numpy as np

from ._lib import Runtime, product_table
from .clock import guess_clock
from .connections import Connection, DelayConnection
from .groups import NeuronGroup, Subgroup, _GroupBase
from .monitors import SpikeMonitor, StateMonitor, MultiStateMonitor
from .stdp import ExponentialSTDP, STDP
from .timedarray import TimedArraySetter
from .synapses import Synapses

__all__ = ["Network", "MagicNetwork", "run", "reinit", "stop", "clear", "network_operation",
           "NetworkOperation", "engine", "set_global_preferences", "get_global_preference"]

_PREFS = {"useweave": False, "precision": 64, "deterministic": True, "device": 0, "persistent": True,
          "spin_limit": None, "check_finite": False, "synapse_events": None}
_table_override = []


def set_global_preferences(**kw):
    """Reference preference registry (globalprefs.py:57-106); engine keys:
    precision (64|32), deterministic (bool), device (int), persistent (bool:
    allow the single-launch step loop for networks of its shape; or 256 or
    512: allow it with that many threads per block), spin_limit (polls of a
    bounded inter-block wait before the run fails with BG_ETIMEOUT; None:
    the engine's default), check_finite (bool: every run ends with a scan of
    the state variables and a NaN or infinity fails it with BG_ENUMERIC),
    synapse_events (True: Synapses always take the event path; False:
    never; None: the engine picks it when the synapses exceed half of L2
    or the network has the shape of its persistent kernel for Synapses)."""
    _PREFS.update(kw)


def get_global_preference(k):
    return _PREFS[k]


@contextlib.contextmanager
def engine(table):
    """Bind networks prepared inside the block to another implementation of
    the engine's C ABI (a FunctionTable)."""
    _table_override.append(table)
    try:
        yield table
    finally:
        _table_override.pop()


def _current_table():
    return _table_override[-1] if _table_override else product_table()


class NetworkOperation(object):
    def __init__(self, function=None, clock=None, when="end"):
        self.function = function
        self.clock = guess_clock(clock)
        self.when = when

    def __call__(self):
        raise NotImplementedError("per-step Python operations are not supported on the engine")


def network_operation(*args, **kwds):
    raise NotImplementedError("network_operation: per-step Python callbacks are not supported on the engine")


class _Binding(object):
    """Owns one engine handle and the id maps of the objects lowered onto it."""

    def __init__(self, net, table, dt):
        self.net = net
        self.rt = Runtime(table, device=_PREFS["device"], precision=_PREFS["precision"],
                          deterministic=_PREFS["deterministic"], dt=dt, persistent=_PREFS["persistent"],
                          spin_limit=_PREFS["spin_limit"], check_finite=_PREFS["check_finite"],
                          synapse_events=_PREFS["synapse_events"])
        self.gids = {}
        self.cids = {}
        self.sids = {}
        self.mids = {}
        self.yids = {}
        self.objects = []

    def read_state(self, grp, var):
        return self.rt.get_state(self.gids[grp], var, len(grp))

    def write_state(self, grp, var, values):
        self.rt.set_state(self.gids[grp], var, values)

    def read_weights(self, c):
        return self.rt.conn_get_weights(self.cids[c], c._nnz())

    def write_weights(self, c, w):
        self.rt.conn_set_weights(self.cids[c], w)

    def write_synapse_terms(self, y, terms):
        self.rt.synapses_set_terms(self.yids[y], terms)

    def read_synapse_var(self, y, k):
        return self.rt.synapses_get_var(self.yids[y], k, len(y))

    def write_synapse_var(self, y, k, values):
        self.rt.synapses_set_var(self.yids[y], k, values)

    def read_traces(self, s):
        return self.rt.stdp_get_traces(self.sids[s], len(s.C.source), len(s.C.target))

    def read_spikes(self, m):
        return self.rt.spikemon_read(self.mids[m])

    def read_states(self, m):
        return self.rt.statemon_read(self.mids[m], len(m._indices))

    def clear_monitor(self, m):
        self.rt.monitor_clear(self.mids[m])

    def release(self):
        """Copy device-held data back into the objects and drop the handle."""
        for o in self.objects:
            if isinstance(o, NeuronGroup):
                S = o._S_host
                o._binding = None
                o._S = S
            elif isinstance(o, Connection):
                w = o._weights()
                o._binding = None
                o._w = w
            elif isinstance(o, STDP):
                o._traces()
                o._binding = None
            elif isinstance(o, Synapses):
                o._sync_vars()
                o._binding = None
            elif isinstance(o, (SpikeMonitor, StateMonitor)):
                o._archive()
                o._binding = None
        self.rt.close()


class Network(object):
    def __init__(self, *args, **kwds):
        self.groups = []
        self.connections = []
        self.operations = []
        self.stdps = []
        self.synapses = []
        self.monitors = []
        self._order = []
        self.clock = None
        self._binding = None
        self.stopped = False
        for o in args:
            self.add(o)

    def add(self, *objs):
        for o in objs:
            if isinstance(o, (list, tuple, set)):
                self.add(*o)
                continue
            if any(o is x for x in self._order):
                continue
            if isinstance(o, NeuronGroup):
                self.groups.append(o)
            elif isinstance(o, Subgroup):
                continue
            elif isinstance(o, (Connection,)):
                self.connections.append(o)
            elif isinstance(o, SpikeMonitor):
                self.connections.append(o)
            elif isinstance(o, StateMonitor):
                self.monitors.append(o)
            elif isinstance(o, STDP):
                self.stdps.append(o)
            elif isinstance(o, Synapses):
                self.synapses.append(o)
            elif isinstance(o, MultiStateMonitor):
                self.add(*o.contained_objects)
                continue
            elif isinstance(o, TimedArraySetter):
                # an explicitly added setter rides with its group
                owner = o.group._owner
                if not any(o is x for x in owner._setters):
                    owner._setters.append(o)
                continue
            elif isinstance(o, NetworkOperation):
                raise NotImplementedError("NetworkOperation objects are not supported on the engine")
            else:
                raise TypeError("cannot add %r to a Network" % (o,))
            self._order.append(o)
            self._invalidate()

    def _invalidate(self):
        if self._binding is not None:
            self._binding.release()
            self._binding = None

    def _all_groups(self):
        owners = []
        for o in self._order:
            cands = []
            if isinstance(o, NeuronGroup):
                cands = [o]
            elif isinstance(o, Connection):
                cands = [o.source._owner, o.target._owner]
            elif isinstance(o, SpikeMonitor):
                cands = [o.source._owner]
            elif isinstance(o, StateMonitor):
                cands = [o.P._owner]
            elif isinstance(o, STDP):
                cands = [o.C.source._owner, o.C.target._owner]
            elif isinstance(o, Synapses):
                cands = [o.source._owner, o.target._owner]
            for g in cands:
                if not any(g is x for x in owners):
                    owners.append(g)
        return owners

    def prepare(self, configure=None):
        """Lower the network onto one engine handle (done by the first run).
        `configure(runtime)`, when given, runs on the new handle before the
        engine builds its step (engine settings such as test hooks)."""
        if self._binding is not None:
            return
        groups = self._all_groups()
        if not groups:
            raise ValueError("empty network")
        clocks = {id(g.clock): g.clock for g in groups}
        if len(clocks) != 1:
            raise NotImplementedError("all objects must share one clock")
        self.clock = groups[0].clock
        # release objects bound to another network
        seen = set()
        for o in list(groups) + list(self._order):
            b = getattr(o, "_binding", None)
            if b is not None and id(b) not in seen:
                seen.add(id(b))
                b.release()
        for s in self.stdps:
            if not any(s.C is c for c in self.connections):
                raise ValueError("STDP on a connection that is not in the network")
        b = _Binding(self, _current_table(), self.clock.dt)
        rt = b.rt
        for g in groups:
            b.gids[g] = g._lower(rt, self.clock.dt)
            b.objects.append(g)
        stdp_of = {id(s.C): s for s in self.stdps}
        for o in self._order:
            if isinstance(o, Connection):
                b.cids[o] = o._lower(rt, b.gids)
                b.objects.append(o)
                s = stdp_of.get(id(o))
                if s is not None:
                    # the STDP updaters follow their connection in the connections slot
                    b.sids[s] = s._lower(rt, b.cids[o])
                    b.objects.append(s)
            elif isinstance(o, SpikeMonitor):
                b.mids[o] = o._lower(rt, b.gids)
                b.objects.append(o)
            elif isinstance(o, StateMonitor):
                b.mids[o] = o._lower(rt, b.gids)
                b.objects.append(o)
            elif isinstance(o, Synapses):
                b.yids[o] = o._lower(rt, b.gids)
                b.objects.append(o)
        if configure is not None:
            configure(rt)
        rt.prepare()
        pending = self.__dict__.pop("_pending_state", None)
        if pending is not None:
            # a pickled network: its dynamic state (rings, histories, traces,
            # counters, monitor records) goes back into the rebuilt engine;
            # each monitor pickled its whole record, whose tail is what the
            # engine held and now holds again, so that tail is dropped here
            rt.load_state(pending)
            for o, mid in b.mids.items():
                if isinstance(o, SpikeMonitor):
                    k = rt.spikemon_count(mid)
                    if k:
                        o._archived = tuple(x[:len(x) - k] for x in o._archived)
                elif isinstance(o, StateMonitor):
                    k = rt.statemon_count(mid)
                    if k:
                        o._archived = tuple(x[:len(x) - k] for x in o._archived)
        for o in b.objects:
            o._binding = b
        self._binding = b

    def __getstate__(self):
        """Pickling (Network.__reduce__, network.py:652): the objects pickle
        with their host-side values, and the engine's dynamic state --
        delay rings, spike histories, refractory bookkeeping, STDP traces,
        counters -- travels as bytes and is loaded into the engine that the
        first run after unpickling builds (the same objects give the same
        engine layout), so run(T1); pickle; unpickle; run(T2) equals
        run(T1 + T2)."""
        d = dict(self.__dict__)
        d["_binding"] = None
        if self._binding is not None:
            d["_pending_state"] = self._binding.rt.save_state()
        return d

    def __setstate__(self, d):
        self.__dict__.update(d)

    def run(self, duration, threads=1, report=None, report_period=10.0):
        self.stopped = False
        self.prepare()
        nsteps = self.clock.set_duration(duration)
        self._binding.rt.run(nsteps, self.clock.step)
        self.clock._n += nsteps

    def stats(self):
        self.prepare()
        return self._binding.rt.stats()

    def reinit(self, states=True):
        self.clock.reinit() if self.clock is not None else None
        if self._binding is not None:
            self._binding.rt.reinit()
        for o in self._order:
            if isinstance(o, (SpikeMonitor, StateMonitor)):
                if isinstance(o, StateMonitor) and self._binding is not None:
                    # state monitors restart with the network
                    self._invalidate()
                o.reinit()
            elif isinstance(o, NeuronGroup) and states:
                o.reinit()

    def stop(self):
        self.stopped = True

    def __contains__(self, o):
        return any(o is x for x in self._order)


# ------------------------------------------------------------------ magic
_magic_cache = {}
_CLASSES = (NeuronGroup, Connection, SpikeMonitor, StateMonitor, STDP, MultiStateMonitor, Synapses)


def _find_instances(level):
    frame = inspect.currentframe()
    for _ in range(level + 1):
        frame = frame.f_back
    found = []
    for d in (frame.f_globals, frame.f_locals):
        for v in list(d.values()):
            if isinstance(v, _CLASSES) and not any(v is x for x in found):
                found.append(v)
            elif isinstance(v, (list, tuple)):
                for w in v:
                    if isinstance(w, _CLASSES) and not any(w is x for x in found):
                        found.append(w)
    return found


def _creation_key(o):
    if isinstance(o, NeuronGroup):
        return (0, o._id)
    if isinstance(o, Connection):
        return (1, o._id)
    return (2, id(o))


class MagicNetwork(Network):
    """Network of every engine object visible in the caller's frame
    (network.py:883-898)."""

    def __init__(self, verbose=False, level=1):
        objs = _find_instances(level + 1)
        Network.__init__(self)
        groups = sorted([o for o in objs if isinstance(o, NeuronGroup)], key=lambda o: o._id)
        conns = sorted([o for o in objs if isinstance(o, Connection)], key=lambda o: o._id)
        rest = [o for o in objs if not isinstance(o, (NeuronGroup, Connection))]
        for o in groups + conns + rest:
            self.add(o)


def _magic(level):
    objs = _find_instances(level + 1)
    key = tuple(sorted(id(o) for o in objs))
    net = _magic_cache.get(key)
    if net is None:
        for k in list(_magic_cache):
            _magic_cache.pop(k)
        net = MagicNetwork(level=level + 1)
        _magic_cache[key] = net
    return net


def run(duration, threads=1, report=None, report_period=10.0):
    """Run every object visible in the caller's frame (network.py:901-938)."""
    net = _magic(1)
    net.run(duration)


def reinit(states=True):
    net = _magic(1)
    net.reinit(states)


def stop():
    pass


def clear(erase=True, all=False):
    for net in _magic_cache.values():
        net._invalidate()
    _magic_cache.clear()
