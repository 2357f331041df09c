"""Connections: construction on the host, compressed rows on the device.

Connection (connection.py:15-463) and DelayConnection (delayconnection.py:
17-337).  Weights are gathered into a construction list while the user
connects (connect_random, connect_full, connect_one_to_one, connect, C[i,j]
= w) and compressed to CSR rows with ascending targets at the first run
(SparseConnectionMatrix, connectionmatrix.py:196-387), or kept as a dense
matrix for ``structure='dense'`` (connectionmatrix.py:141-193).

Random connectivity uses numpy's Generator(PCG64(seed)) per call; the
reference's mix of numpy and Python ``random`` streams cannot be reproduced
under Python 3, so equal seeds give equal matrices within this package only.
"""
import math

import numpy as np

from ._lib import EngineBound
from .groups import NeuronGroup, Subgroup

__all__ = ["Connection", "DelayConnection", "IdentityConnection", "random_matrix_csr",
           "fixed_indegree_csr"]


def _rng(seed):
    if seed is None:
        seed = int(np.random.randint(0, 2 ** 31 - 1))
    return np.random.Generator(np.random.PCG64(seed))


def random_matrix_csr(n, m, p, seed=None):
    """Bernoulli(p) connectivity, rows ascending (construction.py:42-147):
    each row draws k ~ Binomial(m, p) distinct targets."""
    rng = _rng(seed)
    ks = rng.binomial(m, p, size=n)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(ks, out=rowptr[1:])
    cols = np.empty(rowptr[-1], dtype=np.int32)
    for i in range(n):
        if ks[i]:
            cols[rowptr[i]:rowptr[i + 1]] = np.sort(rng.choice(m, ks[i], replace=False))
    return rowptr, cols


def fixed_indegree_csr(n, m, k, seed=None, chunk=1 << 16):
    """Every target j receives exactly k distinct sources drawn uniformly
    (random_matrix_fixed_column, construction.py:149-177), returned as CSR
    over sources with ascending targets.  Vectorised for very large n*k."""
    rng = _rng(seed)
    if k > n:
        raise ValueError("in-degree larger than the source population")
    src_parts = []
    for j0 in range(0, m, chunk):
        j1 = min(m, j0 + chunk)
        # k distinct sources per target: sample with rejection of duplicates
        s = rng.integers(0, n, size=(j1 - j0, k), dtype=np.int64)
        s.sort(axis=1)
        dup = np.zeros_like(s, dtype=bool)
        dup[:, 1:] = s[:, 1:] == s[:, :-1]
        while dup.any():
            s[dup] = rng.integers(0, n, size=int(dup.sum()))
            s.sort(axis=1)
            dup[:] = False
            dup[:, 1:] = s[:, 1:] == s[:, :-1]
        src_parts.append(s)
    src = np.concatenate(src_parts, axis=0)             # (m, k)
    tgt = np.repeat(np.arange(m, dtype=np.int64), k)
    src = src.reshape(-1)
    order = np.argsort(src * m + tgt, kind="stable")
    src = src[order]
    cols = tgt[order].astype(np.int32)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=rowptr[1:])
    return rowptr, cols


class _Construction(object):
    """Entries (i, j, w) in insertion order; a later entry at the same
    position replaces an earlier one, zeros are dropped at compression."""

    def __init__(self, shape):
        self.shape = shape
        self.rows, self.cols, self.vals = [], [], []

    def add(self, i, j, w):
        i = np.atleast_1d(np.asarray(i, dtype=np.int64))
        j = np.atleast_1d(np.asarray(j, dtype=np.int64))
        w = np.broadcast_to(np.asarray(w, dtype=np.float64), i.shape)
        self.rows.append(i)
        self.cols.append(j)
        self.vals.append(np.array(w))

    def add_csr(self, i0, j0, rowptr, cols, w):
        n = len(rowptr) - 1
        i = np.repeat(np.arange(n, dtype=np.int64), np.diff(rowptr)) + i0
        self.add(i, np.asarray(cols, dtype=np.int64) + j0, w)

    def to_csr(self):
        n, m = self.shape
        if not self.rows:
            return np.zeros(n + 1, np.int64), np.zeros(0, np.int32), np.zeros(0)
        i = np.concatenate(self.rows)
        j = np.concatenate(self.cols)
        w = np.concatenate(self.vals)
        if len(self.rows) == 1 and len(i) and np.all(np.diff(i * m + j) > 0):
            key_order = None
        else:
            key = i * m + j
            order = np.argsort(key, kind="stable")
            key = key[order]
            last = np.ones(len(key), bool)
            last[:-1] = key[1:] != key[:-1]
            sel = order[last]
            i, j, w = i[sel], j[sel], w[sel]
            key_order = sel
        nz = w != 0
        i, j, w = i[nz], j[nz], w[nz]
        rowptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(i, minlength=n), out=rowptr[1:])
        return rowptr, j.astype(np.int32), w


class ConnectionMatrixView(object):
    """Read access to a compressed connection matrix (C.W)."""

    def __init__(self, conn):
        self._c = conn

    @property
    def shape(self):
        return (len(self._c.source), len(self._c.target))

    def todense(self):
        c = self._c
        w = c._weights()
        n, m = self.shape
        if c._dense is not None:
            return w.reshape(n, m).copy()
        D = np.zeros((n, m))
        rows = np.repeat(np.arange(n), np.diff(c._rowptr))
        D[rows, c._cols] = w
        return D

    def getnnz(self):
        c = self._c
        c.compress()
        return c._nnz()

    nnz = property(getnnz)

    def get_row(self, i):
        c = self._c
        c.compress()
        w = c._weights()
        if c._dense is not None:
            m = len(c.target)
            return w[i * m:(i + 1) * m].copy()
        return w[c._rowptr[i]:c._rowptr[i + 1]].copy()

    def __getitem__(self, key):
        return self._c.__getitem__(key)


class Connection(EngineBound):
    """Propagates source spikes to a target state variable (connection.py:15).

    ``Connection(source, target, state=0, delay=0*ms, modulation=None,
    structure='sparse', weight=None, sparseness=None, max_delay=5*ms)``.
    A non-float ``delay`` (True, an array, a pair) makes a DelayConnection, as
    in the reference (connection.py:176-181).  Extra keyword ``dtype``
    (float64 default, or float32) sets the weight storage type."""

    _count = 0

    def __new__(cls, source=None, target=None, state=0, delay=0.0, *args, **kwds):
        if cls is Connection and (isinstance(delay, bool) or
                                  not isinstance(delay, (int, float, np.floating, np.integer))):
            return object.__new__(DelayConnection)
        return object.__new__(cls)

    def __init__(self, source, target, state=0, delay=0.0, modulation=None, structure="sparse", weight=None,
                 sparseness=None, max_delay=5e-3, dtype=np.float64, **kwds):
        self.source = source
        self.target = target
        self.state = state
        self.nstate = target.get_var_index(state)
        self._nstate_mod = None if modulation is None else source.get_var_index(modulation)
        if structure not in ("sparse", "dense", "dynamic"):
            raise ValueError("unknown structure %r" % structure)
        self.structure = structure
        self.dtype = np.dtype(dtype)
        self._build = _Construction((len(source), len(target)))
        self._denseW = np.zeros((len(source), len(target))) if structure == "dense" else None
        self.iscompressed = False
        self._rowptr = self._cols = self._w = self._dense = None
        self._wshared = None       # the one weight of every synapse (then _w stays None until needed)
        self._binding = None
        if not isinstance(self, DelayConnection):
            self.delay = int(float(delay) / source.clock.dt)   # homogeneous delay in bins
        Connection._count += 1
        self._id = Connection._count
        self._keyword_based_init(weight=weight, sparseness=sparseness)

    # ------------------------------------------------------------ building
    def _keyword_based_init(self, weight=None, sparseness=None):
        if weight is None and sparseness is None:
            return
        if weight is None:
            weight = 1.0
        if sparseness is None:
            sparseness = 1
        if isinstance(weight, np.ndarray) or hasattr(weight, "tocoo"):
            self.connect(W=weight)
        elif sparseness == 1:
            self.connect_full(weight=weight)
        else:
            self.connect_random(weight=weight, p=sparseness)

    def origin(self, P, Q):
        return (P._origin - self.source._origin, Q._origin - self.target._origin)

    def _check_open(self):
        if self.iscompressed:
            raise RuntimeError("the connection matrix is compressed; use C[i,j] = w or set weights")

    def _insert_dense(self, i0, j0, W):
        W = np.asarray(W, dtype=np.float64)
        if self._denseW is not None:
            self._denseW[i0:i0 + W.shape[0], j0:j0 + W.shape[1]] = W
            return
        ii, jj = np.nonzero(W)
        self._build.add(ii + i0, jj + j0, W[ii, jj])

    def connect(self, source=None, target=None, W=None):
        P = source or self.source
        Q = target or self.target
        self._check_open()
        i0, j0 = self.origin(P, Q)
        if hasattr(W, "tocoo"):
            coo = W.tocoo()
            if self._denseW is not None:
                self._denseW[coo.row + i0, coo.col + j0] = coo.data
            else:
                self._build.add(coo.row.astype(np.int64) + i0, coo.col.astype(np.int64) + j0, coo.data)
        else:
            self._insert_dense(i0, j0, W)

    def connect_random(self, source=None, target=None, p=1.0, weight=1.0, fixed=False, seed=None,
                       sparseness=None, **kwds):
        P = source or self.source
        Q = target or self.target
        if sparseness is not None:
            p = sparseness
        self._check_open()
        i0, j0 = self.origin(P, Q)
        if fixed:
            rowptr, cols = fixed_indegree_csr(len(P), len(Q), int(p * len(P)), seed=seed)
        else:
            rowptr, cols = random_matrix_csr(len(P), len(Q), p, seed=seed)
        rows = np.repeat(np.arange(len(P), dtype=np.int64), np.diff(rowptr))
        if callable(weight):
            try:
                w = np.asarray(weight(rows, cols.astype(np.int64)), dtype=np.float64)
                if w.shape != rows.shape:
                    raise ValueError
            except Exception:
                w = np.array([float(weight(int(a), int(b))) for a, b in zip(rows, cols)])
        else:
            w = float(weight)
        if self._denseW is not None:
            self._denseW[rows + i0, cols + j0] = w
        else:
            self._build.add(rows + i0, cols.astype(np.int64) + j0, w)
        self._after_connect(P, Q, rows + i0, cols.astype(np.int64) + j0, kwds)

    def connect_full(self, source=None, target=None, weight=1.0, **kwds):
        P = source or self.source
        Q = target or self.target
        self._check_open()
        i0, j0 = self.origin(P, Q)
        n, m = len(P), len(Q)
        if callable(weight):
            W = np.zeros((n, m))
            for i in range(n):
                try:
                    W[i, :] = weight(i, 1.0 * np.arange(m))
                except Exception:
                    W[i, :] = [float(weight(i, j)) for j in range(m)]
        else:
            W = float(weight) * np.ones((n, m))
        if self._denseW is not None:
            self._denseW[i0:i0 + n, j0:j0 + m] = W
        else:
            ii, jj = np.meshgrid(np.arange(n), np.arange(m), indexing="ij")
            self._build.add(ii.reshape(-1) + i0, jj.reshape(-1) + j0, W.reshape(-1))
        rows = np.repeat(np.arange(n, dtype=np.int64), m) + i0
        cols = np.tile(np.arange(m, dtype=np.int64), n) + j0
        self._after_connect(P, Q, rows, cols, kwds)

    def connect_one_to_one(self, source=None, target=None, weight=1.0, **kwds):
        P = source or self.source
        Q = target or self.target
        if len(P) != len(Q):
            raise AttributeError("The connected (sub)groups must have the same size.")
        self._check_open()
        i0, j0 = self.origin(P, Q)
        k = np.arange(len(P), dtype=np.int64)
        if self._denseW is not None:
            self._denseW[k + i0, k + j0] = float(weight)
        else:
            self._build.add(k + i0, k + j0, float(weight))
        self._after_connect(P, Q, k + i0, k + j0, kwds)

    def connect_from_sparse(self, W, delay=None, column_access=True):
        self.connect(W=W)
        if delay is not None:
            self.set_delays(delay=delay)

    def connect_csr(self, rowptr, cols, weights, delays=None, delay_steps=None):
        """Set the whole compressed matrix at once (the role of
        connect_from_sparse, connection.py:450-475, without a scipy matrix):
        rowptr (len(source)+1), ascending cols per row, weights per synapse;
        for a DelayConnection, `delays` in seconds or `delay_steps` in bins."""
        self._check_open()
        if self._denseW is not None:
            raise ValueError("connect_csr needs structure='sparse'")
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        if len(rowptr) != len(self.source) + 1 or rowptr[-1] != len(cols):
            raise ValueError("rowptr does not match the source size / number of synapses")
        w = np.asarray(weights)
        if w.ndim == 0:
            # a scalar weight stays one value (no per-synapse array)
            self._rowptr, self._cols, self._w = rowptr, cols, None
            self._wshared = w.astype(self.dtype)[()]
        else:
            self._rowptr, self._cols, self._w = rowptr, cols, np.ascontiguousarray(w.astype(self.dtype, copy=False))
            self._wshared = None
        self._build = None
        self.iscompressed = True
        if isinstance(self, DelayConnection):
            if delay_steps is not None:
                self._dsteps = np.ascontiguousarray(delay_steps, dtype=np.uint8)
                self._dvals = None
            else:
                self._dvals = np.zeros(len(cols)) if delays is None else np.asarray(delays, dtype=float)
        elif delays is not None or delay_steps is not None:
            raise TypeError("delays need a DelayConnection")

    def _after_connect(self, P, Q, rows, cols, kwds):
        if kwds.get("delay") is not None:
            raise TypeError("delay keyword needs a DelayConnection")

    def __setitem__(self, key, value):
        i, j = key
        if self.iscompressed:
            self._set_element(int(i), int(j), float(value))
            return
        if self._denseW is not None:
            self._denseW[i, j] = value
        else:
            self._build.add(i, j, value)

    def __getitem__(self, key):
        i, j = key
        if not self.iscompressed:
            self.compress()
        w = self._weights()
        m = len(self.target)
        if self._dense is not None:
            return w.reshape(-1, m)[i, j]
        a, b = self._rowptr[i], self._rowptr[i + 1]
        k = np.searchsorted(self._cols[a:b], j)
        if k < b - a and self._cols[a + k] == j:
            return w[a + k]
        return 0.0

    def _set_element(self, i, j, x):
        w = self._weights().copy()
        m = len(self.target)
        if self._dense is not None:
            w[i * m + j] = x
        else:
            a, b = self._rowptr[i], self._rowptr[i + 1]
            k = np.searchsorted(self._cols[a:b], j)
            if not (k < b - a and self._cols[a + k] == j):
                raise NotImplementedError("inserting a synapse into a compressed matrix is not supported")
            w[a + k] = x
        self._set_weights(w)

    # ---------------------------------------------------------- compression
    def compress(self):
        if self.iscompressed:
            return
        if self._denseW is not None:
            self._dense = True
            self._w = self._denseW.reshape(-1).astype(self.dtype)
            self._denseW = None
        else:
            self._rowptr, self._cols, w = self._build.to_csr()
            self._w = w.astype(self.dtype)
            self._build = None
        self.iscompressed = True
        self._compress_extra()

    def _compress_extra(self):
        pass

    def _nnz(self):
        return len(self._cols) if self._w is None else len(self._w)

    def _host_state(self, d):
        # a shared weight stays one value; other weights may be plastic
        if self._wshared is None:
            d["_w"] = self._binding.read_weights(self).astype(self.dtype)

    def _weights(self):
        if self._binding is not None:
            self._w = self._binding.read_weights(self).astype(self.dtype)
            self._wshared = None
        elif self._w is None and self._wshared is not None:
            self._w = np.full(len(self._cols), self._wshared, dtype=self.dtype)
            self._wshared = None
        return self._w

    def _set_weights(self, w):
        self._wshared = None
        self._w = np.asarray(w).astype(self.dtype)
        if self._binding is not None:
            self._binding.write_weights(self, self._w)

    @property
    def W(self):
        self.compress()
        return ConnectionMatrixView(self)

    # ---------------------------------------------------------------- lowering
    def _lower(self, rt, gids):
        self.compress()
        src, tgt = self.source._owner, self.target._owner
        mod = -1 if self._nstate_mod is None else self._nstate_mod
        if self._dense is None and self._wshared is not None:
            return rt.conn_add_shared(gids[src], self.source._origin, len(self.source), gids[tgt],
                                      self.target._origin, len(self.target), self.nstate, self._rowptr, self._cols,
                                      self._wshared, self.dtype, delay_steps=self.delay, mod_var=mod)
        w = self._weights()
        if self._dense is not None:
            return rt.conn_add_dense(gids[src], self.source._origin, len(self.source), gids[tgt],
                                     self.target._origin, len(self.target), self.nstate,
                                     w.reshape(len(self.source), len(self.target)), self.delay, mod)
        return rt.conn_add(gids[src], self.source._origin, len(self.source), gids[tgt], self.target._origin,
                           len(self.target), self.nstate, self._rowptr, self._cols, w, delay_steps=self.delay,
                           mod_var=mod)

    def reinit(self):
        pass

    def __repr__(self):
        return "%s(%r, %r, state=%r)" % (type(self).__name__, self.source, self.target, self.nstate)


class DelayConnection(Connection):
    """Heterogeneous postsynaptic delays (delayconnection.py:17-337).

    Each synapse's delay d (seconds) becomes ``int(d / dt)`` steps, computed
    as ``int((1/dt) * d)`` like the reference (delayconnection.py:152); the
    ring has ``int(max_delay/dt) + 1`` rows (delayconnection.py:94)."""

    def __init__(self, source, target, state=0, modulation=None, structure="sparse", weight=None,
                 sparseness=None, delay=None, max_delay=5e-3, dtype=np.float64, **kwds):
        self._delay_init = True
        self._md = int(max_delay / target.clock.dt) + 1
        self._idt = 1.0 / target.clock.dt
        self._delay_ops = []
        self._d = None
        Connection.__init__(self, source, target, state=state, delay=0.0, modulation=modulation,
                            structure="sparse" if structure == "dense" else structure, weight=weight,
                            sparseness=sparseness, dtype=dtype)
        self._dense_requested = structure == "dense"
        if delay is True:
            delay = None
        if delay is not None:
            self.set_delays(delay=delay)
        if self._md > 255:
            raise NotImplementedError("max_delay of more than 254 steps is not supported")

    # delays are recorded as operations and applied to the compressed rows
    def set_delays(self, source=None, target=None, delay=None):
        if delay is None:
            return
        P = source or self.source
        Q = target or self.target
        i0, j0 = self.origin(P, Q)
        self._delay_ops.append((i0, i0 + len(P), j0, j0 + len(Q), delay))
        if self.iscompressed:
            self._apply_delay_ops()

    def connect(self, source=None, target=None, W=None, delay=None):
        """Connection.connect, then the delays of the inserted block
        (delayconnection.py:315-318)."""
        Connection.connect(self, source=source, target=target, W=W)
        if delay is not None:
            self.set_delays(source, target, delay)

    def _after_connect(self, P, Q, rows, cols, kwds):
        d = kwds.get("delay")
        if d is not None:
            self.set_delays(P, Q, d)

    def _compress_extra(self):
        self._dvals = np.zeros(len(self._cols))
        self._apply_delay_ops()

    def _apply_delay_ops(self):
        n = len(self.source)
        rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(self._rowptr))
        for (i0, i1, j0, j1, delay) in self._delay_ops:
            sel = (rows >= i0) & (rows < i1) & (self._cols >= j0) & (self._cols < j1)
            idx = np.nonzero(sel)[0]
            if isinstance(delay, (int, float, np.floating, np.integer)):
                self._dvals[idx] = float(delay)
            elif isinstance(delay, (tuple, list)) and len(delay) == 2:
                lo, hi = delay
                self._dvals[idx] = np.random.rand(len(idx)) * (hi - lo) + lo
            elif callable(delay):
                import inspect
                nargs = len(inspect.signature(delay).parameters)
                if nargs == 0:
                    self._dvals[idx] = [float(delay()) for _ in idx]
                else:
                    try:
                        self._dvals[idx] = np.asarray(delay(rows[idx] - i0, self._cols[idx].astype(np.int64) - j0),
                                                      dtype=float)
                    except Exception:
                        self._dvals[idx] = [float(delay(int(a) - i0, int(b) - j0))
                                            for a, b in zip(rows[idx], self._cols[idx])]
            else:
                D = np.asarray(delay.todense() if hasattr(delay, "todense") else delay, dtype=float)
                self._dvals[idx] = D[rows[idx] - i0, self._cols[idx] - j0]
        self._delay_ops = []

    def _delay_steps(self):
        if getattr(self, "_dvals", None) is None and getattr(self, "_dsteps", None) is not None:
            if len(self._dsteps) and int(self._dsteps.max()) >= self._md:
                raise ValueError("synaptic delay beyond max_delay")
            return self._dsteps
        steps = (self._idt * self._dvals).astype(np.int64)
        if len(steps) and (steps.min() < 0 or steps.max() >= self._md):
            raise ValueError("synaptic delay beyond max_delay")
        return steps.astype(np.uint8)

    def _delay_seconds(self):
        """Per-synapse delays in seconds, CSR order (delays given in bins
        count as bins * dt)."""
        self.compress()
        if getattr(self, "_dvals", None) is None:
            return np.asarray(self._dsteps, dtype=np.float64) * float(self.target.clock.dt)
        return np.asarray(self._dvals, dtype=np.float64)

    @property
    def delay(self):
        return _DelayView(self)

    @delay.setter
    def delay(self, value):
        self.set_delays(delay=value)

    def _lower(self, rt, gids):
        self.compress()
        src, tgt = self.source._owner, self.target._owner
        mod = -1 if self._nstate_mod is None else self._nstate_mod
        if self._wshared is not None:
            return rt.conn_add_shared(gids[src], self.source._origin, len(self.source), gids[tgt],
                                      self.target._origin, len(self.target), self.nstate, self._rowptr, self._cols,
                                      self._wshared, self.dtype, delay_steps=0, delays=self._delay_steps(),
                                      ring_depth=self._md, mod_var=mod)
        return rt.conn_add(gids[src], self.source._origin, len(self.source), gids[tgt], self.target._origin,
                           len(self.target), self.nstate, self._rowptr, self._cols, self._weights(),
                           delay_steps=0, delays=self._delay_steps(), ring_depth=self._md, mod_var=mod)


class _DelayView(object):
    """``C.delay[i, :] = values`` / ``C.delay[i, j]`` (seconds)."""

    def __init__(self, c):
        self._c = c

    def __setitem__(self, key, value):
        c = self._c
        c.compress()
        if c._binding is not None:
            raise NotImplementedError("changing delays after the first run is not supported")
        i, j = key
        n = len(c.source)
        rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(c._rowptr))
        value = np.asarray(value, dtype=float)
        if isinstance(i, (int, np.integer)) and isinstance(j, slice) and j == slice(None):
            a, b = c._rowptr[i], c._rowptr[i + 1]
            c._dvals[a:b] = value[c._cols[a:b]] if value.ndim else value
        elif isinstance(j, (int, np.integer)) and isinstance(i, slice) and i == slice(None):
            sel = np.nonzero(c._cols == j)[0]
            c._dvals[sel] = value[rows[sel]] if value.ndim else value
        else:
            a, b = c._rowptr[i], c._rowptr[i + 1]
            k = np.searchsorted(c._cols[a:b], j)
            c._dvals[a + k] = float(value)

    def __getitem__(self, key):
        c = self._c
        c.compress()
        i, j = key
        a, b = c._rowptr[i], c._rowptr[i + 1]
        if isinstance(j, slice):
            out = np.zeros(len(c.target))
            out[c._cols[a:b]] = c._dvals[a:b]
            return out
        k = np.searchsorted(c._cols[a:b], j)
        return c._dvals[a + k] if k < b - a and c._cols[a + k] == j else 0.0


class IdentityConnection(Connection):
    """One-to-one connection with a single weight (otherconnections.py)."""

    def __init__(self, source, target, state=0, weight=1.0, delay=0.0):
        Connection.__init__(self, source, target, state=state, delay=delay)
        self.connect_one_to_one(weight=weight)
