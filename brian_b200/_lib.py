"""ctypes binding of the C ABI in include/brian_b200.h.

`Runtime` wraps one network handle of a library that exports the bg_net
function table.  The product library is ``libbrian_b200.so`` (CUDA, sm_100a);
loading fails loudly when it is missing or no CUDA device is present -- there
is no CPU path in the product.
"""
import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbrian_b200.so")

_i32, _i64, _dbl, _u64, _vp = ct.c_int32, ct.c_int64, ct.c_double, ct.c_uint64, ct.c_void_p
_P = ct.POINTER

# name -> (argtypes) ; every function returns int32 status
SIGNATURES = {
    "version": [],
    "last_error": [ct.c_char_p, _i64],
    "net_create": [ct.c_int, ct.c_int, ct.c_int, _dbl, _P(_vp)],
    "net_destroy": [_vp],
    "group_add": [_vp, _i64, ct.c_int, _vp, _P(_i32)],
    "group_set_linear": [_vp, _i32, _vp, _vp],
    "group_set_threshold": [_vp, _i32, ct.c_int, ct.c_int, _dbl, ct.c_int],
    "group_set_poisson": [_vp, _i32, ct.c_int, _u64],
    "group_set_generator": [_vp, _i32, _i64, _vp, _vp],
    "group_set_reset": [_vp, _i32, ct.c_int, ct.c_int, _dbl, ct.c_int],
    "group_set_refractory": [_vp, _i32, _dbl, _i32, ct.c_int, _dbl],
    "group_set_empirical": [_vp, _i32, _i32],
    "group_set_model": [_vp, _i32, _vp],
    "group_set_timed_array": [_vp, _i32, ct.c_int, _i64, _i64, _vp, _i64, _i64, ct.c_int, _dbl, _dbl, _i64, _vp],
    "conn_add": [_vp, _i32, _i64, _i64, _i32, _i64, _i64, ct.c_int, _i64, _vp, _vp, _vp, ct.c_int,
                 _i32, _vp, _i32, ct.c_int, _P(_i32)],
    "conn_add_dense": [_vp, _i32, _i64, _i64, _i32, _i64, _i64, ct.c_int, _vp, ct.c_int, _i32, ct.c_int,
                       _P(_i32)],
    "conn_get_weights": [_vp, _i32, _vp],
    "conn_set_weights": [_vp, _i32, _vp],
    "stdp_add": [_vp, _i32, _vp, _dbl, _dbl, _dbl, _dbl, ct.c_int, _i32, _i32, _P(_i32)],
    "synapses_add": [_vp, _i32, _i64, _i64, _i32, _i64, _i64, _i64, _vp, _vp, _vp, ct.c_int, _vp, _vp, _vp,
                     _P(_i32)],
    "synapses_set_terms": [_vp, _i32, _vp],
    "synapses_set_code": [_vp, _i32, _i32, _vp, ct.c_char_p, ct.c_char_p, _i32, _vp, _i32, _vp, _i32, _vp],
    "synapses_get_var": [_vp, _i32, _i32, _vp],
    "synapses_set_var": [_vp, _i32, _i32, _vp],
    "stdp_set_update": [_vp, _i32, ct.c_int, ct.c_int, _dbl],
    "stdp_add_delayed": [_vp, _i32, _vp, _dbl, _dbl, _dbl, _dbl, ct.c_int, _i32, _i32, _vp, _vp, _P(_i32)],
    "stdp_get_traces": [_vp, _i32, _vp, _vp],
    "spikemon_add": [_vp, _i32, _i64, _i64, _i32, _P(_i32)],
    "statemon_add": [_vp, _i32, ct.c_int, _i64, _vp, _i32, _P(_i32)],
    "spikemon_count": [_vp, _i32, _P(_i64)],
    "spikemon_read": [_vp, _i32, _vp, _vp, _i64, _P(_i64)],
    "statemon_count": [_vp, _i32, _P(_i64)],
    "statemon_read": [_vp, _i32, _vp, _vp, _i64, _P(_i64)],
    "monitor_clear": [_vp, _i32],
    "net_prepare": [_vp],
    "net_run": [_vp, _i64, _i64],
    "group_get_state": [_vp, _i32, ct.c_int, _vp],
    "group_set_state": [_vp, _i32, ct.c_int, _vp],
    "net_reinit": [_vp],
    "net_stats": [_vp, _P(_i64), _P(_i64), _P(_dbl)],
    "net_counters": [_vp, _vp, _vp],
    "net_state_bytes": [_vp, _P(_i64)],
    "net_save_state": [_vp, ct.c_char_p, _i64, _P(_i64)],
    "net_load_state": [_vp, ct.c_char_p, _i64],
    "net_save": [_vp, ct.c_char_p],
    "net_load": [_vp, ct.c_char_p],
}

# entry points of the CUDA engine only
ENGINE_ONLY = {
    "net_profile": [_vp, _i64, _i64, _vp, _i64, _P(_i64)],
    "net_item_name": [_vp, _i64, ct.c_char_p, _i64],
    "fixed_indegree_csr": [_i64, _i64, _i64, _u64, _vp, _vp],
    "net_set_persistent": [_vp, ct.c_int],
    "conn_add_shared": [_vp, _i32, _i64, _i64, _i32, _i64, _i64, ct.c_int, _i64, _vp, _vp, _dbl, ct.c_int, _i32,
                        _vp, _i32, ct.c_int, _P(_i32)],
    "net_persistent_threads": [_vp, _P(_i32)],
    "net_set_spin_limit": [_vp, _i64],
    "net_set_synapse_events": [_vp, ct.c_int],
    "import_device_ptr": [_vp, _vp, _i64, ct.c_int, _P(_i32)],
    "group_use_buffer": [_vp, _i32, _i32],
    "group_padded_size": [_vp, _i32, _P(_i64)],
    "net_debug_hold_arrival": [_vp, _i32],
    "net_set_check_finite": [_vp, ct.c_int],
    "fit_compile_check": [ct.c_int, _vp, _dbl, ct.c_int, ct.c_int, ct.c_char_p, _i64],
    "fit_create": [_P(_vp), ct.c_int, ct.c_int, _vp, _dbl, ct.c_int, ct.c_int],
    "fit_destroy": [_vp],
    "fit_set_input": [_vp, _vp, _i64],
    "fit_set_targets": [_vp, _vp, _i64],
    "fit_set_sims": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32],
    "fit_set_record": [_vp, _i32],
    "fit_reinit": [_vp],
    "fit_run": [_vp, _i32, _i32],
    "fit_read": [_vp, _vp, _vp, _vp],
    "fit_read_spikes": [_vp, _vp, _vp],
    "fit_set_gamma": [_vp, _i64, _i32, _vp, _vp, _dbl],
    "fit_set_params": [_vp, _i32, _vp],
    "fit_evaluate": [_vp, _vp, _vp],
    "fit_features": [_vp, _vp],
    "fit_train_features": [_vp, _i64, _vp, _vp, _vp, _vp, _P(ct.c_float)],
    "mlp_last_forward_ms": [_vp, _P(ct.c_float)],
    "spike_features": [ct.c_int, _i64, _vp, _vp, _vp, _vp, _i64, _dbl, _vp],
    "fit_set_blocks_per_sm": [_vp, _i32],
    "mlp_create": [_P(_vp), ct.c_int, ct.c_int],
    "mlp_destroy": [_vp],
    "mlp_set_params": [_vp, ct.c_int, _vp, _vp],
    "mlp_get_params": [_vp, ct.c_int, _vp, _vp],
    "mlp_forward": [_vp, _vp, _i64, _vp],
    "mlp_set_data": [_vp, _vp, _vp, _i64],
    "mlp_train": [_vp, ct.c_int, ct.c_int, ct.c_float, _u64, _vp, _P(ct.c_float)],
    "mlp_gradients": [_vp, ct.c_int, _P(ct.c_float), _vp, _vp],
    "mlp_epoch_order": [_vp, _u64, _i64],
    "mlp_step_gradients": [_vp, ct.c_int, _i64, _P(ct.c_float), _P(_vp), _P(_i64)],
    "mlp_apply_gradients": [_vp, _vp, ct.c_float, ct.c_float],
    "gemm_bf16": [_i64, _i64, _i64, _vp, _vp, _vp, _vp],
    "fit_autotune": [_vp, _vp, _P(_i32), _vp],
    "fit_pso_init": [_vp, _i32, _vp, _vp, _vp, _dbl, _dbl, _dbl, _u64],
    "fit_pso_evaluate_initial": [_vp],
    "fit_pso_run": [_vp, _i32, _vp, _vp],
    "fit_pso_best": [_vp, _vp, _vp],
    "fit_pso_state": [_vp, _vp, _vp, _vp, _vp],
    "fit_stats": [_vp, _vp, ct.c_int],
    "batch_create": [_vp, _i32, _P(_vp)],
    "batch_free": [_vp],
    "batch_run": [_vp, _vp, _vp],
    "batch_set_shape": [_vp, _i32, _i32],
    "batch_get_shape": [_vp, _P(_i32), _P(_i32), _P(_i32), _P(_i32)],
    "batch_autotune": [_vp, _i32, _P(_dbl)],
    "batch_stats": [_vp, _P(_i64), _P(_dbl)],
}


class EngineError(RuntimeError):
    """An engine call failed; `code` is its BG_* status (BG_EINVAL -1,
    BG_ENOMEM -2, BG_ECUDA -3, BG_ETIMEOUT -4, BG_ENUMERIC -5, BG_ESTATE -6,
    BG_ENOSYS -7, BG_ECOMPILE -8)."""

    def __init__(self, msg, code=None):
        RuntimeError.__init__(self, msg)
        self.code = code


class EngineBound(object):
    """Objects that a Network lowers onto an engine handle.  They pickle
    without the handle: `_host_state(d)` puts the values the engine holds
    (states, plastic weights, traces, monitor records) into the pickled dict
    `d`, leaving the live object as it is."""

    def _host_state(self, d):
        pass

    def __getstate__(self):
        d = dict(self.__dict__)
        if d.get("_binding") is not None:
            self._host_state(d)
        d["_binding"] = None
        return d

    def __setstate__(self, d):
        self.__dict__.update(d)


class FunctionTable(object):
    """Typed view of one library's entry points under a name prefix."""

    def __init__(self, path, prefix, signatures=SIGNATURES):
        if not os.path.exists(path):
            raise EngineError("engine library not found: %s (run `python -m brian_b200.build`)" % path)
        self.path = path
        self.prefix = prefix
        self.lib = ct.CDLL(path)
        for name, args in signatures.items():
            fn = getattr(self.lib, prefix + name)
            fn.argtypes = args
            fn.restype = ct.c_int
            setattr(self, name, fn)

    def check(self, status, what):
        if status != 0:
            buf = ct.create_string_buffer(1024)
            self.last_error(buf, 1024)
            raise EngineError("%s failed (%d): %s" % (what, status, buf.value.decode(errors="replace")), status)


_product = None


def product_table():
    """The CUDA engine (libbrian_b200.so).  Raises if it cannot be loaded."""
    global _product
    if _product is None:
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build()
        _product = FunctionTable(LIB_PATH, "bg_", dict(SIGNATURES, **ENGINE_ONLY))
    return _product


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p) if a is not None else None


class Runtime(object):
    """One network handle on a function table."""

    def __init__(self, table=None, device=0, precision=64, deterministic=True, dt=1e-4, persistent=True,
                 spin_limit=None, check_finite=False, synapse_events=None):
        self.t = table if table is not None else product_table()
        self.h = ct.c_void_p()
        self.precision = precision
        self.t.check(self.t.net_create(device, precision, 1 if deterministic else 0, float(dt),
                                       ct.byref(self.h)), "net_create")
        if persistent is not True and hasattr(self.t, "net_set_persistent"):
            self.t.check(self.t.net_set_persistent(self.h, int(persistent)), "net_set_persistent")
        if spin_limit is not None and hasattr(self.t, "net_set_spin_limit"):
            self.t.check(self.t.net_set_spin_limit(self.h, int(spin_limit)), "net_set_spin_limit")
        if check_finite and hasattr(self.t, "net_set_check_finite"):
            self.t.check(self.t.net_set_check_finite(self.h, 1), "net_set_check_finite")
        if synapse_events is not None and hasattr(self.t, "net_set_synapse_events"):
            self.t.check(self.t.net_set_synapse_events(self.h, 1 if synapse_events else 2), "net_set_synapse_events")

    def import_device_ptr(self, ptr, nbytes, precision):
        bid = _i32()
        self._c(self.t.import_device_ptr(self.h, ct.c_void_p(int(ptr)), int(nbytes), 0 if precision == 64 else 1,
                                         ct.byref(bid)), "import_device_ptr")
        return bid.value

    def group_use_buffer(self, gid, bid):
        self._c(self.t.group_use_buffer(self.h, gid, bid), "group_use_buffer")

    def group_padded_size(self, gid):
        n = _i64()
        self._c(self.t.group_padded_size(self.h, gid, ct.byref(n)), "group_padded_size")
        return n.value

    def save_state(self):
        """The network's dynamic state as bytes (bg_net_save_state)."""
        n = _i64()
        self._c(self.t.net_state_bytes(self.h, ct.byref(n)), "net_state_bytes")
        buf = ct.create_string_buffer(max(1, n.value))
        w = _i64()
        self._c(self.t.net_save_state(self.h, buf, n.value, ct.byref(w)), "net_save_state")
        return buf.raw[:w.value]

    def load_state(self, data):
        """Load bytes from save_state into this (identically built) network."""
        data = bytes(data)
        self._c(self.t.net_load_state(self.h, data, len(data)), "net_load_state")

    def debug_hold_arrival(self, block):
        """Test hook of the bounded waits: persistent block `block` never
        publishes its step arrivals (set before prepare)."""
        self.t.check(self.t.net_debug_hold_arrival(self.h, int(block)), "net_debug_hold_arrival")

    def close(self):
        if self.h:
            self.t.net_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st, what):
        self.t.check(st, what)

    # ------------------------------------------------------------ building
    def group_add(self, S0):
        S0 = np.ascontiguousarray(S0, dtype=np.float64)
        nvar, n = S0.shape
        gid = _i32()
        self._c(self.t.group_add(self.h, n, nvar, _ptr(S0), ct.byref(gid)), "group_add")
        self._ng = max(getattr(self, "_ng", 0), gid.value + 1)
        return gid.value

    def group_set_linear(self, gid, A, C):
        A = np.ascontiguousarray(A, dtype=np.float64)
        C = None if C is None else np.ascontiguousarray(C, dtype=np.float64)
        self._c(self.t.group_set_linear(self.h, gid, _ptr(A), _ptr(C)), "group_set_linear")

    def group_set_timed_array(self, gid, var, origin, count, values, mode, t_init, adt, first_step, bp):
        values = np.ascontiguousarray(values, dtype=np.float64)
        bp = None if bp is None or len(bp) == 0 else np.ascontiguousarray(bp, dtype=np.int64)
        self._c(self.t.group_set_timed_array(self.h, gid, int(var), int(origin), int(count), _ptr(values),
                                             values.shape[0], values.shape[1], int(mode), float(t_init), float(adt),
                                             int(first_step), _ptr(bp)), "group_set_timed_array")

    def group_set_threshold(self, gid, kind, var=0, value=0.0, var2=0):
        self._c(self.t.group_set_threshold(self.h, gid, kind, var, float(value), var2), "group_set_threshold")

    def group_set_poisson(self, gid, rate_var, seed):
        self._c(self.t.group_set_poisson(self.h, gid, rate_var, int(seed) & ((1 << 64) - 1)),
                "group_set_poisson")

    def group_set_generator(self, gid, steps, idx):
        steps = np.ascontiguousarray(steps, dtype=np.int64)
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        self._c(self.t.group_set_generator(self.h, gid, len(steps), _ptr(steps), _ptr(idx)),
                "group_set_generator")

    def group_set_reset(self, gid, kind, var=0, value=0.0, var2=0):
        self._c(self.t.group_set_reset(self.h, gid, kind, var, float(value), var2), "group_set_reset")

    def group_set_refractory(self, gid, refractory_time, period, var, value):
        self._c(self.t.group_set_refractory(self.h, gid, float(refractory_time), int(period), var,
                                            float(value)), "group_set_refractory")

    def group_set_empirical(self, gid, steps):
        self._c(self.t.group_set_empirical(self.h, gid, int(steps)), "group_set_empirical")

    def group_set_model(self, gid, code, update=True, threshold=True, reset=True):
        """Generated C of the group's model (codegen.ModelCode); the parts
        left out keep the built-in linear update / threshold / reset."""
        def b(x, keep):
            return (x or "").encode() if keep else b""
        m = FitModel(b(",".join(code.state), True), b(code.update, update), b"", b(code.threshold, threshold),
                     b(code.reset, reset), b"", b"")
        self._model_refs = getattr(self, "_model_refs", []) + [m]
        self._c(self.t.group_set_model(self.h, gid, ct.byref(m)), "group_set_model")

    def conn_add(self, src, so, sn, tgt, to, tn, var, rowptr, cols, w, delay_steps=0, delays=None,
                 ring_depth=0, mod_var=-1):
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        w = np.ascontiguousarray(w)
        if w.dtype not in (np.float32, np.float64):
            w = w.astype(np.float64)
        wbits = 32 if w.dtype == np.float32 else 64
        d = None if delays is None else np.ascontiguousarray(delays, dtype=np.uint8)
        cid = _i32()
        self._c(self.t.conn_add(self.h, src, so, sn, tgt, to, tn, var, len(cols), _ptr(rowptr), _ptr(cols),
                                _ptr(w), wbits, int(delay_steps), _ptr(d), int(ring_depth), int(mod_var),
                                ct.byref(cid)), "conn_add")
        self._nc = max(getattr(self, "_nc", 0), cid.value + 1)
        return cid.value

    def conn_add_shared(self, src, so, sn, tgt, to, tn, var, rowptr, cols, weight, dtype, delay_steps=0,
                        delays=None, ring_depth=0, mod_var=-1):
        """conn_add for synapses that all carry `weight` (stored as `dtype`):
        no weight array crosses the boundary.  Tables without the entry
        point get the full array."""
        if not hasattr(self.t, "conn_add_shared"):
            return self.conn_add(src, so, sn, tgt, to, tn, var, rowptr, cols,
                                 np.full(len(cols), weight, dtype=dtype), delay_steps, delays, ring_depth, mod_var)
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        wbits = 32 if np.dtype(dtype) == np.float32 else 64
        d = None if delays is None else np.ascontiguousarray(delays, dtype=np.uint8)
        cid = _i32()
        self._c(self.t.conn_add_shared(self.h, src, so, sn, tgt, to, tn, var, len(cols), _ptr(rowptr), _ptr(cols),
                                       float(weight), wbits, int(delay_steps), _ptr(d), int(ring_depth),
                                       int(mod_var), ct.byref(cid)), "conn_add_shared")
        self._nc = max(getattr(self, "_nc", 0), cid.value + 1)
        return cid.value

    def conn_add_dense(self, src, so, sn, tgt, to, tn, var, W, delay_steps=0, mod_var=-1):
        W = np.ascontiguousarray(W)
        if W.dtype not in (np.float32, np.float64):
            W = W.astype(np.float64)
        wbits = 32 if W.dtype == np.float32 else 64
        cid = _i32()
        self._c(self.t.conn_add_dense(self.h, src, so, sn, tgt, to, tn, var, _ptr(W), wbits, int(delay_steps),
                                      int(mod_var), ct.byref(cid)), "conn_add_dense")
        self._nc = max(getattr(self, "_nc", 0), cid.value + 1)
        return cid.value

    def conn_get_weights(self, cid, count):
        out = np.empty(count, dtype=np.float64)
        self._c(self.t.conn_get_weights(self.h, cid, _ptr(out)), "conn_get_weights")
        return out

    def conn_set_weights(self, cid, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        self._c(self.t.conn_set_weights(self.h, cid, _ptr(w)), "conn_set_weights")

    def stdp_add(self, cid, decay, Ap, Am, wmin, wmax, interactions, pre_delay, post_delay):
        decay = np.ascontiguousarray(decay, dtype=np.float64)
        sid = _i32()
        self._c(self.t.stdp_add(self.h, cid, _ptr(decay), float(Ap), float(Am), float(wmin), float(wmax),
                                int(interactions), int(pre_delay), int(post_delay), ct.byref(sid)), "stdp_add")
        return sid.value

    def stdp_add_delayed(self, cid, decay, Ap, Am, wmin, wmax, interactions, pre_delay, hist_len, lag_pre, lag_post):
        decay = np.ascontiguousarray(decay, dtype=np.float64)
        lag_pre = np.ascontiguousarray(lag_pre, dtype=np.uint8)
        lag_post = np.ascontiguousarray(lag_post, dtype=np.uint8)
        sid = _i32()
        self._c(self.t.stdp_add_delayed(self.h, cid, _ptr(decay), float(Ap), float(Am), float(wmin), float(wmax),
                                        int(interactions), int(pre_delay), int(hist_len), _ptr(lag_pre),
                                        _ptr(lag_post), ct.byref(sid)), "stdp_add_delayed")
        return sid.value

    def synapses_add(self, src_gid, src_origin, src_n, tgt_gid, tgt_origin, tgt_n, pre, post, delay, op_var, op_sub,
                     terms):
        pre = np.ascontiguousarray(pre, dtype=np.int32)
        post = np.ascontiguousarray(post, dtype=np.int32)
        delay = np.ascontiguousarray(delay, dtype=np.int32)
        op_var = np.ascontiguousarray(op_var, dtype=np.int32)
        op_sub = np.ascontiguousarray(op_sub, dtype=np.int32)
        terms = np.ascontiguousarray(terms, dtype=np.float64)
        sid = _i32()
        self._c(self.t.synapses_add(self.h, src_gid, src_origin, src_n, tgt_gid, tgt_origin, tgt_n, len(pre),
                                    _ptr(pre), _ptr(post), _ptr(delay), len(op_var), _ptr(op_var), _ptr(op_sub),
                                    _ptr(terms), ct.byref(sid)), "synapses_add")
        return sid.value

    def synapses_set_code(self, yid, sv, pre_code, post_code, slot_var, writes, pre_var):
        sv = np.ascontiguousarray(sv, dtype=np.float64)
        a = lambda v: np.ascontiguousarray(v, dtype=np.int32) if len(v) else None
        sl, wr, pv = a(slot_var), a(writes), a(pre_var)
        self._c(self.t.synapses_set_code(self.h, int(yid), int(sv.shape[0]), _ptr(sv) if sv.size else None,
                                         pre_code.encode(), post_code.encode(), len(slot_var), _ptr(sl), len(writes),
                                         _ptr(wr), len(pre_var), _ptr(pv)), "synapses_set_code")

    def synapses_get_var(self, yid, k, n):
        out = np.empty(n, dtype=np.float64)
        self._c(self.t.synapses_get_var(self.h, int(yid), int(k), _ptr(out)), "synapses_get_var")
        return out

    def synapses_set_var(self, yid, k, values):
        values = np.ascontiguousarray(values, dtype=np.float64)
        self._c(self.t.synapses_set_var(self.h, int(yid), int(k), _ptr(values)), "synapses_set_var")

    def synapses_set_terms(self, sid, terms):
        terms = np.ascontiguousarray(terms, dtype=np.float64)
        self._c(self.t.synapses_set_terms(self.h, sid, _ptr(terms)), "synapses_set_terms")

    def stdp_set_update(self, sid, pre_mode, post_mode, wmax_exact):
        self._c(self.t.stdp_set_update(self.h, sid, int(pre_mode), int(post_mode), float(wmax_exact)),
                "stdp_set_update")

    def stdp_get_traces(self, sid, npre, npost):
        a = np.empty(npre)
        b = np.empty(npost)
        self._c(self.t.stdp_get_traces(self.h, sid, _ptr(a), _ptr(b)), "stdp_get_traces")
        return a, b

    def spikemon_add(self, gid, origin, n, delay=0):
        mid = _i32()
        self._c(self.t.spikemon_add(self.h, gid, origin, n, delay, ct.byref(mid)), "spikemon_add")
        return mid.value

    def statemon_add(self, gid, var, idx, timestep=1):
        idx = None if idx is None else np.ascontiguousarray(idx, dtype=np.int32)
        mid = _i32()
        self._c(self.t.statemon_add(self.h, gid, var, 0 if idx is None else len(idx), _ptr(idx), timestep,
                                    ct.byref(mid)), "statemon_add")
        return mid.value

    def spikemon_count(self, mid):
        n = _i64()
        self._c(self.t.spikemon_count(self.h, mid, ct.byref(n)), "spikemon_count")
        return n.value

    def statemon_count(self, mid):
        n = _i64()
        self._c(self.t.statemon_count(self.h, mid, ct.byref(n)), "statemon_count")
        return n.value

    def spikemon_read(self, mid):
        n = _i64()
        self._c(self.t.spikemon_count(self.h, mid, ct.byref(n)), "spikemon_count")
        steps = np.empty(n.value, dtype=np.int64)
        idx = np.empty(n.value, dtype=np.int32)
        got = _i64()
        self._c(self.t.spikemon_read(self.h, mid, _ptr(steps), _ptr(idx), n.value, ct.byref(got)), "spikemon_read")
        return steps[:got.value], idx[:got.value]

    def statemon_read(self, mid, width):
        n = _i64()
        self._c(self.t.statemon_count(self.h, mid, ct.byref(n)), "statemon_count")
        vals = np.empty((n.value, width), dtype=np.float64)
        steps = np.empty(n.value, dtype=np.int64)
        got = _i64()
        self._c(self.t.statemon_read(self.h, mid, _ptr(vals), _ptr(steps), n.value, ct.byref(got)),
                "statemon_read")
        return steps[:got.value], vals[:got.value]

    def monitor_clear(self, mid):
        self._c(self.t.monitor_clear(self.h, mid), "monitor_clear")

    # ------------------------------------------------------------- running
    def prepare(self):
        self._c(self.t.net_prepare(self.h), "net_prepare")

    def run(self, nsteps, clock_step0):
        self._c(self.t.net_run(self.h, int(nsteps), int(clock_step0)), "net_run")

    def get_state(self, gid, var, n):
        out = np.empty(n, dtype=np.float64)
        self._c(self.t.group_get_state(self.h, gid, var, _ptr(out)), "group_get_state")
        return out

    def set_state(self, gid, var, values):
        values = np.ascontiguousarray(values, dtype=np.float64)
        self._c(self.t.group_set_state(self.h, gid, var, _ptr(values)), "group_set_state")

    def reinit(self):
        self._c(self.t.net_reinit(self.h), "net_reinit")

    def counters(self, ngroups, nconns):
        # the engine writes one entry per group and per connection it holds
        g = np.zeros(max(1, ngroups, getattr(self, "_ng", 0)), dtype=np.int64)
        c = np.zeros(max(1, nconns, getattr(self, "_nc", 0)), dtype=np.int64)
        self._c(self.t.net_counters(self.h, _ptr(g), _ptr(c)), "net_counters")
        return g[:ngroups], c[:nconns]

    def profile(self, nsteps, clock_step0):
        # mean device ms of each launch of a step, with the launch names
        cap = 256
        ms = np.zeros(cap)
        n = _i64()
        self._c(self.t.net_profile(self.h, int(nsteps), int(clock_step0), _ptr(ms), cap, ct.byref(n)), "net_profile")
        out = []
        buf = ct.create_string_buffer(128)
        for i in range(n.value):
            self._c(self.t.net_item_name(self.h, i, buf, 128), "net_item_name")
            out.append((buf.value.decode(), float(ms[i])))
        return out

    def stats(self):
        s, l, ms = _i64(), _i64(), _dbl()
        self._c(self.t.net_stats(self.h, ct.byref(s), ct.byref(l), ct.byref(ms)), "net_stats")
        out = {"steps": s.value, "launches": l.value, "last_run_ms": ms.value}
        if hasattr(self.t, "net_persistent_threads"):
            th = _i32()
            self._c(self.t.net_persistent_threads(self.h, ct.byref(th)), "net_persistent_threads")
            out["persistent_threads"] = th.value
        return out


def fixed_indegree_csr_native(n_src, n_tgt, k, seed):
    """Native construction of a fixed in-degree connectivity (see
    include/brian_b200.h bg_fixed_indegree_csr)."""
    t = product_table()
    rowptr = np.empty(n_src + 1, dtype=np.int64)
    cols = np.empty(n_tgt * k, dtype=np.int32)
    t.check(t.fixed_indegree_csr(n_src, n_tgt, k, int(seed) & ((1 << 64) - 1), _ptr(rowptr), _ptr(cols)),
            "fixed_indegree_csr")
    return rowptr, cols


class FitModel(ct.Structure):
    """bg_fit_model: the generated model code handed to the fitting kernel."""
    _fields_ = [("state_names", ct.c_char_p), ("update_code", ct.c_char_p), ("update_fast_code", ct.c_char_p),
                ("threshold_code", ct.c_char_p), ("reset_code", ct.c_char_p), ("aux_decl", ct.c_char_p),
                ("setup_code", ct.c_char_p)]

    @classmethod
    def of(cls, code):
        def b(x):
            return (x or "").encode()
        m = cls(b(",".join(code.state)), b(code.update), b(getattr(code, "update_fast", "")), b(code.threshold),
                b(code.reset), b(getattr(code, "aux_decl", "")), b(getattr(code, "setup", "")))
        return m


class FitHandle(object):
    """One batched-fitting handle (bg_fit_* in include/brian_b200.h)."""

    def __init__(self, code, dt, delta_steps, exclusive=True, precision=64, device=0, table=None):
        self.t = table if table is not None else product_table()
        self.h = ct.c_void_p()
        self.code = code
        self.nstate = len(code.state)
        self.precision = precision
        self._model = FitModel.of(code)
        self.t.check(self.t.fit_create(ct.byref(self.h), int(device), int(precision), ct.byref(self._model),
                                       float(dt), int(delta_steps), 1 if exclusive else 0), "fit_create")
        self.ns = 0
        self.rec_cap = 0

    def close(self):
        if self.h:
            self.t.fit_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st, what):
        self.t.check(st, what)

    def set_input(self, I):
        I = np.ascontiguousarray(I, dtype=np.float64)
        self._c(self.t.fit_set_input(self.h, _ptr(I), len(I)), "fit_set_input")

    def set_targets(self, spiketimes_steps):
        s = np.ascontiguousarray(spiketimes_steps, dtype=np.int32)
        self._c(self.t.fit_set_targets(self.h, _ptr(s), len(s)), "fit_set_targets")

    def set_sims(self, S0, I_offset, nsteps, spk_offset, spk_end, delay=None, refractory=None, onset=0):
        S0 = np.ascontiguousarray(S0, dtype=np.float64)
        ns = S0.shape[1]
        a = [np.ascontiguousarray(I_offset, dtype=np.int64), np.ascontiguousarray(nsteps, dtype=np.int32),
             np.ascontiguousarray(spk_offset, dtype=np.int64), np.ascontiguousarray(spk_end, dtype=np.int64)]
        d = None if delay is None else np.ascontiguousarray(delay, dtype=np.int32)
        r = None if refractory is None else np.ascontiguousarray(refractory, dtype=np.int32)
        for x in a + [d, r]:
            if x is not None and len(x) != ns:
                raise ValueError("per-simulation arrays must have %d entries" % ns)
        self._c(self.t.fit_set_sims(self.h, ns, _ptr(S0), _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(a[3]), _ptr(d),
                                    _ptr(r), int(onset)), "fit_set_sims")
        self.ns = ns

    def set_record(self, cap):
        self._c(self.t.fit_set_record(self.h, int(cap)), "fit_set_record")
        self.rec_cap = int(cap)

    def reinit(self):
        self._c(self.t.fit_reinit(self.h), "fit_reinit")

    def run(self, Tstart, Tend):
        self._c(self.t.fit_run(self.h, int(Tstart), int(Tend)), "fit_run")

    def read(self, state=False):
        c = np.empty(self.ns, dtype=np.int32)
        n = np.empty(self.ns, dtype=np.int32)
        S = np.empty((self.nstate, self.ns)) if state else None
        self._c(self.t.fit_read(self.h, _ptr(c), _ptr(n), _ptr(S)), "fit_read")
        return (c, n, S) if state else (c, n)

    def read_spikes(self):
        counts = np.empty(self.ns, dtype=np.int32)
        steps = np.empty((self.ns, max(1, self.rec_cap)), dtype=np.int32)
        self._c(self.t.fit_read_spikes(self.h, _ptr(counts), _ptr(steps)), "fit_read_spikes")
        return counts, steps

    def set_gamma(self, nparticles, slices, target_length, target_rate, delta):
        tl = np.ascontiguousarray(target_length, dtype=np.int32)
        tr = np.ascontiguousarray(target_rate, dtype=np.float64)
        self._c(self.t.fit_set_gamma(self.h, int(nparticles), int(slices), _ptr(tl), _ptr(tr), float(delta)),
                "fit_set_gamma")
        self.npart = int(nparticles)

    def set_params(self, dim_var):
        dv = np.ascontiguousarray(dim_var, dtype=np.int32)
        self._c(self.t.fit_set_params(self.h, len(dv), _ptr(dv)), "fit_set_params")
        self.ndim = len(dv)

    def evaluate(self, X):
        X = np.ascontiguousarray(X, dtype=np.float64)
        out = np.empty(self.npart)
        self._c(self.t.fit_evaluate(self.h, _ptr(X), _ptr(out)), "fit_evaluate")
        return out

    def features(self):
        out = np.empty((self.ns, 64), dtype=np.float32)
        self._c(self.t.fit_features(self.h, _ptr(out)), "fit_features")
        return out

    def train_features(self, trains_steps, I_offset):
        """Features of given trains (clock steps) whose inputs start at
        I_offset in this handle's input; returns (features, device ms)."""
        steps = np.concatenate([np.asarray(x, dtype=np.int32) for x in trains_steps]) if len(trains_steps) else \
            np.zeros(0, np.int32)
        if len(steps) == 0:
            steps = np.zeros(1, np.int32)
        offs = np.concatenate([[0], np.cumsum([len(x) for x in trains_steps])]).astype(np.int64)
        ioff = np.ascontiguousarray(I_offset, dtype=np.int64)
        out = np.empty((len(trains_steps), 64), dtype=np.float32)
        ms = ct.c_float()
        self._c(self.t.fit_train_features(self.h, len(trains_steps), _ptr(steps), _ptr(offs), _ptr(ioff), _ptr(out),
                                          ct.byref(ms)), "fit_train_features")
        return out, ms.value

    def set_blocks_per_sm(self, b):
        self._c(self.t.fit_set_blocks_per_sm(self.h, int(b)), "fit_set_blocks_per_sm")

    def autotune(self, X=None):
        """Fastest launch shape for a full run (results do not depend on it);
        returns (blocks per SM, ms per candidate)."""
        X = None if X is None else np.ascontiguousarray(X, dtype=np.float64)
        b = _i32()
        ms = np.zeros(6, dtype=np.float32)
        self._c(self.t.fit_autotune(self.h, _ptr(X), ct.byref(b), _ptr(ms)), "fit_autotune")
        return b.value, ms

    def pso_init(self, group_size, X0, xmin, xmax, omega, c1, c2, seed):
        X0 = np.ascontiguousarray(X0, dtype=np.float64)
        lo = np.ascontiguousarray(xmin, dtype=np.float64)
        hi = np.ascontiguousarray(xmax, dtype=np.float64)
        self._c(self.t.fit_pso_init(self.h, int(group_size), _ptr(X0), _ptr(lo), _ptr(hi), float(omega), float(c1),
                                    float(c2), int(seed) & ((1 << 64) - 1)), "fit_pso_init")
        self.ngroups = self.npart // int(group_size)

    def pso_evaluate_initial(self):
        self._c(self.t.fit_pso_evaluate_initial(self.h), "fit_pso_evaluate_initial")

    def pso_run(self, iterations, trace=True, timing=True):
        tr = np.empty((iterations, self.ngroups)) if trace else None
        ms = np.empty(iterations, dtype=np.float32) if timing else None
        self._c(self.t.fit_pso_run(self.h, int(iterations), _ptr(tr), _ptr(ms)), "fit_pso_run")
        return tr, ms

    def pso_best(self):
        X = np.empty((self.ndim, self.ngroups))
        f = np.empty(self.ngroups)
        self._c(self.t.fit_pso_best(self.h, _ptr(X), _ptr(f)), "fit_pso_best")
        return X, f

    def pso_state(self):
        X = np.empty((self.ndim, self.npart))
        V = np.empty_like(X)
        Xl = np.empty_like(X)
        fl = np.empty(self.npart)
        self._c(self.t.fit_pso_state(self.h, _ptr(X), _ptr(V), _ptr(Xl), _ptr(fl)), "fit_pso_state")
        return X, V, Xl, fl

    def stats(self):
        out = np.zeros(5)
        self._c(self.t.fit_stats(self.h, _ptr(out), 5), "fit_stats")
        return {"last_sim_ms": out[0], "sim_launches": int(out[1]), "neuron_steps": int(out[2]),
                "max_steps": int(out[3]), "last_eval_ms": out[4]}


def fit_compile_check(code, dt, delta_steps, exclusive=True, precision=64):
    """Compile a model's fitting kernel with NVRTC without a device; returns
    the compiler log, raises EngineError on failure."""
    t = product_table()
    log = ct.create_string_buffer(1 << 16)
    model = FitModel.of(code)
    t.check(t.fit_compile_check(int(precision), ct.byref(model), float(dt), int(delta_steps),
                                1 if exclusive else 0, log, 1 << 16), "fit_compile_check")
    return log.value.decode(errors="replace")


MLP_ROWS = (512, 512, 512, 64)
MLP_COLS = (64, 512, 512, 512)


class DeviceVector(object):
    """A float32 vector in device memory owned by an engine handle, exposed
    through __cuda_array_interface__ (torch.as_tensor(v, device="cuda")
    gives a view of it, e.g. for an all-reduce)."""

    def __init__(self, ptr, n, device=0):
        self.ptr, self.n, self.device = int(ptr), int(n), int(device)

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.n,), "typestr": "<f4", "data": (self.ptr, False), "version": 3, "strides": None}

    def torch(self):
        import torch
        return torch.as_tensor(self, device="cuda:%d" % self.device)


class MLPHandle(object):
    """The proposal network (bg_mlp_* in include/brian_b200.h)."""

    def __init__(self, ydim=5, device=0, table=None):
        self.t = table if table is not None else product_table()
        self.h = ct.c_void_p()
        self.ydim = ydim
        self.device = int(device)
        self.rows = 0
        self.t.check(self.t.mlp_create(ct.byref(self.h), int(device), int(ydim)), "mlp_create")

    def close(self):
        if self.h:
            self.t.mlp_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st, what):
        self.t.check(st, what)

    def set_params(self, layer, W, b):
        W = np.ascontiguousarray(W, dtype=np.float32)
        b = np.ascontiguousarray(b, dtype=np.float32)
        assert W.shape == (MLP_ROWS[layer], MLP_COLS[layer]) and b.shape == (MLP_ROWS[layer],)
        self._c(self.t.mlp_set_params(self.h, int(layer), _ptr(W), _ptr(b)), "mlp_set_params")

    def get_params(self, layer):
        W = np.empty((MLP_ROWS[layer], MLP_COLS[layer]), dtype=np.float32)
        b = np.empty(MLP_ROWS[layer], dtype=np.float32)
        self._c(self.t.mlp_get_params(self.h, int(layer), _ptr(W), _ptr(b)), "mlp_get_params")
        return W, b

    def forward(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.empty((len(X), 2 * self.ydim), dtype=np.float32)
        self._c(self.t.mlp_forward(self.h, _ptr(X), len(X), _ptr(out)), "mlp_forward")
        return out

    def last_forward_ms(self):
        ms = ct.c_float()
        self._c(self.t.mlp_last_forward_ms(self.h, ct.byref(ms)), "mlp_last_forward_ms")
        return ms.value

    def set_data(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        self._c(self.t.mlp_set_data(self.h, _ptr(X), _ptr(Y), len(X)), "mlp_set_data")
        self.rows = len(X)

    # ---- data-parallel steps (bg_mlp_epoch_order / step_gradients / apply_gradients)
    def epoch_order(self, seed, epoch):
        self._c(self.t.mlp_epoch_order(self.h, int(seed) & ((1 << 64) - 1), int(epoch)), "mlp_epoch_order")

    def step_gradients(self, batch, row0):
        """Mean loss of rows [row0, row0+batch) of the epoch order and the
        flat gradient, a DeviceVector into the handle."""
        loss, p, n = ct.c_float(), _vp(), _i64()
        self._c(self.t.mlp_step_gradients(self.h, int(batch), int(row0), ct.byref(loss), ct.byref(p), ct.byref(n)),
                "mlp_step_gradients")
        return loss.value, DeviceVector(p.value, n.value, self.device)

    def apply_gradients(self, grad, lr, scale=1.0):
        ptr = grad.ptr if isinstance(grad, DeviceVector) else int(grad)
        self._c(self.t.mlp_apply_gradients(self.h, ct.c_void_p(ptr), float(lr), float(scale)), "mlp_apply_gradients")

    def train(self, epochs, batch, lr, seed):
        loss = np.zeros(max(1, epochs), dtype=np.float32)
        ms = ct.c_float()
        self._c(self.t.mlp_train(self.h, int(epochs), int(batch), float(lr), int(seed) & ((1 << 64) - 1),
                                 _ptr(loss), ct.byref(ms)), "mlp_train")
        return loss[:epochs], ms.value

    def gradients(self, batch):
        dW = [np.zeros((MLP_ROWS[l], MLP_COLS[l]), dtype=np.float32) for l in range(4)]
        db = [np.zeros(MLP_ROWS[l], dtype=np.float32) for l in range(4)]
        pW = (ct.c_void_p * 4)(*[_ptr(x).value for x in dW])
        pb = (ct.c_void_p * 4)(*[_ptr(x).value for x in db])
        loss = ct.c_float()
        self._c(self.t.mlp_gradients(self.h, int(batch), ct.byref(loss), pW, pb), "mlp_gradients")
        return loss.value, dW, db


def spike_features(trains_steps, inputs, dt, device=0):
    """Features of given trains (lists of clock steps) with their inputs."""
    t = product_table()
    steps = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.int32) for x in trains_steps])
                                 if len(trains_steps) else np.zeros(0, np.int32), dtype=np.int32)
    offs = np.concatenate([[0], np.cumsum([len(x) for x in trains_steps])]).astype(np.int64)
    I = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64) for x in inputs]))
    ioff = np.concatenate([[0], np.cumsum([len(x) for x in inputs])[:-1]]).astype(np.int64)
    out = np.empty((len(trains_steps), 64), dtype=np.float32)
    if len(steps) == 0:
        steps = np.zeros(1, np.int32)
    t.check(t.spike_features(int(device), len(trains_steps), _ptr(steps), _ptr(offs), _ptr(I), _ptr(ioff), len(I),
                             float(dt), _ptr(out)), "spike_features")
    return out


class BatchRuntime(object):
    """One bg_batch handle over the engine handles of several Runtimes."""

    def __init__(self, runtimes):
        self.t = runtimes[0].t
        if not hasattr(self.t, "batch_create"):
            raise EngineError("batches need the CUDA engine")
        self.runtimes = list(runtimes)            # the handles must outlive the batch
        hs = (_vp * len(runtimes))(*[r.h.value for r in runtimes])
        self.h = ct.c_void_p()
        self.t.check(self.t.batch_create(hs, len(runtimes), ct.byref(self.h)), "batch_create")

    def run(self, nsteps, cs0):
        nsteps = np.ascontiguousarray(nsteps, dtype=np.int64)
        cs0 = np.ascontiguousarray(cs0, dtype=np.int64)
        self.t.check(self.t.batch_run(self.h, _ptr(nsteps), _ptr(cs0)), "batch_run")

    def set_shape(self, shape, lanes):
        self.t.check(self.t.batch_set_shape(self.h, int(shape), int(lanes)), "batch_set_shape")

    def shape(self):
        v = [_i32() for _ in range(4)]
        self.t.check(self.t.batch_get_shape(self.h, *[ct.byref(x) for x in v]), "batch_get_shape")
        return dict(shape=v[0].value, threads=v[1].value, neurons_per_thread=v[2].value, lanes=v[3].value)

    def autotune(self, steps):
        ms = _dbl()
        self.t.check(self.t.batch_autotune(self.h, int(steps), ct.byref(ms)), "batch_autotune")
        return ms.value

    def stats(self):
        n, ms = _i64(), _dbl()
        self.t.check(self.t.batch_stats(self.h, ct.byref(n), ct.byref(ms)), "batch_stats")
        return {"launches": n.value, "last_run_ms": ms.value}

    def close(self):
        if self.h:
            self.t.batch_free(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
