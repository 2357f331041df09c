"""Test oracle for brian_b200 (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  ``table()`` returns the CPU restatement (oracle.cpp) as a
FunctionTable with the same C ABI as the CUDA engine, so a network can be
replayed into it with ``brian_b200.network.engine(table())``.
"""
import ctypes as ct
import os

HERE = os.path.dirname(os.path.abspath(__file__))

_table = None


def table():
    global _table
    if _table is None:
        from . import build
        build.build_oracle()
        from brian_b200._lib import FunctionTable
        _table = FunctionTable(build.ORACLE_SO, "or_")
        _table.lib.or_philox_uniform.argtypes = [ct.c_uint64, ct.c_int64, ct.c_int64]
        _table.lib.or_philox_uniform.restype = ct.c_double
    return _table


def philox_uniform(seed, step, i):
    return table().lib.or_philox_uniform(seed, step, i)


def fixed_indegree_csr(n_src, n_tgt, k, seed):
    """The oracle's fixed in-degree construction (the same draws as the
    engine's bg_fixed_indegree_csr), as (rowptr int64, cols int32)."""
    import numpy as np
    lib = table().lib
    lib.or_fixed_indegree_csr.argtypes = [ct.c_int64, ct.c_int64, ct.c_int64, ct.c_uint64, ct.c_void_p, ct.c_void_p]
    lib.or_fixed_indegree_csr.restype = ct.c_int
    rowptr = np.empty(n_src + 1, dtype=np.int64)
    cols = np.empty(n_tgt * k, dtype=np.int32)
    st = lib.or_fixed_indegree_csr(n_src, n_tgt, k, int(seed) & ((1 << 64) - 1), rowptr.ctypes.data, cols.ctypes.data)
    if st != 0:
        raise ValueError("or_fixed_indegree_csr failed (%d)" % st)
    return rowptr, cols


def reference_spike_container():
    """ctypes handle to the reference's own C++ SpikeContainer (compiled from
    the reference tree into oracle/_ref), or None when it was not built."""
    from . import build
    if not os.path.exists(build.REF_SO):
        try:
            build.build_reference()
        except Exception:
            return None
    if not os.path.exists(build.REF_SO):
        return None
    lib = ct.CDLL(build.REF_SO)
    lib.ref_sc_create.restype = ct.c_void_p
    lib.ref_sc_create.argtypes = [ct.c_int]
    lib.ref_sc_destroy.argtypes = [ct.c_void_p]
    lib.ref_sc_push.argtypes = [ct.c_void_p, ct.POINTER(ct.c_long), ct.c_int]
    lib.ref_sc_get_spikes.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.POINTER(ct.c_long), ct.c_int]
    lib.ref_sc_get_spikes.restype = ct.c_int
    lib.ref_sc_getslice.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.POINTER(ct.c_long), ct.c_int]
    lib.ref_sc_getslice.restype = ct.c_int
    return lib
