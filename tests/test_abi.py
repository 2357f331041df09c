"""The C ABI: every function declared in include/*.h is exported by the
engine library (and, under the or_ prefix, by the oracle)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:BG_API\s+)?(?:int|double|void)\s+\**(bg_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared()
    assert "bg_net_create" in names and "bg_net_run" in names
    assert len(names) >= 30


def test_engine_library_exports_all():
    from brian_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_exports_network_abi():
    import oracle
    from brian_b200._lib import SIGNATURES
    lib = oracle.table().lib
    missing = ["or_" + n for n in SIGNATURES if not hasattr(lib, "or_" + n)]
    assert not missing, missing


def test_product_table_has_typed_signatures():
    from brian_b200._lib import SIGNATURES
    names = set("bg_" + n for n in SIGNATURES)
    assert names <= set(declared())


def test_oracle_fixed_indegree_equals_engine_builder():
    """The oracle's construction draws the same connectivity as the engine's
    host-side bg_fixed_indegree_csr (so the CPU baseline can build the
    benchmark network without the engine library)."""
    import numpy as np
    import oracle
    from brian_b200._lib import fixed_indegree_csr_native
    for n_src, n_tgt, k, seed in ((2000, 3000, 160, 7), (500, 777, 500, 11), (10, 5, 0, 3)):
        r1, c1 = oracle.fixed_indegree_csr(n_src, n_tgt, k, seed)
        r2, c2 = fixed_indegree_csr_native(n_src, n_tgt, k, seed)
        assert np.array_equal(r1, r2) and np.array_equal(c1, c2)
        assert r1[-1] == n_tgt * k
        # every target exactly k distinct sources
        src = np.repeat(np.arange(n_src), np.diff(r1))
        if k:
            assert np.all(np.bincount(c1, minlength=n_tgt) == k)
            assert len(np.unique(src.astype(np.int64) * n_tgt + c1)) == len(c1)
