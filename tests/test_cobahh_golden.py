"""The reference's COBAHH regression (dev/tests/correctness/
test_optimizations.py:10-128): 4000 Hodgkin-Huxley neurons integrated by
exponential Euler for 1 s, EmpiricalThreshold, fixed connectivity; its 156 843
recorded spikes (tests/golden/cobahh.npz, made by make_cobahh_golden.py) are
matched exactly -- step and index of every spike -- by the oracle (the
generated model compiled by gcc, glibc exp) and by the GPU engine (the same
model compiled by NVRTC, CUDA exp)."""
import numpy as np
import pytest

import scenarios
import brian_b200 as b
from brian_b200.network import engine


def _check(r):
    assert len(r["golden_idx"]) == 156843
    assert np.array_equal(r["steps"], r["golden_steps"])
    assert np.array_equal(r["idx"], r["golden_idx"])


def test_oracle_reproduces_cobahh_golden():
    import oracle
    b.clear()
    b.reinit_default_clock()
    with engine(oracle.table()):
        r = scenarios.cobahh(10000)
    _check(r)


@pytest.mark.gpu
def test_gpu_reproduces_cobahh_golden(gpu_table):
    b.clear()
    b.reinit_default_clock()
    r = scenarios.cobahh(10000)
    _check(r)
