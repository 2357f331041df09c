"""Golden vectors from the reference tree (tests/golden/cuba_reference.json,
made by tests/golden/make_golden.py) and published known-answer vectors."""
import json
import os

import numpy as np
import pytest

import brian_b200 as b
from brian_b200 import ms, mV
from brian_b200.equations import linear_propagator
from brian_b200.network import engine

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cuba_reference.json")))


def test_cuba_propagator_matches_reference_cpp_constants():
    """A = expm(M dt), C = -A.B + B against the constants the reference's C++
    benchmark hard-codes (8 significant digits)."""
    eqs = b.Equations("dv/dt=(ge+gi-(v-El))/taum : volt\ndge/dt=-ge/taue : volt\ndgi/dt=-gi/taui : volt",
                      taum=20 * ms, taue=5 * ms, taui=10 * ms, El=-49 * mV)
    A, C = linear_propagator(eqs, 0.1 * ms)
    g = GOLDEN["cuba_propagator"]
    At = np.array(g["A_transposed"])
    np.testing.assert_allclose(A.T, At, rtol=0, atol=5e-9)
    np.testing.assert_allclose(C * 1e3, g["C_mV"], rtol=0, atol=5e-9)
    # and the exact values of scipy.linalg.expm on this host
    assert A[0, 0] == 0.9950124791926823 and A[1, 1] == 0.9801986733067553


def test_cuba_benchmark_spike_count_in_reference_range(oracle_table):
    """The reference's CUBA benchmark (N=4000, p=80/N, refractory 5 ms, 2.5 s):
    the oracle's spike count falls within the spread of the reference's own
    recorded runs (C++ and Brian), widened by 5%."""
    import scenarios
    counts = GOLDEN["cuba_benchmark_spike_counts"]
    ref = counts["cpp"]["4000"] + counts["brian_compile_nounits"]["4000"]
    with engine(oracle_table):
        r = scenarios.cuba(N=4000, steps=25000, refractory=5 * ms, seed=4)
    n = len(r["spk0.idx"])
    assert 0.95 * min(ref) <= n <= 1.05 * max(ref), (n, min(ref), max(ref))


@pytest.mark.parametrize("ctr,key,out", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(ctr, key, out):
    """Philox4x32-10 (Salmon et al., SC'11) against the Random123 known-answer
    vectors; the uniform draw of PoissonGroup is built from its output."""
    import oracle
    # uniform(seed, step, i) packs (step, i) into the counter and seed into the key
    step = ctr[0] | (ctr[1] << 32)
    i = ctr[2] | (ctr[3] << 32)
    seed = key[0] | (key[1] << 32)
    u = oracle.philox_uniform(seed, step, i)
    a, bb = out[0] >> 5, out[1] >> 6
    assert u == (a * 67108864 + bb) / 9007199254740992.0
