"""The reference's testfeatures/test_connect.py:5-66 restated: delay
matrices of a DelayConnection built with connect / connect_random /
connect_full / connect_one_to_one over subgroups, delays given as a value,
a (min, max) range, a function of no argument and a function of (i, j)
relative to the subgroups' origins."""
import numpy as np
import pytest

import brian_b200 as b

FULL = np.array([[1, 1, 2, 2],
                 [1, 1, 2, 2],
                 [4, 4, 0, 10],
                 [4, 4, 1, 11]])
DIAG = np.array([[1, 0, 2, 0],
                 [0, 1, 0, 2],
                 [4, 0, 0, 0],
                 [0, 4, 0, 11]])


def _delay_matrix(C):
    return np.array([np.asarray(C.delay[i, :]) for i in range(4)])


@pytest.mark.parametrize("structure", ["dense", "sparse", "dynamic"])
@pytest.mark.parametrize("method", ["connect", "connect_random", "connect_full", "connect_one_to_one"])
def test_delay_connect_with_subgroups(structure, method):
    b.clear()
    G = b.NeuronGroup(4, model="V:1")
    C = b.Connection(G, G, "V", delay=True, structure=structure)
    blocks = [((0, 2), (0, 2), 1), ((0, 2), (2, 4), (2.1, 2.2)), ((2, 4), (0, 2), lambda: 4),
              ((2, 4), (2, 4), lambda i, j: i + 10 * j)]
    for (a, bb), (c, d), delay in blocks:
        P, Q = G[a:bb], G[c:d]
        if method == "connect":
            C.connect(P, Q, W=np.ones((2, 2)), delay=delay)
        elif method == "connect_random":
            C.connect_random(P, Q, p=1, weight=1, delay=delay)
        elif method == "connect_full":
            C.connect_full(P, Q, weight=1, delay=delay)
        else:
            C.connect_one_to_one(P, Q, weight=1, delay=delay)
    want = DIAG if method == "connect_one_to_one" else FULL
    np.testing.assert_array_equal(np.array(_delay_matrix(C), dtype=int), want)
