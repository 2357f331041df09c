"""Reference known-answer tests on the CPU oracle (pins the oracle)."""
import pytest

import kats
from brian_b200.network import engine


@pytest.mark.parametrize("kat", kats.ALL, ids=[k.__name__ for k in kats.ALL])
def test_kat_oracle(kat, oracle_table):
    with engine(oracle_table):
        kat()
