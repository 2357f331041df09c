import sys, os
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine library")


@pytest.fixture(scope="session")
def oracle_table():
    import oracle
    return oracle.table()


@pytest.fixture(scope="session")
def gpu_table():
    from brian_b200._lib import product_table
    return product_table()


@pytest.fixture(autouse=True)
def _fresh_clock():
    from brian_b200 import reinit_default_clock, clear, define_default_clock
    define_default_clock(0.1e-3)
    reinit_default_clock()
    clear()
    yield
    clear()
