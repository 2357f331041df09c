"""Reference known-answer tests on the CUDA engine."""
import pytest

import kats


@pytest.mark.gpu
@pytest.mark.parametrize("kat", kats.ALL, ids=[k.__name__ for k in kats.ALL])
def test_kat_gpu(kat, gpu_table):
    kat()
