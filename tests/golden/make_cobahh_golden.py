"""Build tests/golden/cobahh.npz from the reference's COBAHH regression data
(dev/tests/correctness/test_optimizations.py:10-128 and its three data
files): the excitatory and inhibitory 0/1 connection matrices (3200 x 4000
and 800 x 4000) as CSR, and the 156 843 reference spikes as (index, step)
at dt = 0.1 ms.  Run once where the reference tree is available:

    python tests/golden/make_cobahh_golden.py /path/to/reference
"""
import os
import sys

import numpy as np

DT = 1e-4


def csr(dense):
    rows, cols = np.nonzero(dense > 0)
    rowptr = np.zeros(dense.shape[0] + 1, dtype=np.int32)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), cols.astype(np.int16)


def main(ref):
    d = os.path.join(ref, "dev", "tests", "correctness")
    ce = np.loadtxt(os.path.join(d, "Ce_matrix.txt.gz"))
    ci = np.loadtxt(os.path.join(d, "Ci_matrix.txt.gz"))
    spikes = np.loadtxt(os.path.join(d, "COBAHH_spikes.txt.gz"))
    assert ce.shape == (3200, 4000) and ci.shape == (800, 4000)
    ce_rowptr, ce_cols = csr(ce)
    ci_rowptr, ci_cols = csr(ci)
    spk_i = spikes[:, 0].astype(np.int16)
    spk_step = np.rint(spikes[:, 1] / DT).astype(np.int32)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cobahh.npz")
    np.savez_compressed(out, ce_rowptr=ce_rowptr, ce_cols=ce_cols, ci_rowptr=ci_rowptr, ci_cols=ci_cols,
                        spk_i=spk_i, spk_step=spk_step)
    print(out, os.path.getsize(out), "bytes;", len(spk_i), "spikes;", len(ce_cols), "+", len(ci_cols), "synapses")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BRIAN_REFERENCE", "/root/reference"))
