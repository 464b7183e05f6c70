"""The chain form of the FP64 SpMV, on the CPU.

The CUDA path runs the largest block-rows of irregular matrices as one
multiply-add chain per (sub-row, column): the values of the blocks whose
mask has that bit, in block order, evaluated from +0.0, then the reduce tree
over a sub-row's chains.  The oracle's restatement of that regrouping
(oracle_beta_spmv_f64_chains) must equal its restatement of the reference's
kernel order (oracle_beta_spmv_f64, pinned to the reference itself) bit for
bit for finite x: this checks, on the host, that the regrouping changes no
rounding.
"""
import numpy as np
import pytest

import oracle
from spc5_b200 import matrices as M


def cases():
    yield M.powerlaw(20000, seed=7)
    yield M.random_csr(1000, 1200, 0.02, seed=1, empty_row_frac=0.2)
    yield M.random_csr(333, 64, 0.5, seed=2)
    yield M.banded(4099, 150, 0.1, seed=8)
    yield M.stencil27(9)
    yield M.dense(200)
    yield M.from_coo(5, 3, [0, 2, 4], [2, 0, 1], [1.5, -2.0, 3.25])
    yield M.from_coo(7, 7, [], [], [])


@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_chains_equal_the_kernel_order(r):
    for k, csr in enumerate(cases()):
        brptr, headers, vals = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, csr.values)
        x = M.x_vector(csr.ncols, 40 + k)
        y0 = M.x_vector(csr.nrows, 60 + k)
        want = oracle.beta_spmv_f64(r, csr.nrows, brptr, headers, vals, x, y0.copy())
        got = oracle.beta_spmv_f64_chains(r, csr.nrows, brptr, headers, vals, x, y0.copy())
        assert got.tobytes() == want.tobytes(), (csr.name, r)
