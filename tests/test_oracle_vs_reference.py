"""Pin the oracle restatement against the reference compiled from its sources.

oracle/_ref/libspc5ref.so is src/spc5.hpp itself behind a C shim
(oracle/ref_shim.cpp, oracle/Makefile).  On random and structured matrices
the restatement must give identical converted arrays and bit-identical
AVX-512 SpMV results.
"""
import numpy as np
import pytest

import oracle
from spc5_b200 import matrices as M

pytestmark = pytest.mark.skipif(not (oracle.ref_available() and oracle.cpu_has_avx512()),
                                reason="reference library not built or CPU without AVX-512")


def cases():
    for seed in range(5):
        yield M.random_csr(40 + 17 * seed, 33 + 11 * seed, 0.1 + 0.05 * seed, seed, empty_row_frac=0.1)
    yield M.powerlaw(2000, seed=3)
    yield M.stencil27(7)
    yield M.banded(500, 40, 0.1, seed=4)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_restatement_matches_reference(dt, r):
    for csr in cases():
        vals = csr.values.astype(dt)
        ref = oracle.RefMatrix(csr.rowptr, csr.colidx, vals, csr.ncols)
        nb = ref.block_count(r)
        assert nb == oracle.block_count(r, csr.rowptr, csr.colidx, dt)
        ref.convert(r)
        rb, rh, rv = ref.arrays()
        ob, oh, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, vals)
        assert np.array_equal(rb, ob) and np.array_equal(rh, oh) and rv.tobytes() == ov.tobytes()
        x = M.x_vector(csr.ncols, 21, dt)
        yr = np.zeros(csr.nrows + 7, dtype=dt)
        ref.spmv(x, yr)
        yo = np.zeros(csr.nrows, dtype=dt)
        (oracle.beta_spmv_f64 if dt == np.float64 else oracle.beta_spmv_f32)(r, csr.nrows, ob, oh, ov, x, yo)
        assert yr[: csr.nrows].tobytes() == yo.tobytes()


def test_omp_path_equals_sequential():
    csr = M.powerlaw(5000, seed=9)
    x = oracle.x_padded(M.x_vector(csr.ncols, 1))
    for r in (1, 2, 4, 8):
        ref = oracle.RefMatrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
        ref.convert(r)
        y1 = np.zeros(csr.nrows + 7)
        ref.spmv(x[: csr.ncols], y1)
        ref.split(3)
        y2 = np.zeros(csr.nrows + 7)
        ref.time_spmv_omp(x, y2, 1)
        assert y1[: csr.nrows].tobytes() == y2[: csr.nrows].tobytes()
