"""COO -> CSR on the device and the beta -> COO decode (round trips)."""
import numpy as np
import pytest
import torch

import oracle
import spc5_b200 as S
from spc5_b200 import matrices as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_unsorted_coo_to_csr_then_convert(cuda, dt):
    csr = M.powerlaw(20000, seed=9).astype(dt)
    rows = np.repeat(np.arange(csr.nrows, dtype=np.int32), np.diff(csr.rowptr))
    perm = np.random.default_rng(1).permutation(csr.nnz)
    m = S.coo_matrix(csr.nrows, csr.ncols, rows[perm], csr.colidx[perm], csr.values[perm])
    assert m.format == S.FORMAT_CSR and m.numberOfNNZ == csr.nnz
    for r in (1, 4):
        mm = S.coo_matrix(csr.nrows, csr.ncols, torch.from_numpy(rows).cuda(),
                          torch.from_numpy(csr.colidx).cuda(), torch.from_numpy(csr.values).cuda(),
                          sorted=True)
        S.CSR_to_SPC5(mm, S.FORMAT_OF_R[r])
        m2 = S.coo_matrix(csr.nrows, csr.ncols, rows[perm], csr.colidx[perm], csr.values[perm])
        S.CSR_to_SPC5(m2, S.FORMAT_OF_R[r])
        ob, oh, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, csr.values)
        for mat in (mm, m2):
            b, h, v = mat.arrays()
            assert np.array_equal(b, ob) and np.array_equal(h, oh) and v.tobytes() == ov.tobytes()


def test_coo_rejects_duplicates_and_bad_rows(cuda):
    with pytest.raises(S.SPC5Error):
        S.coo_matrix(3, 3, [0, 0, 1], [1, 1, 2], np.ones(3))
    with pytest.raises(S.SPC5Error):
        S.coo_matrix(3, 3, [0, 5], [1, 1], np.ones(2))


@pytest.mark.parametrize("r", [1, 2, 4, 8])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_decode_round_trip(cuda, r, dt):
    for csr in (M.random_csr(500, 700, 0.05, seed=3, empty_row_frac=0.2), M.stencil27(8)):
        csr = csr.astype(dt)
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
        S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
        rows, cols, vals = (t.cpu().numpy() for t in S.decode_coo(m))
        b, h, v = m.arrays()
        orow, ocol, oval = oracle.beta_to_coo(r, csr.nrows, b, h, v)
        assert np.array_equal(rows, orow) and np.array_equal(cols, ocol) and vals.tobytes() == oval.tobytes()
        order = np.lexsort((cols, rows))
        assert np.array_equal(cols[order], csr.colidx) and vals[order].tobytes() == csr.values.tobytes()
