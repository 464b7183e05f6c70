"""Invariants of the seeded synthetic matrix generators (host logic)."""
import numpy as np

from spc5_b200 import matrices as M


def check_csr(a):
    assert a.rowptr[0] == 0 and a.rowptr[-1] == len(a.colidx) == len(a.values)
    assert np.all(np.diff(a.rowptr) >= 0)
    assert a.colidx.min(initial=0) >= 0 and a.colidx.max(initial=-1) < a.ncols
    rows = np.repeat(np.arange(a.nrows), np.diff(a.rowptr))
    key = rows.astype(np.int64) * a.ncols + a.colidx
    assert np.all(np.diff(key) > 0), "columns must be strictly increasing inside rows"


def test_poisson_sizes():
    a = M.poisson2d(512)
    check_csr(a)
    assert a.nrows == 262144 and a.nnz == 1308672
    assert set(np.unique(a.values)) == {-1.0, 4.0}


def test_stencil27_small():
    a = M.stencil27(6)
    check_csr(a)
    assert a.nnz == (3 * 6 - 2) ** 3  # (3g-2)^3 entries; g = 160 gives 109,215,352
    d = a.to_dense()
    assert np.all(np.diag(d) == 26.0)
    off = d[(d != 0) & ~np.eye(a.nrows, dtype=bool)]
    assert np.all(np.abs(off + 1.0) <= 1e-3)


def test_powerlaw_shape():
    a = M.powerlaw(20000, seed=1)
    check_csr(a)
    lens = np.diff(a.rowptr)
    assert lens.min() >= 1 and lens.max() <= 2000
    assert 10 < lens.mean() < 20
    assert np.all(np.abs(a.values) <= 1.0)


def test_powerlaw_deterministic():
    a, b = M.powerlaw(5000, seed=4), M.powerlaw(5000, seed=4)
    assert np.array_equal(a.colidx, b.colidx) and np.array_equal(a.values, b.values)


def test_banded_and_dense():
    a = M.banded(300, 7, 0.1, seed=3)
    check_csr(a)
    rows = np.repeat(np.arange(a.nrows), np.diff(a.rowptr))
    assert np.all(np.abs(rows - a.colidx) <= 7)
    d = M.dense(9)
    check_csr(d)
    assert d.to_dense()[3, 5] == 8.0


def test_matrix_market_round_trip(tmp_path):
    p = tmp_path / "m.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n% c\n4 4 4\n1 1 2.0\n3 1 -1.5\n"
                 "4 2 0.5\n4 4 1.0\n")
    a = M.read_matrix_market(str(p))
    check_csr(a)
    d = a.to_dense()
    assert d[2, 0] == -1.5 and d[0, 2] == -1.5 and d[3, 1] == 0.5 and d[1, 3] == 0.5 and a.nnz == 6
