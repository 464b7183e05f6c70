"""The oracle restatement against the golden fixtures made by the reference.

tests/golden/golden.npz holds outputs of the reference's own code
(src/spc5.hpp compiled from its sources; tests/golden/make_golden.py):
converted arrays, block counts, AVX-512 SpMV results, CSR SpMV results and
the format-selection model.  The restatement in oracle/spc5_oracle.c must
reproduce the integer/byte arrays exactly and the kernel results bit for bit.
"""
import numpy as np
import pytest

import oracle

DTYPES = [("f64", np.float64), ("f32", np.float32)]


def names(golden):
    return [str(n) for n in golden["names"]]


def test_golden_has_cases(golden):
    assert len(names(golden)) >= 8


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_conversion_bit_exact(golden, tag, dt, r):
    for n in names(golden):
        rp, ci = golden[f"{n}/rowptr"], golden[f"{n}/colidx"]
        vals = golden[f"{n}/values"].astype(dt)
        brptr, headers, v = oracle.csr_to_beta(r, rp, ci, vals)
        assert np.array_equal(brptr, golden[f"{n}/{tag}/r{r}/rowsSize"]), n
        assert np.array_equal(headers, golden[f"{n}/{tag}/r{r}/headers"]), n
        assert v.tobytes() == golden[f"{n}/{tag}/r{r}/values"].tobytes(), n
        assert oracle.block_count(r, rp, ci, dt) == int(golden[f"{n}/{tag}/r{r}/block_count"]), n


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_spmv_bit_exact(golden, tag, dt, r):
    for n in names(golden):
        nrows = int(golden[f"{n}/nrows"])
        x = golden[f"{n}/x"].astype(dt)
        y = np.zeros(nrows, dtype=dt)
        f = oracle.beta_spmv_f64 if dt == np.float64 else oracle.beta_spmv_f32
        f(r, nrows, golden[f"{n}/{tag}/r{r}/rowsSize"], golden[f"{n}/{tag}/r{r}/headers"],
          golden[f"{n}/{tag}/r{r}/values"], x, y)
        assert y.tobytes() == golden[f"{n}/{tag}/r{r}/y"].tobytes(), n


def test_csr_spmv_close(golden):
    for n in names(golden):
        nrows = int(golden[f"{n}/nrows"])
        y = np.zeros(nrows)
        y, absrow = oracle.csr_spmv_f64(golden[f"{n}/rowptr"], golden[f"{n}/colidx"],
                                        golden[f"{n}/values"], golden[f"{n}/x"], y)
        err = np.abs(y - golden[f"{n}/y_csr"]) / np.maximum(absrow, 1e-300)
        assert err.max(initial=0.0) <= 1e-14, n


def test_find_best_matches_reference(golden):
    for n in names(golden):
        rp, ci = golden[f"{n}/rowptr"], golden[f"{n}/colidx"]
        blocks = [int(golden[f"{n}/f64/r{r}/block_count"]) for r in (1, 2, 4)]
        r, est = oracle.find_best(True, int(rp[-1]), blocks)
        assert r == int(golden[f"{n}/find_best_r"]), n
        assert est == pytest.approx(float(golden[f"{n}/find_best_est"]), rel=1e-15), n


@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_decode_round_trip(golden, r):
    for n in names(golden):
        nrows = int(golden[f"{n}/nrows"])
        rows, cols, vals = oracle.beta_to_coo(r, nrows, golden[f"{n}/f64/r{r}/rowsSize"],
                                              golden[f"{n}/f64/r{r}/headers"],
                                              golden[f"{n}/f64/r{r}/values"])
        order = np.lexsort((cols, rows))
        rp = oracle.coo_sorted_to_csr(nrows, rows[order])
        assert np.array_equal(rp, golden[f"{n}/rowptr"]), n
        assert np.array_equal(cols[order], golden[f"{n}/colidx"]), n
        assert np.array_equal(vals[order], golden[f"{n}/values"]), n


def test_threadsplit_covers_rows(golden):
    for n in names(golden):
        nrows = int(golden[f"{n}/nrows"])
        for r in (1, 2, 4, 8):
            start, cnt, voff = oracle.threadsplit(r, nrows, golden[f"{n}/f64/r{r}/rowsSize"],
                                                  golden[f"{n}/f64/r{r}/headers"], 4)
            assert start[0] == 0 and int((start + cnt)[cnt > 0].max(initial=0)) <= nrows
            assert cnt.sum() == nrows
            assert np.all(np.diff(voff) >= 0) and voff[-1] <= len(golden[f"{n}/values"])
