"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference (berenger-eu/spc5) ships no golden vectors, so this script runs
the reference's own code -- src/spc5.hpp compiled from its sources into
oracle/_ref/libspc5ref.so by oracle/Makefile -- on small seeded matrices and
stores its outputs:

* ``rowsSize``, ``blocksColumnIndexesWithMasks`` and ``values`` after
  ``CSR_to_SPC5`` (spc5.hpp:989-1018) for r = 1, 2, 4, 8, double and float;
* ``numberOfBlocks`` and the ``SPC5_{r}rVc_block_count`` results;
* ``y`` after one ``SPC5_Spmv`` (the AVX-512 kernels, spc5.hpp:2309-2715)
  on a zero y and a seeded x;
* ``y`` of ``CSR_Spmv_scalar`` (spc5.hpp:116-127) and ``SPC5_find_best``.

Run from the repository root (needs the reference sources):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from spc5_b200 import matrices as M  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "golden.npz")


def cases():
    """Small matrices covering the shapes the kernels branch on."""
    yield "poisson_12", M.poisson2d(12)
    yield "stencil27_5", M.stencil27(5, seed=2)
    yield "random_61x70", M.random_csr(61, 70, 0.12, seed=11, empty_row_frac=0.15)
    yield "random_dense_rows", M.random_csr(19, 40, 0.8, seed=12)
    yield "banded_97", M.banded(97, 9, 0.3, seed=13)
    yield "dense_17", M.dense(17)
    # last columns of the matrix inside a block window: col + VS > ncols
    yield "edge_cols", M.from_coo(9, 20, [0, 0, 1, 3, 3, 3, 5, 8, 8], [19, 12, 18, 0, 17, 19, 6, 3, 19],
                                  np.linspace(-1, 1, 9))
    yield "one_row", M.from_coo(1, 64, [0] * 10, [0, 1, 7, 8, 15, 16, 31, 40, 62, 63],
                                np.arange(1, 11, dtype=np.float64))
    yield "powerlaw_300", M.powerlaw(300, seed=5)


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    data = {}
    names = []
    for name, csr in cases():
        names.append(name)
        data[f"{name}/nrows"] = np.int64(csr.nrows)
        data[f"{name}/ncols"] = np.int64(csr.ncols)
        data[f"{name}/rowptr"] = csr.rowptr
        data[f"{name}/colidx"] = csr.colidx
        data[f"{name}/values"] = csr.values
        x = M.x_vector(csr.ncols, seed=7)
        data[f"{name}/x"] = x
        refm = oracle.RefMatrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
        ycsr = np.zeros(csr.nrows + 7)
        refm.csr_spmv(x, ycsr)
        data[f"{name}/y_csr"] = ycsr[: csr.nrows]
        best_r, est = refm.find_best()
        data[f"{name}/find_best_r"] = np.int64(best_r)
        data[f"{name}/find_best_est"] = np.float64(est)
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            for r in (1, 2, 4, 8):
                m = oracle.RefMatrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols)
                data[f"{name}/{tag}/r{r}/block_count"] = np.int64(m.block_count(r))
                m.convert(r)
                brptr, headers, vals = m.arrays()
                data[f"{name}/{tag}/r{r}/rowsSize"] = brptr
                data[f"{name}/{tag}/r{r}/headers"] = headers
                data[f"{name}/{tag}/r{r}/values"] = vals
                yp = np.zeros(csr.nrows + 7, dtype=dt)
                m.spmv(x.astype(dt), yp)
                data[f"{name}/{tag}/r{r}/y"] = yp[: csr.nrows]
    data["names"] = np.array(names)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes, {len(names)} matrices)")


if __name__ == "__main__":
    main()
