"""Seeded synthetic sparse matrices in CSR (int32 indices, float64 values).

The reference benchmarks SuiteSparse matrices downloaded at run time and a
dense ``v = i + j`` matrix (examples/load_mm_and_compare.cpp:431-449).  Those
files are not available offline, so the workloads here are seeded synthetic
matrices with the shapes, sizes and value distributions of the workloads this
project is measured on:

* :func:`poisson2d`   -- 5-point Laplacian on a G x G grid (diag 4, off -1)
* :func:`powerlaw`    -- power-law row lengths with diagonal-centred runs
* :func:`stencil27`   -- 27-point stencil on a G^3 grid (diag 26, neighbours
  -1 + U[-1e-3, 1e-3])
* :func:`banded`      -- banded random matrix (batched workloads)
* :func:`dense`       -- the reference driver's dense ``i + j`` matrix
* :func:`random_csr`  -- small irregular matrices for parity tests

All generators are vectorised numpy and deterministic for a given seed
(``numpy.random.Generator(PCG64(seed))``).  A Matrix Market reader
(:func:`read_matrix_market`) mirrors the reference's ``loadMM``
(examples/load_mm_and_compare.cpp:286-428): symmetric files are mirrored and
entries are sorted by (row, column).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class CSR:
    nrows: int
    ncols: int
    rowptr: np.ndarray  # int32, nrows + 1
    colidx: np.ndarray  # int32, nnz
    values: np.ndarray  # float64 (or float32), nnz
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def astype(self, dtype) -> "CSR":
        return CSR(self.nrows, self.ncols, self.rowptr, self.colidx,
                   self.values.astype(dtype), self.name)

    def to_dense(self) -> np.ndarray:
        d = np.zeros((self.nrows, self.ncols), dtype=self.values.dtype)
        rows = np.repeat(np.arange(self.nrows), np.diff(self.rowptr))
        d[rows, self.colidx] = self.values
        return d


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _from_sorted_keys(nrows: int, ncols: int, rows: np.ndarray, cols: np.ndarray,
                      values: np.ndarray, name: str) -> CSR:
    counts = np.bincount(rows, minlength=nrows).astype(np.int64)
    rowptr = np.zeros(nrows + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    if rowptr[-1] >= 2**31:
        raise ValueError("nnz does not fit int32 indices")
    return CSR(nrows, ncols, rowptr.astype(np.int32), cols.astype(np.int32, copy=False),
               np.ascontiguousarray(values), name)


def from_coo(nrows: int, ncols: int, rows, cols, values, name: str = "", sum_duplicates=False) -> CSR:
    """CSR from unsorted COO, sorting by (row, column) like COO_unsorted_to_CSR
    (src/spc5.hpp:107-114).  Duplicates are kept unless ``sum_duplicates``."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    values = np.asarray(values)
    key = rows * ncols + cols
    order = np.argsort(key, kind="stable")
    key, values = key[order], values[order]
    if sum_duplicates and len(key):
        uniq, start = np.unique(key, return_index=True)
        values = np.add.reduceat(values, start)
        key = uniq
    return _from_sorted_keys(nrows, ncols, (key // ncols).astype(np.int64), key % ncols, values, name)


# ---------------------------------------------------------------------------
# structured matrices
# ---------------------------------------------------------------------------

def poisson2d(g: int = 512) -> CSR:
    """5-point Laplacian on a g x g grid: diagonal 4.0, neighbours -1.0."""
    n = g * g
    idx = np.arange(n, dtype=np.int64)
    iy, ix = idx // g, idx % g
    offs = [(-g, iy > 0), (-1, ix > 0), (0, np.ones(n, bool)), (1, ix < g - 1), (g, iy < g - 1)]
    cols = np.stack([idx + o for o, _ in offs], axis=1)
    valid = np.stack([m for _, m in offs], axis=1)
    vals = np.where(np.arange(5)[None, :] == 2, 4.0, -1.0) * np.ones((n, 1))
    counts = valid.sum(axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    return CSR(n, n, rowptr.astype(np.int32), cols[valid].astype(np.int32), vals[valid].astype(np.float64),
               f"poisson2d_{g}")


def stencil27(g: int = 160, seed: int = 2) -> CSR:
    """27-point stencil on a g^3 grid: diagonal 26.0, neighbours -1.0 plus a
    U[-1e-3, 1e-3] perturbation drawn in storage order with ``seed``."""
    n = g ** 3
    idx = np.arange(n, dtype=np.int64)
    iz, iy, ix = idx // (g * g), (idx // g) % g, idx % g
    nnz_upper = n * 27
    cols = np.empty((n, 27), dtype=np.int32)
    valid = np.empty((n, 27), dtype=bool)
    k = 0
    for dz in (-1, 0, 1):  # ascending column order: dz, then dy, then dx
        mz = (iz + dz >= 0) & (iz + dz < g)
        for dy in (-1, 0, 1):
            mzy = mz & (iy + dy >= 0) & (iy + dy < g)
            for dx in (-1, 0, 1):
                cols[:, k] = (idx + dz * g * g + dy * g + dx).astype(np.int32)
                valid[:, k] = mzy & (ix + dx >= 0) & (ix + dx < g)
                k += 1
    del iz, iy, ix
    counts = valid.sum(axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    colidx = cols[valid]
    is_diag = np.zeros((n, 27), dtype=bool)
    is_diag[:, 13] = True
    diag = is_diag[valid]
    del cols, is_diag
    rng = _rng(seed)
    vals = -1.0 + rng.uniform(-1e-3, 1e-3, size=len(colidx))
    vals[diag] = 26.0
    assert len(colidx) <= nnz_upper
    return CSR(n, n, rowptr.astype(np.int32), colidx, vals, f"stencil27_{g}")


def dense(dim: int) -> CSR:
    """The reference driver's dense matrix, v = i + j (load_mm_and_compare.cpp:431-449)."""
    i = np.repeat(np.arange(dim, dtype=np.int64), dim)
    j = np.tile(np.arange(dim, dtype=np.int64), dim)
    rowptr = (np.arange(dim + 1, dtype=np.int64) * dim).astype(np.int32)
    return CSR(dim, dim, rowptr, j.astype(np.int32), (i + j).astype(np.float64), f"dense_{dim}")


def banded(n: int, bandwidth: int, density: float = 0.1, seed: int = 3) -> CSR:
    """Random banded matrix: each entry with |i - j| <= bandwidth is present
    with probability ``density`` (the diagonal always), values U[-1, 1]."""
    rng = _rng(seed)
    w = 2 * bandwidth + 1
    rows_out, cols_out = [], []
    chunk = max(1, (1 << 24) // w)
    for r0 in range(0, n, chunk):
        r1 = min(n, r0 + chunk)
        rr = np.arange(r0, r1, dtype=np.int64)
        off = np.arange(-bandwidth, bandwidth + 1, dtype=np.int64)
        cc = rr[:, None] + off[None, :]
        keep = (rng.random((r1 - r0, w)) < density) | (off[None, :] == 0)
        keep &= (cc >= 0) & (cc < n)
        rows_out.append(np.broadcast_to(rr[:, None], cc.shape)[keep])
        cols_out.append(cc[keep])
    rows = np.concatenate(rows_out)
    cols = np.concatenate(cols_out)
    vals = rng.uniform(-1.0, 1.0, size=len(cols))
    return _from_sorted_keys(n, n, rows, cols, vals, f"banded_{n}_{bandwidth}")


# ---------------------------------------------------------------------------
# power-law matrix
# ---------------------------------------------------------------------------

POWERLAW_SHIFT = 3  # mean row length of min(2000, Zipf(1.8) + 3) is ~15.8


def powerlaw(n: int = 4_000_000, s: float = 1.8, max_len: int = 2000, seed: int = 1,
             run_fraction: float = 0.7, run_max: int = 16, sigma_frac: float = 0.01,
             shift: int = POWERLAW_SHIFT) -> CSR:
    """Power-law matrix.

    Row length L_i = min(max_len, Z_i + shift) with Z_i ~ Zipf(s) (support
    1, 2, ...).  A plain Zipf(1.8) clipped to [1, 2000] has mean 12.8; the
    shift of 3 calibrates the mean to ~15.8 (about 63M entries at n = 4M).
    round(run_fraction * L_i) of the row's columns come in contiguous runs
    of length U[1, run_max] starting near the diagonal (start = i + round(N(0,
    sigma_frac * n)), clipped into [0, n - len]); a run is cut at the row's
    run budget.  The remaining columns are uniform on [0, n).  Duplicate
    columns inside a row are merged (the first value kept), so the realised
    nnz is slightly below sum(L_i).  Values are U[-1, 1].
    """
    rng = _rng(seed)
    z = rng.zipf(s, size=n).astype(np.int64)
    lens = np.minimum(z + shift, max_len).astype(np.int64)
    del z
    n_run = np.rint(run_fraction * lens).astype(np.int64)
    n_uni = lens - n_run
    # runs: one global stream of run lengths cut at every row boundary
    total_run = int(n_run.sum())
    n_runs_est = int(total_run / ((run_max + 1) / 2.0) * 1.05) + 1024
    run_len = rng.integers(1, run_max + 1, size=n_runs_est, dtype=np.int64)
    run_end = np.cumsum(run_len)
    while run_end[-1] < total_run:
        extra = rng.integers(1, run_max + 1, size=n_runs_est // 4 + 1024, dtype=np.int64)
        run_end = np.concatenate([run_end, run_end[-1] + np.cumsum(extra)])
    run_end = run_end[: int(np.searchsorted(run_end, total_run)) + 1]
    run_end[-1] = total_run
    row_end = np.cumsum(n_run)
    cuts = np.union1d(run_end, row_end[n_run > 0])
    seg_start = np.concatenate([[0], cuts[:-1]])
    seg_len = cuts - seg_start
    seg_row = np.searchsorted(row_end, seg_start, side="right")
    centre = seg_row + np.rint(rng.normal(0.0, sigma_frac * n, size=len(seg_start))).astype(np.int64)
    start_col = np.clip(centre, 0, n - seg_len)
    del centre, cuts
    run_rows = np.repeat(seg_row, seg_len)
    run_cols = np.repeat(start_col - seg_start, seg_len) + np.arange(total_run, dtype=np.int64)
    del seg_row, seg_len, start_col, seg_start
    uni_rows = np.repeat(np.arange(n, dtype=np.int64), n_uni)
    uni_cols = rng.integers(0, n, size=len(uni_rows), dtype=np.int64)
    rows = np.concatenate([run_rows, uni_rows])
    cols = np.concatenate([run_cols, uni_cols])
    del run_rows, run_cols, uni_rows, uni_cols
    key = rows * n + cols
    del rows, cols
    key.sort()
    keep = np.empty(len(key), dtype=bool)
    keep[0] = True
    np.not_equal(key[1:], key[:-1], out=keep[1:])
    key = key[keep]
    del keep
    vals = rng.uniform(-1.0, 1.0, size=len(key))
    rows = key // n
    cols = key - rows * n
    del key
    return _from_sorted_keys(n, n, rows, cols, vals, f"powerlaw_{n}")


# ---------------------------------------------------------------------------
# small irregular matrices for parity tests
# ---------------------------------------------------------------------------

def random_csr(nrows: int, ncols: int, density: float, seed: int, empty_row_frac: float = 0.0,
               dtype=np.float64) -> CSR:
    rng = _rng(seed)
    mask = rng.random((nrows, ncols)) < density
    if empty_row_frac > 0:
        mask[rng.random(nrows) < empty_row_frac, :] = False
    rows, cols = np.nonzero(mask)
    vals = rng.uniform(-1.0, 1.0, size=len(rows)).astype(dtype)
    return _from_sorted_keys(nrows, ncols, rows.astype(np.int64), cols.astype(np.int64), vals,
                             f"random_{nrows}x{ncols}_{density}_{seed}")


def x_vector(n: int, seed: int, dtype=np.float64) -> np.ndarray:
    """x ~ U[-1, 1] with the given seed."""
    return _rng(seed).uniform(-1.0, 1.0, size=n).astype(dtype)


# ---------------------------------------------------------------------------
# Matrix Market
# ---------------------------------------------------------------------------

def read_matrix_market(path: str) -> CSR:
    """Coordinate Matrix Market reader following loadMM
    (examples/load_mm_and_compare.cpp:286-428): 1-based indices, symmetric
    matrices mirrored (diagonal once), pattern entries get value 1.0, entries
    sorted by (row, column)."""
    with open(path) as f:
        header = f.readline().lower().split()
        if len(header) < 5 or header[0] != "%%matrixmarket" or header[2] != "coordinate":
            raise ValueError("only coordinate Matrix Market files are supported")
        field, symmetry = header[3], header[4]
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        nr, nc, nz = (int(t) for t in line.split())
        data = np.loadtxt(f, ndmin=2) if nz else np.zeros((0, 3))
    rows = data[:, 0].astype(np.int64) - 1
    cols = data[:, 1].astype(np.int64) - 1
    vals = data[:, 2].astype(np.float64) if field != "pattern" else np.ones(len(rows))
    if symmetry in ("symmetric", "skew-symmetric", "hermitian"):
        off = rows != cols
        sign = -1.0 if symmetry == "skew-symmetric" else 1.0
        rows, cols, vals = (np.concatenate([rows, cols[off]]), np.concatenate([cols, rows[off]]),
                            np.concatenate([vals, sign * vals[off]]))
    return from_coo(nr, nc, rows, cols, vals, name=path)
