"""CPU oracle for the SPC5 beta(r,VS) hot path -- TEST INFRASTRUCTURE ONLY.

Two checkers live here, both loaded with ctypes over numpy arrays:

* ``liboracle.so`` -- ``spc5_oracle.c``, a plain-C restatement of the
  reference's conversion, block counter, kernels, CSR SpMV and speed model
  (each function cites the ``src/spc5.hpp`` lines it restates).
* ``_ref/libspc5ref.so`` -- the reference header itself (``src/spc5.hpp``),
  compiled from its own sources by ``oracle/Makefile`` behind
  ``ref_shim.cpp``.  It pins the restatement and is the timed CPU baseline.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product package ``spc5_b200``
never does: it has no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libspc5ref.so")

_P = C.c_void_p
_I = C.c_int
_L = C.c_long
_D = C.c_double


def ref_src() -> str:
    """The reference's ``src/`` directory: ``$REF_SRC``, else the default of
    oracle/Makefile (the one place that names it)."""
    env = os.environ.get("REF_SRC")
    if env:
        return env
    out = subprocess.run(["make", "-s", "-C", HERE, "print-ref-src"], capture_output=True, text=True)
    return out.stdout.strip()


def build(ref: bool = True) -> None:
    """Compile liboracle.so, and _ref/libspc5ref.so when the reference sources exist."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    src = ref_src()
    if ref and src and os.path.exists(os.path.join(src, "spc5.hpp")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={src}"], check=True)


def _ptr(a):
    return a.ctypes.data_as(_P) if a is not None else None


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        l = C.CDLL(ORACLE_SO)
        l.oracle_csr_to_beta.restype = _L
        l.oracle_csr_to_beta.argtypes = [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P]
        l.oracle_block_count.restype = _L
        l.oracle_block_count.argtypes = [_I, _I, _I, _P, _P]
        l.oracle_blockrow_counts.restype = None
        l.oracle_blockrow_counts.argtypes = [_I, _I, _I, _P, _P, _P]
        l.oracle_beta_spmv_f64_chains.restype = _I
        l.oracle_beta_spmv_f64_chains.argtypes = [_I, _I, _P, _P, _P, _P, _P]
        for name in ("oracle_beta_spmv_f64", "oracle_beta_spmv_f32", "oracle_beta_spmv_mixed"):
            f = getattr(l, name)
            f.restype = None
            f.argtypes = [_I, _I, _P, _P, _P, _P, _P]
        l.oracle_beta_spmm_f64.restype = None
        l.oracle_beta_spmm_f64.argtypes = [_I, _I, _P, _P, _P, _I, _P, _L, _P, _L]
        l.oracle_csr_spmv_f64.restype = None
        l.oracle_csr_spmv_f64.argtypes = [_I, _P, _P, _P, _P, _P, _P]
        l.oracle_beta_to_coo.restype = _L
        l.oracle_beta_to_coo.argtypes = [_I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P]
        l.oracle_coo_sorted_to_csr.restype = None
        l.oracle_coo_sorted_to_csr.argtypes = [_I, _L, _P, _P]
        l.oracle_find_best.restype = _I
        l.oracle_find_best.argtypes = [_I, _L, _P, _P]
        l.oracle_threadsplit.restype = None
        l.oracle_threadsplit.argtypes = [_I, _I, _I, _I, _P, _P, _I, _P, _P, _P]
        _lib = l
    return _lib


def layout(dtype):
    """(VS, mask bytes, value bytes) of the reference layout for a value dtype."""
    dt = np.dtype(dtype)
    if dt == np.float64:
        return 8, 1, 8
    if dt == np.float32:
        return 16, 2, 4
    raise ValueError(f"unsupported dtype {dt}")


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def block_count(r, rowptr, colidx, dtype=np.float64) -> int:
    vs, _, _ = layout(dtype)
    rowptr, colidx = _i32(rowptr), _i32(colidx)
    return int(lib().oracle_block_count(r, vs, len(rowptr) - 1, _ptr(rowptr), _ptr(colidx)))


def blockrow_counts(r, rowptr, colidx, dtype=np.float64):
    vs, _, _ = layout(dtype)
    rowptr, colidx = _i32(rowptr), _i32(colidx)
    n = len(rowptr) - 1
    out = np.zeros((n + r - 1) // r, dtype=np.int32)
    lib().oracle_blockrow_counts(r, vs, n, _ptr(rowptr), _ptr(colidx), _ptr(out))
    return out


def csr_to_beta(r, rowptr, colidx, values):
    """Convert CSR to beta(r,VS); returns (blockrowptr, headers uint8, values)."""
    values = np.ascontiguousarray(values)
    vs, mb, vb = layout(values.dtype)
    rowptr, colidx = _i32(rowptr), _i32(colidx)
    n = len(rowptr) - 1
    nb = block_count(r, rowptr, colidx, values.dtype)
    brptr = np.zeros((n + r - 1) // r + 1, dtype=np.int32)
    headers = np.zeros(nb * (4 + r * mb), dtype=np.uint8)
    out_vals = np.zeros(len(values), dtype=values.dtype)
    got = lib().oracle_csr_to_beta(r, vs, mb, vb, n, _ptr(rowptr), _ptr(colidx), _ptr(values),
                                   _ptr(brptr), _ptr(headers), _ptr(out_vals))
    assert got == nb
    return brptr, headers, out_vals


def x_padded(x, pad=15):
    """Copy of x with the reference's SPC5_VEC_PADDING_X zeros appended."""
    xp = np.zeros(len(x) + pad, dtype=x.dtype)
    xp[: len(x)] = x
    return xp


def beta_spmv_f64(r, nrows, brptr, headers, values, x, y):
    """y += A x in the AVX-512 kernel's order; y is updated in place (float64)."""
    xp = x_padded(np.ascontiguousarray(x, dtype=np.float64))
    assert y.dtype == np.float64 and y.flags.c_contiguous
    lib().oracle_beta_spmv_f64(r, nrows, _ptr(_i32(brptr)), _ptr(np.ascontiguousarray(headers)),
                               _ptr(np.ascontiguousarray(values, dtype=np.float64)), _ptr(xp), _ptr(y))
    return y


def beta_spmv_f64_chains(r, nrows, brptr, headers, values, x, y):
    """y += A x evaluated as per-(sub-row, column) multiply-add chains (the
    CUDA chain part's form); equals beta_spmv_f64 bit for bit for finite x."""
    xp = x_padded(np.ascontiguousarray(x, dtype=np.float64))
    assert y.dtype == np.float64 and y.flags.c_contiguous
    st = lib().oracle_beta_spmv_f64_chains(r, nrows, _ptr(_i32(brptr)), _ptr(np.ascontiguousarray(headers)),
                                           _ptr(np.ascontiguousarray(values, dtype=np.float64)), _ptr(xp),
                                           _ptr(y))
    if st != 0:
        raise MemoryError("oracle_beta_spmv_f64_chains")
    return y


def beta_spmv_f32(r, nrows, brptr, headers, values, x, y):
    xp = x_padded(np.ascontiguousarray(x, dtype=np.float32))
    assert y.dtype == np.float32 and y.flags.c_contiguous
    lib().oracle_beta_spmv_f32(r, nrows, _ptr(_i32(brptr)), _ptr(np.ascontiguousarray(headers)),
                               _ptr(np.ascontiguousarray(values, dtype=np.float32)), _ptr(xp), _ptr(y))
    return y


def beta_spmv_mixed(r, nrows, brptr, headers, values, x, y):
    xp = x_padded(np.ascontiguousarray(x, dtype=np.float32))
    assert y.dtype == np.float64 and y.flags.c_contiguous
    lib().oracle_beta_spmv_mixed(r, nrows, _ptr(_i32(brptr)), _ptr(np.ascontiguousarray(headers)),
                                 _ptr(np.ascontiguousarray(values, dtype=np.float32)), _ptr(xp), _ptr(y))
    return y


def beta_spmv_mixed8(r, nrows, brptr, headers, values, x, y):
    """Mixed precision in the 8-column layout (float values with the headers
    of the double conversion, float x, FP64 y): every chain is the FP64
    kernel's chain on the values and x widened to double -- the product of two
    floats is exact in FP64 -- so this is beta_spmv_f64 on the widened arrays
    (core_SPC5_{r}rVc_Spmv_double, src/spc5.hpp:2309-2632)."""
    return beta_spmv_f64(r, nrows, brptr, headers, np.asarray(values, dtype=np.float32).astype(np.float64),
                         np.asarray(x, dtype=np.float32).astype(np.float64), y)


def csr_to_beta_v8(r, rowptr, colidx, values):
    """Arrays of the 8-column layout with float values: the double conversion
    of the pattern (src/spc5.hpp:165-228), values rounded to float."""
    b, h, v = csr_to_beta(r, rowptr, colidx, np.asarray(values, dtype=np.float32).astype(np.float64))
    return b, h, v.astype(np.float32)


def csr_spmv_f64(rowptr, colidx, values, x, y):
    """y += A x row by row (CSR_Spmv_scalar); returns (y, sum_j |a_ij x_j| per row)."""
    rowptr, colidx = _i32(rowptr), _i32(colidx)
    n = len(rowptr) - 1
    absrow = np.zeros(n, dtype=np.float64)
    lib().oracle_csr_spmv_f64(n, _ptr(rowptr), _ptr(colidx),
                              _ptr(np.ascontiguousarray(values, dtype=np.float64)),
                              _ptr(np.ascontiguousarray(x, dtype=np.float64)), _ptr(y), _ptr(absrow))
    return y, absrow


def beta_to_coo(r, nrows, brptr, headers, values):
    values = np.ascontiguousarray(values)
    vs, mb, vb = layout(values.dtype)
    nnz = len(values)
    rows = np.zeros(nnz, dtype=np.int32)
    cols = np.zeros(nnz, dtype=np.int32)
    vals = np.zeros(nnz, dtype=values.dtype)
    k = lib().oracle_beta_to_coo(r, vs, mb, vb, nrows, _ptr(_i32(brptr)), _ptr(np.ascontiguousarray(headers)),
                                 _ptr(values), _ptr(rows), _ptr(cols), _ptr(vals))
    assert k == nnz
    return rows, cols, vals


def coo_sorted_to_csr(nrows, rows):
    rows = _i32(rows)
    rowptr = np.zeros(nrows + 1, dtype=np.int32)
    lib().oracle_coo_sorted_to_csr(nrows, len(rows), _ptr(rows), _ptr(rowptr))
    return rowptr


def find_best(is_double, nnz, blocks_r124):
    b = np.ascontiguousarray(blocks_r124, dtype=np.int64)
    est = C.c_double(0.0)
    r = lib().oracle_find_best(1 if is_double else 0, int(nnz), _ptr(b), C.byref(est))
    return int(r), float(est.value)


def threadsplit(r, nrows, brptr, headers, nthreads, dtype=np.float64):
    vs, mb, _ = layout(dtype)
    start = np.zeros(nthreads, dtype=np.int32)
    cnt = np.zeros(nthreads, dtype=np.int32)
    voff = np.zeros(nthreads, dtype=np.int64)
    lib().oracle_threadsplit(r, vs, mb, nrows, _ptr(_i32(brptr)), _ptr(np.ascontiguousarray(headers)),
                             nthreads, _ptr(start), _ptr(cnt), _ptr(voff))
    return start, cnt, voff


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref/libspc5ref.so)
# --------------------------------------------------------------------------

_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
    except OSError:
        return False
    return all(t in flags for t in ("avx512f", "avx512cd", "avx512bw", "avx512dq", "avx512vl"))


def ref():
    global _ref
    if _ref is None:
        l = C.CDLL(REF_SO)
        for pre, ct in (("ref_f64", C.c_double), ("ref_f32", C.c_float)):
            getattr(l, pre + "_create").restype = _P
            getattr(l, pre + "_create").argtypes = [_I, _I, _I, _P, _P, _P]
            getattr(l, pre + "_destroy").restype = None
            getattr(l, pre + "_destroy").argtypes = [_P]
            getattr(l, pre + "_block_count").restype = _I
            getattr(l, pre + "_block_count").argtypes = [_P, _I]
            getattr(l, pre + "_convert").restype = _I
            getattr(l, pre + "_convert").argtypes = [_P, _I]
            getattr(l, pre + "_get").restype = None
            getattr(l, pre + "_get").argtypes = [_P, _P, _P, _P]
            getattr(l, pre + "_spmv").restype = None
            getattr(l, pre + "_spmv").argtypes = [_P, _P, _P]
            getattr(l, pre + "_find_best").restype = _I
            getattr(l, pre + "_find_best").argtypes = [_P, _P]
            getattr(l, pre + "_split").restype = _I
            getattr(l, pre + "_split").argtypes = [_P, _I]
            getattr(l, pre + "_time_spmv_omp").restype = _D
            getattr(l, pre + "_time_spmv_omp").argtypes = [_P, _P, _P, _I]
        l.ref_f64_csr_spmv.restype = None
        l.ref_f64_csr_spmv.argtypes = [_P, _P, _P]
        l.ref_f64_spmv_omp.restype = None
        l.ref_f64_spmv_omp.argtypes = [_P, _P, _P]
        l.ref_max_threads.restype = _I
        l.ref_has_openmp.restype = _I
        _ref = l
    return _ref


class RefMatrix:
    """A reference ``SPC5Mat<T>`` built from CSR and driven through the reference API."""

    def __init__(self, rowptr, colidx, values, ncols=None):
        self.values_in = np.ascontiguousarray(values)
        self.dtype = self.values_in.dtype
        self.pre = "ref_f64" if self.dtype == np.float64 else "ref_f32"
        self.rowptr = _i32(rowptr)
        self.colidx = _i32(colidx)
        self.nrows = len(self.rowptr) - 1
        self.ncols = int(ncols if ncols is not None else (self.colidx.max() + 1 if len(self.colidx) else 0))
        self.nnz = len(self.values_in)
        self.r = 0
        self.h = getattr(ref(), self.pre + "_create")(self.nrows, self.ncols, self.nnz, _ptr(self.rowptr),
                                                      _ptr(self.colidx), _ptr(self.values_in))

    def __del__(self):
        if getattr(self, "h", None):
            getattr(ref(), self.pre + "_destroy")(self.h)
            self.h = None

    def _f(self, name):
        return getattr(ref(), self.pre + "_" + name)

    def block_count(self, r):
        return int(self._f("block_count")(self.h, r))

    def find_best(self):
        est = C.c_double(0.0)
        r = self._f("find_best")(self.h, C.byref(est))
        return int(r), float(est.value)

    def csr_spmv(self, x, y):
        ref().ref_f64_csr_spmv(self.h, _ptr(x_padded(x)), _ptr(y))
        return y

    def convert(self, r):
        nb = self._f("convert")(self.h, r)
        if nb < 0:
            raise ValueError(f"reference conversion failed for r={r}")
        self.r = r
        self.nblocks = nb
        return nb

    def arrays(self):
        _, mb, _ = layout(self.dtype)
        nbr = (self.nrows + self.r - 1) // self.r
        brptr = np.zeros(nbr + 1, dtype=np.int32)
        headers = np.zeros(self.nblocks * (4 + self.r * mb), dtype=np.uint8)
        vals = np.zeros(self.nnz, dtype=self.dtype)
        self._f("get")(self.h, _ptr(brptr), _ptr(headers), _ptr(vals))
        return brptr, headers, vals

    def spmv(self, x, y_padded):
        """y += A x with the reference kernels; y_padded must hold nrows + 7 entries."""
        self._f("spmv")(self.h, _ptr(x_padded(np.ascontiguousarray(x, dtype=self.dtype))), _ptr(y_padded))
        return y_padded

    def split(self, nthreads):
        return int(self._f("split")(self.h, nthreads))

    def time_spmv_omp(self, x_padded_arr, y, loops):
        return float(self._f("time_spmv_omp")(self.h, _ptr(x_padded_arr), _ptr(y), loops))
