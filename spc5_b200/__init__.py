"""spc5_b200 -- SPC5's beta(r,VS) SpMV hot path on B200 (sm_100a).

Python mirror of the reference's operator interface (src/spc5.hpp) over the
C ABI of ``libspc5cuda.so`` (include/spc5cuda.h).  The names follow the
reference: ``SPC5Mat``, ``CSR_to_SPC5``, ``SPC5_Spmv``, ``SPC5_block_count``,
``SPC5_find_best``, ``core_SPC5_{r}rVc_Spmv_{double,float}``.  Vectors are
torch CUDA tensors (plumbing only: device memory and the current stream); all
compute runs in the hand-written CUDA kernels of ``csrc/``.  There is no CPU
fallback: if the library is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspc5cuda.so")

# SPC5_MATRIX_TYPE (spc5.hpp:17-24)
UNDEFINED_FORMAT = 0
FORMAT_CSR = 1
FORMAT_1rVc_WT = 2
FORMAT_2rVc = 3
FORMAT_4rVc = 4
FORMAT_8rVc = 5
FORMAT_OF_R = {1: FORMAT_1rVc_WT, 2: FORMAT_2rVc, 4: FORMAT_4rVc, 8: FORMAT_8rVc}
R_OF_FORMAT = {v: k for k, v in FORMAT_OF_R.items()}

# SPC5_VEC_PADDING (spc5.hpp:26-29): not needed by these kernels, kept for callers
SPC5_VEC_PADDING_X = 15
SPC5_VEC_PADDING_Y = 7

F64 = 0
F32 = 1
# float values in the 8-column layout of SPC5Mat<double> (mixed-precision calls only)
F32_V8 = 2

EXPORTED_SYMBOLS = [
    "spc5cuda_status_string", "spc5cuda_get_last_error", "spc5cuda_set_stream",
    "core_SPC5_1rVc_Spmv_double", "core_SPC5_2rVc_Spmv_double", "core_SPC5_4rVc_Spmv_double",
    "core_SPC5_8rVc_Spmv_double", "core_SPC5_1rVc_Spmv_float", "core_SPC5_2rVc_Spmv_float",
    "core_SPC5_4rVc_Spmv_float", "core_SPC5_8rVc_Spmv_float",
    "spc5cuda_core_spmv_f64", "spc5cuda_core_spmv_f32",
    "spc5cuda_mat_create_csr", "spc5cuda_mat_create_beta", "spc5cuda_mat_destroy",
    "spc5cuda_mat_info", "spc5cuda_block_count", "spc5cuda_convert", "spc5cuda_get_arrays",
    "spc5cuda_spmv", "spc5cuda_spmv_mixed", "spc5cuda_spmm", "spc5cuda_spmm_mixed",
    "spc5cuda_find_best", "spc5cuda_autotune", "spc5cuda_batch_create", "spc5cuda_batch_launch",
    "spc5cuda_batch_info", "spc5cuda_batch_destroy", "spc5cuda_server_create",
    "spc5cuda_server_add_matrix", "spc5cuda_server_submit", "spc5cuda_server_wait",
    "spc5cuda_server_drain", "spc5cuda_server_get_stats", "spc5cuda_server_destroy",
    "spc5cuda_mat_create_coo", "spc5cuda_decode_coo", "spc5cuda_core_spmv_f64_noalloc",
    "spc5cuda_mat_set_kernel", "spc5cuda_mat_kernel", "spc5cuda_mat_spmv_launches",
]

TUNE_MODEL = 0
TUNE_MEASURE = 1

# SpMV kernel selection (spc5cuda_mat_set_kernel)
KERNEL_AUTO = 0
KERNEL_GROUPS = 1
KERNEL_ROWS = 2
KERNEL_SORTED = 3


class SPC5Error(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _lib().spc5cuda_status_string(status).decode() if _LIB is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else msg)


class spc5cuda_tune(C.Structure):
    _fields_ = [("r", C.c_int), ("pad", C.c_int), ("blocks", C.c_long * 4), ("est_us", C.c_double * 4)]


class spc5cuda_server_config(C.Structure):
    _fields_ = [("slots", C.c_int), ("max_k", C.c_int), ("hbm_budget", C.c_long), ("mixed", C.c_int),
                ("plan_serial", C.c_int)]


class spc5cuda_server_stats(C.Structure):
    _fields_ = [("completed", C.c_long), ("launches", C.c_long), ("mean_k", C.c_double),
                ("p50_us", C.c_double), ("p99_us", C.c_double), ("max_us", C.c_double),
                ("req_per_s", C.c_double), ("resident_bytes", C.c_long), ("matrices", C.c_int),
                ("pad", C.c_int)]


class spc5cuda_info(C.Structure):
    _fields_ = [("value_type", C.c_int), ("format", C.c_int), ("r", C.c_int), ("vs", C.c_int),
                ("nrows", C.c_int), ("ncols", C.c_int), ("nnz", C.c_long), ("nblocks", C.c_long),
                ("header_bytes", C.c_long), ("device_bytes", C.c_long)]


_LIB = None
_P = C.c_void_p
_I = C.c_int
_L = C.c_long


def _lib():
    """Load libspc5cuda.so; raises if the CUDA library was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m spc5_b200.build` "
                               "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        lib.spc5cuda_status_string.restype = C.c_char_p
        lib.spc5cuda_status_string.argtypes = [_I]
        lib.spc5cuda_get_last_error.restype = _I
        lib.spc5cuda_set_stream.restype = None
        lib.spc5cuda_set_stream.argtypes = [_P]
        for t in ("double", "float"):
            for r in (1, 2, 4, 8):
                f = getattr(lib, f"core_SPC5_{r}rVc_Spmv_{t}")
                f.restype = None
                f.argtypes = [_L, _P, _P, _P, _P, _P]
        for n in ("spc5cuda_core_spmv_f64", "spc5cuda_core_spmv_f32"):
            getattr(lib, n).restype = _I
            getattr(lib, n).argtypes = [_I, _L, _P, _P, _P, _P, _P, _P]
        lib.spc5cuda_mat_create_csr.restype = _I
        lib.spc5cuda_mat_create_csr.argtypes = [C.POINTER(_P), _I, _I, _I, _L, _P, _P, _P, _I, _P]
        lib.spc5cuda_mat_create_beta.restype = _I
        lib.spc5cuda_mat_create_beta.argtypes = [C.POINTER(_P), _I, _I, _I, _I, _L, _L, _P, _P, _P,
                                                 _I, _P]
        lib.spc5cuda_mat_destroy.restype = _I
        lib.spc5cuda_mat_destroy.argtypes = [_P]
        lib.spc5cuda_mat_info.restype = _I
        lib.spc5cuda_mat_info.argtypes = [_P, C.POINTER(spc5cuda_info)]
        lib.spc5cuda_mat_set_kernel.restype = _I
        lib.spc5cuda_mat_set_kernel.argtypes = [_P, _I]
        lib.spc5cuda_mat_kernel.restype = _I
        lib.spc5cuda_mat_kernel.argtypes = [_P, C.POINTER(_I)]
        lib.spc5cuda_mat_spmv_launches.restype = _I
        lib.spc5cuda_mat_spmv_launches.argtypes = [_P, C.POINTER(_I)]
        lib.spc5cuda_block_count.restype = _I
        lib.spc5cuda_block_count.argtypes = [_P, _I, C.POINTER(_L), _P]
        lib.spc5cuda_convert.restype = _I
        lib.spc5cuda_convert.argtypes = [_P, _I, _P]
        lib.spc5cuda_get_arrays.restype = _I
        lib.spc5cuda_get_arrays.argtypes = [_P, _P, _P, _P, _I, _P]
        lib.spc5cuda_spmv.restype = _I
        lib.spc5cuda_spmv.argtypes = [_P, _P, _P, _P]
        lib.spc5cuda_spmv_mixed.restype = _I
        lib.spc5cuda_spmv_mixed.argtypes = [_P, _P, _P, _P]
        for n in ("spc5cuda_spmm", "spc5cuda_spmm_mixed"):
            getattr(lib, n).restype = _I
            getattr(lib, n).argtypes = [_P, _I, _P, _L, _P, _L, _P]
        lib.spc5cuda_find_best.restype = _I
        lib.spc5cuda_find_best.argtypes = [_P, C.POINTER(_I), C.POINTER(C.c_double), _P]
        lib.spc5cuda_autotune.restype = _I
        lib.spc5cuda_autotune.argtypes = [_P, _I, C.POINTER(spc5cuda_tune), _P]
        lib.spc5cuda_batch_create.restype = _I
        lib.spc5cuda_batch_create.argtypes = [C.POINTER(_P), _I, _P, _P, _P, _P, _P, _P, _I, _P]
        lib.spc5cuda_batch_launch.restype = _I
        lib.spc5cuda_batch_launch.argtypes = [_P, _P]
        lib.spc5cuda_batch_info.restype = _I
        lib.spc5cuda_batch_info.argtypes = [_P, C.POINTER(_I), C.POINTER(_L)]
        lib.spc5cuda_batch_destroy.restype = _I
        lib.spc5cuda_batch_destroy.argtypes = [_P]
        lib.spc5cuda_server_create.restype = _I
        lib.spc5cuda_server_create.argtypes = [C.POINTER(_P), C.POINTER(spc5cuda_server_config)]
        lib.spc5cuda_server_add_matrix.restype = _I
        lib.spc5cuda_server_add_matrix.argtypes = [_P, _P, C.POINTER(_I)]
        lib.spc5cuda_server_submit.restype = _I
        lib.spc5cuda_server_submit.argtypes = [_P, _I, _P, _P, C.POINTER(_L)]
        lib.spc5cuda_server_wait.restype = _I
        lib.spc5cuda_server_wait.argtypes = [_P, _L, C.c_double, C.POINTER(C.c_double)]
        lib.spc5cuda_server_drain.restype = _I
        lib.spc5cuda_server_drain.argtypes = [_P, C.c_double]
        lib.spc5cuda_server_get_stats.restype = _I
        lib.spc5cuda_server_get_stats.argtypes = [_P, C.POINTER(spc5cuda_server_stats), _I]
        lib.spc5cuda_server_destroy.restype = _I
        lib.spc5cuda_server_destroy.argtypes = [_P]
        lib.spc5cuda_mat_create_coo.restype = _I
        lib.spc5cuda_mat_create_coo.argtypes = [C.POINTER(_P), _I, _I, _I, _L, _P, _P, _P, _I, _I, _P]
        lib.spc5cuda_decode_coo.restype = _I
        lib.spc5cuda_decode_coo.argtypes = [_P, _P, _P, _P, _P]
        _LIB = lib
    return _LIB


def lib():
    return _lib()


def _check(status: int, what: str = "") -> None:
    if status != 0:
        raise SPC5Error(status, what)


def _stream(stream=None):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _dptr(t, dtype=None, what="tensor"):
    """Device pointer of a contiguous CUDA tensor (checked)."""
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{what} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{what} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{what} must be {dtype}, got {t.dtype}")
    return C.c_void_p(t.data_ptr())


def _np_ptr(a):
    return a.ctypes.data_as(_P)


def _value_type(dtype) -> int:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return F64
    if dt == np.float32:
        return F32
    raise TypeError(f"unsupported value dtype {dt}")


class SPC5Mat:
    """Device-resident counterpart of the reference's ``SPC5Mat<T>``
    (spc5.hpp:44-62).  Build one with :func:`csr_matrix` (or
    :func:`beta_matrix`), convert it in place with :func:`CSR_to_SPC5`."""

    def __init__(self, handle, keep=None):
        self._h = handle
        self._keep = keep

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.spc5cuda_mat_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def info(self) -> spc5cuda_info:
        inf = spc5cuda_info()
        _check(_lib().spc5cuda_mat_info(self._h, C.byref(inf)), "spc5cuda_mat_info")
        return inf

    def set_kernel(self, kernel: int) -> None:
        """Select the SpMV kernel: KERNEL_AUTO, KERNEL_GROUPS, KERNEL_ROWS or KERNEL_SORTED."""
        _check(_lib().spc5cuda_mat_set_kernel(self._h, int(kernel)), "spc5cuda_mat_set_kernel")

    @property
    def spmv_launches(self) -> int:
        """Kernel launches one SPC5_Spmv of this converted matrix makes (one per part of the
        length-sorted plan, else 1)."""
        n = C.c_int(0)
        _check(_lib().spc5cuda_mat_spmv_launches(self._h, C.byref(n)), "spc5cuda_mat_spmv_launches")
        return n.value

    @property
    def kernel(self) -> int:
        """The SpMV kernel in use: KERNEL_GROUPS, KERNEL_ROWS or KERNEL_SORTED (KERNEL_AUTO before
        conversion)."""
        k = C.c_int(0)
        _check(_lib().spc5cuda_mat_kernel(self._h, C.byref(k)), "spc5cuda_mat_kernel")
        return k.value

    @property
    def format(self) -> int:
        return self.info().format

    @property
    def r(self) -> int:
        return self.info().r

    @property
    def numberOfRows(self) -> int:
        return self.info().nrows

    @property
    def numberOfColumns(self) -> int:
        return self.info().ncols

    @property
    def numberOfNNZ(self) -> int:
        return self.info().nnz

    @property
    def numberOfBlocks(self) -> int:
        return self.info().nblocks

    @property
    def dtype(self):
        """Value dtype (float32 for both F32 and F32_V8 handles)."""
        return np.float64 if self.info().value_type == F64 else np.float32

    @property
    def value_type(self) -> int:
        return self.info().value_type

    def arrays(self):
        """Host copies of (rowsSize, blocksColumnIndexesWithMasks, values)."""
        inf = self.info()
        if inf.r == 0:
            raise SPC5Error(4, "arrays(): matrix is not converted")
        nbr = (inf.nrows + inf.r - 1) // inf.r
        brptr = np.zeros(nbr + 1, dtype=np.int32)
        headers = np.zeros(inf.header_bytes, dtype=np.uint8)
        values = np.zeros(inf.nnz, dtype=np.float64 if inf.value_type == F64 else np.float32)
        _check(_lib().spc5cuda_get_arrays(self._h, _np_ptr(brptr), _np_ptr(headers), _np_ptr(values),
                                          1, None), "spc5cuda_get_arrays")
        return brptr, headers, values


def csr_matrix(rowptr, colidx, values, ncols: int, dtype=None, stream=None, value_type=None) -> SPC5Mat:
    """A CSR ``SPC5Mat`` from host numpy arrays or CUDA tensors (int32
    indices, sorted columns per row).  ``dtype`` (float64/float32) casts the
    values; float32 gives the VS = 16 layout used by the float and mixed
    kernels.  ``value_type=F32_V8`` casts the values to float32 and keeps the
    8-column layout of the double format (the mixed-precision calls only)."""
    import torch
    if value_type == F32_V8:
        dtype = np.float32
    on_device = isinstance(rowptr, torch.Tensor) and rowptr.is_cuda
    if on_device:
        vals = values if dtype is None else values.to(getattr(torch, np.dtype(dtype).name))
        vt = _value_type(np.float64 if vals.dtype == torch.float64 else np.float32)
        nrows = rowptr.numel() - 1
        nnz = colidx.numel()
        ptrs = (_dptr(rowptr, torch.int32, "rowptr"), _dptr(colidx, torch.int32, "colidx"),
                _dptr(vals, None, "values"))
        keep = (rowptr, colidx, vals)
    else:
        rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        ci = np.ascontiguousarray(colidx, dtype=np.int32)
        vals = np.ascontiguousarray(values, dtype=dtype if dtype is not None else None)
        vt = _value_type(vals.dtype)
        nrows = len(rp) - 1
        nnz = len(ci)
        ptrs = (_np_ptr(rp), _np_ptr(ci), _np_ptr(vals))
        keep = (rp, ci, vals)
    if value_type == F32_V8:
        vt = F32_V8
    h = C.c_void_p()
    st = _stream(stream) if torch.cuda.is_available() else None
    _check(_lib().spc5cuda_mat_create_csr(C.byref(h), vt, nrows, int(ncols), nnz, *ptrs,
                                          1 if on_device else 0, st), "spc5cuda_mat_create_csr")
    del keep
    return SPC5Mat(h)


def coo_matrix(nrows: int, ncols: int, rows, cols, values, sorted: bool = False,
               stream=None) -> SPC5Mat:
    """A CSR ``SPC5Mat`` from COO triplets, built on the device
    (COO_sorted_to_CSR / COO_unsorted_to_CSR, spc5.hpp:77-114).  Host numpy
    arrays or CUDA tensors; int32 indices."""
    import torch
    on_device = isinstance(rows, torch.Tensor) and rows.is_cuda
    if on_device:
        vt = _value_type(np.float64 if values.dtype == torch.float64 else np.float32)
        ptrs = (_dptr(rows, torch.int32, "rows"), _dptr(cols, torch.int32, "cols"), _dptr(values))
        nnz = rows.numel()
        keep = (rows, cols, values)
    else:
        r_ = np.ascontiguousarray(rows, dtype=np.int32)
        c_ = np.ascontiguousarray(cols, dtype=np.int32)
        v_ = np.ascontiguousarray(values)
        vt = _value_type(v_.dtype)
        ptrs = (_np_ptr(r_), _np_ptr(c_), _np_ptr(v_))
        nnz = len(r_)
        keep = (r_, c_, v_)
    h = C.c_void_p()
    _check(_lib().spc5cuda_mat_create_coo(C.byref(h), vt, int(nrows), int(ncols), nnz, *ptrs,
                                          1 if on_device else 0, 1 if sorted else 0, _stream(stream)),
           "spc5cuda_mat_create_coo")
    del keep
    return SPC5Mat(h)


def decode_coo(mat: SPC5Mat, stream=None):
    """(rows, cols, values) CUDA tensors of a converted matrix in storage order."""
    import torch
    inf = mat.info()
    dt = torch.float64 if inf.value_type == F64 else torch.float32
    rows = torch.empty(inf.nnz, dtype=torch.int32, device="cuda")
    cols = torch.empty(inf.nnz, dtype=torch.int32, device="cuda")
    vals = torch.empty(inf.nnz, dtype=dt, device="cuda")
    _check(_lib().spc5cuda_decode_coo(mat.handle, C.c_void_p(rows.data_ptr()), C.c_void_p(cols.data_ptr()),
                                      C.c_void_p(vals.data_ptr()), _stream(stream)), "decode_coo")
    return rows, cols, vals


def beta_matrix(r: int, nrows: int, ncols: int, rowsSize, headers, values, stream=None,
                value_type=None) -> SPC5Mat:
    """An ``SPC5Mat`` from already-converted host arrays (e.g. the reference's
    ``SPC5Mat`` after ``CSR_to_SPC5``).  ``value_type=F32_V8``: float values
    with the 8-column headers of the double format."""
    brptr = np.ascontiguousarray(rowsSize, dtype=np.int32)
    hdr = np.ascontiguousarray(headers, dtype=np.uint8)
    vals = np.ascontiguousarray(values)
    vt = _value_type(vals.dtype)
    if value_type == F32_V8:
        if vals.dtype != np.float32:
            raise TypeError("F32_V8 values must be float32")
        vt = F32_V8
    stride = 4 + r * (2 if vt == F32 else 1)
    if len(hdr) % stride:
        raise ValueError("header array size is not a multiple of the block stride")
    h = C.c_void_p()
    _check(_lib().spc5cuda_mat_create_beta(C.byref(h), vt, r, nrows, ncols, len(vals), len(hdr) // stride,
                                           _np_ptr(brptr), _np_ptr(hdr), _np_ptr(vals), 0,
                                           _stream(stream)), "spc5cuda_mat_create_beta")
    return SPC5Mat(h)


def SPC5_block_count(mat: SPC5Mat, fmt: int, stream=None) -> int:
    """Block count of converting ``mat`` (CSR) to ``fmt``; the reference's
    wrapper (spc5.hpp:1120-1148) computes it and drops it, this returns it."""
    r = R_OF_FORMAT.get(fmt)
    if r is None:
        raise SPC5Error(4, "SPC5_block_count : Unknown format type")
    out = C.c_long(0)
    _check(_lib().spc5cuda_block_count(mat.handle, r, C.byref(out), _stream(stream)),
           "spc5cuda_block_count")
    return int(out.value)


def CSR_to_SPC5(mat: SPC5Mat, fmt: int, stream=None) -> None:
    """In-place conversion on the device (CSR_to_SPC5, spc5.hpp:989-1018)."""
    _check(_lib().spc5cuda_convert(mat.handle, int(fmt), _stream(stream)), "CSR_to_SPC5")


def SPC5_Spmv(mat: SPC5Mat, x, y, stream=None) -> None:
    """y += A x (SPC5_Spmv, spc5.hpp:1090-1118); x, y CUDA tensors of the
    matrix's value type."""
    import torch
    dt = torch.float64 if mat.dtype == np.float64 else torch.float32
    _check(_lib().spc5cuda_spmv(mat.handle, _dptr(x, dt, "x"), _dptr(y, dt, "y"), _stream(stream)),
           "SPC5_Spmv")


def SPC5_Spmv_mixed(mat: SPC5Mat, x, y, stream=None) -> None:
    """y += A x with FP32 values and x, FP64 accumulation and y."""
    import torch
    _check(_lib().spc5cuda_spmv_mixed(mat.handle, _dptr(x, torch.float32, "x"),
                                      _dptr(y, torch.float64, "y"), _stream(stream)), "SPC5_Spmv_mixed")


def SPC5_Spmm(mat: SPC5Mat, X, Y, stream=None) -> None:
    """Y += A X for k right-hand sides.  X is (ncols, k) and Y (nrows, k),
    row-major CUDA tensors (the k values of one row contiguous); column j of Y
    is bit-identical to SPC5_Spmv with column j of X."""
    import torch
    dt = torch.float64 if mat.dtype == np.float64 else torch.float32
    if X.dim() != 2 or Y.dim() != 2 or X.shape[1] != Y.shape[1]:
        raise ValueError("X and Y must be 2-D with the same number of columns")
    if X.stride(1) != 1 or Y.stride(1) != 1:
        raise ValueError("X and Y must be row-major (unit stride along k)")
    k = X.shape[1]
    _check(_lib().spc5cuda_spmm(mat.handle, k, C.c_void_p(_check_dev(X, dt, "X")), X.stride(0),
                                C.c_void_p(_check_dev(Y, dt, "Y")), Y.stride(0), _stream(stream)),
           "SPC5_Spmm")


def SPC5_Spmm_mixed(mat: SPC5Mat, X, Y, stream=None) -> None:
    """Y += A X with FP32 values and X, FP64 accumulation and Y (row-major)."""
    import torch
    if X.dim() != 2 or Y.dim() != 2 or X.shape[1] != Y.shape[1]:
        raise ValueError("X and Y must be 2-D with the same number of columns")
    if X.stride(1) != 1 or Y.stride(1) != 1:
        raise ValueError("X and Y must be row-major (unit stride along k)")
    k = X.shape[1]
    _check(_lib().spc5cuda_spmm_mixed(mat.handle, k, C.c_void_p(_check_dev(X, torch.float32, "X")),
                                      X.stride(0), C.c_void_p(_check_dev(Y, torch.float64, "Y")),
                                      Y.stride(0), _stream(stream)), "SPC5_Spmm_mixed")


def _check_dev(t, dtype, what):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{what} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{what} must be {dtype}, got {t.dtype}")
    return t.data_ptr()


def SPC5_find_best(mat: SPC5Mat, stream=None):
    """(r, estimate) of the reference's speed model, SPC5_find_best
    (spc5.hpp:1151-1223), on block counts taken on the device (CSR handle)."""
    r, est = C.c_int(0), C.c_double(0.0)
    _check(_lib().spc5cuda_find_best(mat.handle, C.byref(r), C.byref(est), _stream(stream)),
           "SPC5_find_best")
    return int(r.value), float(est.value)


def autotune(mat: SPC5Mat, mode: int = TUNE_MODEL, stream=None) -> dict:
    """The B200 autotuner on a CSR handle: {'r', 'blocks': {r: n}, 'est_us': {r: t}}."""
    t = spc5cuda_tune()
    _check(_lib().spc5cuda_autotune(mat.handle, int(mode), C.byref(t), _stream(stream)), "autotune")
    rs = (1, 2, 4, 8)
    return {"r": int(t.r), "blocks": {r: int(t.blocks[i]) for i, r in enumerate(rs)},
            "est_us": {r: float(t.est_us[i]) for i, r in enumerate(rs)}}


class Batch:
    """Many converted matrices, each with its own row-major X (ncols x k) and
    Y (nrows x k) CUDA tensors, launched together as one CUDA graph."""

    def __init__(self, mats, Xs, Ys, mixed=False, stream=None):
        import torch
        n = len(mats)
        self._keep = (list(mats), list(Xs), list(Ys))
        hm = (_P * max(1, n))(*[m.handle for m in mats])
        ks = (_I * max(1, n))(*[int(X.shape[1]) for X in Xs])
        xp = (_P * max(1, n))(*[X.data_ptr() for X in Xs])
        yp = (_P * max(1, n))(*[Y.data_ptr() for Y in Ys])
        lx = (_L * max(1, n))(*[int(X.stride(0)) for X in Xs])
        ly = (_L * max(1, n))(*[int(Y.stride(0)) for Y in Ys])
        for X, Y in zip(Xs, Ys):
            if not (X.is_cuda and Y.is_cuda) or X.stride(1) != 1 or Y.stride(1) != 1:
                raise ValueError("X and Y must be row-major CUDA tensors")
        self._h = C.c_void_p()
        _check(_lib().spc5cuda_batch_create(C.byref(self._h), n, C.cast(hm, _P), C.cast(ks, _P),
                                            C.cast(xp, _P), C.cast(lx, _P), C.cast(yp, _P),
                                            C.cast(ly, _P), 1 if mixed else 0, _stream(stream)),
               "spc5cuda_batch_create")
        del torch

    def launch(self, stream=None):
        _check(_lib().spc5cuda_batch_launch(self._h, _stream(stream)), "spc5cuda_batch_launch")

    def info(self):
        nc, nj = C.c_int(0), C.c_long(0)
        _check(_lib().spc5cuda_batch_info(self._h, C.byref(nc), C.byref(nj)), "spc5cuda_batch_info")
        return int(nc.value), int(nj.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.spc5cuda_batch_destroy(h)
            self._h = None


class Server:
    """Request loop over resident matrices (continuous batching of
    same-matrix requests into multi-RHS launches, admission by HBM footprint,
    latency percentiles).  A request computes y = A x for device tensors."""

    def __init__(self, slots=4, max_k=16, hbm_budget=None, mixed=False, plan_serial=False):
        import torch
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info()
            hbm_budget = int(free * 0.9)
        cfg = spc5cuda_server_config(int(slots), int(max_k), int(hbm_budget), 1 if mixed else 0,
                                     1 if plan_serial else 0)
        self.mixed = bool(mixed)
        self._h = C.c_void_p()
        self._mats = []
        self._live = {}
        _check(_lib().spc5cuda_server_create(C.byref(self._h), C.byref(cfg)), "spc5cuda_server_create")

    def add_matrix(self, mat: SPC5Mat) -> int:
        i = C.c_int(-1)
        _check(_lib().spc5cuda_server_add_matrix(self._h, mat.handle, C.byref(i)), "add_matrix")
        self._mats.append(mat)
        return int(i.value)

    def submit(self, mat_id: int, x, y) -> int:
        """Queues y = A_mat_id x (x, y CUDA tensors kept alive until wait/drain)."""
        rid = C.c_long(0)
        _check(_lib().spc5cuda_server_submit(self._h, int(mat_id), C.c_void_p(x.data_ptr()),
                                             C.c_void_p(y.data_ptr()), C.byref(rid)), "submit")
        self._live[int(rid.value)] = (x, y)
        return int(rid.value)

    def wait(self, rid: int, timeout_s: float = 60.0) -> float:
        lat = C.c_double(0.0)
        _check(_lib().spc5cuda_server_wait(self._h, int(rid), float(timeout_s), C.byref(lat)), "wait")
        self._live.pop(int(rid), None)
        return float(lat.value)

    def drain(self, timeout_s: float = 120.0) -> None:
        _check(_lib().spc5cuda_server_drain(self._h, float(timeout_s)), "drain")
        self._live.clear()

    def stats(self, reset: bool = False) -> dict:
        st = spc5cuda_server_stats()
        _check(_lib().spc5cuda_server_get_stats(self._h, C.byref(st), 1 if reset else 0), "stats")
        return {f[0]: getattr(st, f[0]) for f in st._fields_ if f[0] != "pad"}

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.spc5cuda_server_destroy(h)
            self._h = None

    def __del__(self):
        self.close()


def core_spmv(r: int, nbRows: int, rowsSizes, headers, values, x, y, stream=None) -> None:
    """The drop-in kernel ``core_SPC5_{r}rVc_Spmv_{double,float}`` over device
    tensors, through its explicit-stream C entry point."""
    import torch
    f = _lib().spc5cuda_core_spmv_f64 if values.dtype == torch.float64 else _lib().spc5cuda_core_spmv_f32
    _check(f(int(r), int(nbRows), _dptr(rowsSizes, torch.int32, "rowsSizes"),
             _dptr(headers, torch.uint8, "headers"), _dptr(values, None, "values"),
             _dptr(x, values.dtype, "x"), _dptr(y, values.dtype, "y"), _stream(stream)),
           f"core_SPC5_{r}rVc_Spmv")


def core_spmv_void(r: int, nbRows: int, rowsSizes, headers, values, x, y, stream=None) -> None:
    """Calls the exact reference-named void symbol ``core_SPC5_{r}rVc_Spmv_{T}``
    (stream from ``spc5cuda_set_stream``) and checks ``spc5cuda_get_last_error``."""
    import torch
    t = "double" if values.dtype == torch.float64 else "float"
    lib_ = _lib()
    lib_.spc5cuda_set_stream(_stream(stream))
    getattr(lib_, f"core_SPC5_{r}rVc_Spmv_{t}")(int(nbRows), _dptr(rowsSizes, torch.int32),
                                                 _dptr(headers, torch.uint8), _dptr(values),
                                                 _dptr(x, values.dtype), _dptr(y, values.dtype))
    _check(lib_.spc5cuda_get_last_error(), f"core_SPC5_{r}rVc_Spmv_{t}")
