"""The allocation-free FP64 drop-in, spc5cuda_core_spmv_f64_noalloc.

Some callers may not allocate device memory while they run (a fixed memory
budget set at start-up, a real-time loop, a pool owned by another
framework).  This entry point keeps its scratch in a fixed device array
instead of allocating per call.  Checked here through the C ABI against the
ordinary drop-in, spc5cuda_core_spmv_f64, bit for bit, on two calls in a
row (the second call reuses the scratch the first one left behind).  The
file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import spc5_b200 as S
from spc5_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _lib():
    lib = S.lib()
    f = lib.spc5cuda_core_spmv_f64_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_long] + [C.c_void_p] * 6
    return lib


def _arrays(csr, r):
    m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
    S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
    return [torch.from_numpy(a).cuda() for a in m.arrays()]


def _call(fn, r, nrows, arrs, x, y):
    brptr, headers, values = arrs
    st = fn(r, nrows, C.c_void_p(brptr.data_ptr()), C.c_void_p(headers.data_ptr()),
            C.c_void_p(values.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, S.lib().spc5cuda_status_string(st)


@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_noalloc_equals_dropin_two_calls(cuda, r):
    lib = _lib()
    # two different matrices in a row: the second call must not depend on
    # what the first left in the shared scratch
    for csr, seed in ((M.powerlaw(60000, seed=31), 1), (M.stencil27(17), 2)):
        arrs = _arrays(csr, r)
        x = torch.from_numpy(M.x_vector(csr.ncols, seed)).cuda()
        y0 = torch.from_numpy(M.x_vector(csr.nrows, seed + 10)).cuda()
        y_ref, y_new = y0.clone(), y0.clone()
        for _ in range(2):
            _call(lib.spc5cuda_core_spmv_f64, r, csr.nrows, arrs, x, y_ref)
            _call(lib.spc5cuda_core_spmv_f64_noalloc, r, csr.nrows, arrs, x, y_new)
        torch.cuda.synchronize()
        assert y_new.cpu().numpy().tobytes() == y_ref.cpu().numpy().tobytes()


def test_noalloc_rejects_too_many_block_rows(cuda):
    lib = _lib()
    z = torch.zeros(4, dtype=torch.float64, device="cuda")
    zi = torch.zeros(4, dtype=torch.int32, device="cuda")
    st = lib.spc5cuda_core_spmv_f64_noalloc(1, (1 << 20) + 1, C.c_void_p(zi.data_ptr()),
                                            C.c_void_p(zi.data_ptr()), C.c_void_p(z.data_ptr()),
                                            C.c_void_p(z.data_ptr()), C.c_void_p(z.data_ptr()),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 1  # SPC5CUDA_ERR_INVALID, before any device work
