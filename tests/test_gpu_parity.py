"""Parity of the CUDA path (through the C ABI) with the oracle and the
reference's golden outputs.

Bars:
* conversion (CSR_to_SPC5 on the device): rowsSize, headers and values
  identical byte for byte to the reference's;
* FP64 / FP32 SpMV: y identical bit for bit to the reference's AVX-512
  kernels (finite x), which the oracle restates and golden.npz records;
* mixed precision: identical to the oracle's definition, and within 1e-6
  normwise relative error of the FP64 CSR oracle (componentwise error
  |dy_i| / sum_j |a_ij x_j| <= 2.5e-7, two FP32 roundings of a and x).
"""
import numpy as np
import pytest
import torch

import oracle
import spc5_b200 as S
from spc5_b200 import matrices as M

pytestmark = pytest.mark.gpu

DTYPES = [("f64", np.float64), ("f32", np.float32)]
TORCH = {np.float64: torch.float64, np.float32: torch.float32}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def names(golden):
    return [str(n) for n in golden["names"]]


def converted(csr, dt, r):
    m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols)
    S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
    return m


def gpu_spmv(m, x, y0):
    y = dev(y0)
    S.SPC5_Spmv(m, dev(x), y)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def golden_csr(golden, n):
    return M.CSR(int(golden[f"{n}/nrows"]), int(golden[f"{n}/ncols"]), golden[f"{n}/rowptr"],
                 golden[f"{n}/colidx"], golden[f"{n}/values"], n)


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_convert_matches_reference(cuda, golden, tag, dt, r):
    for n in names(golden):
        csr = golden_csr(golden, n)
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols)
        assert S.SPC5_block_count(m, S.FORMAT_OF_R[r]) == int(golden[f"{n}/{tag}/r{r}/block_count"])
        S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
        assert m.format == S.FORMAT_OF_R[r] and m.numberOfBlocks == int(golden[f"{n}/{tag}/r{r}/block_count"])
        brptr, headers, vals = m.arrays()
        assert np.array_equal(brptr, golden[f"{n}/{tag}/r{r}/rowsSize"]), n
        assert np.array_equal(headers, golden[f"{n}/{tag}/r{r}/headers"]), n
        assert vals.tobytes() == golden[f"{n}/{tag}/r{r}/values"].tobytes(), n


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_spmv_matches_reference(cuda, golden, tag, dt, r):
    for n in names(golden):
        csr = golden_csr(golden, n)
        m = converted(csr, dt, r)
        y = gpu_spmv(m, golden[f"{n}/x"].astype(dt), np.zeros(csr.nrows, dtype=dt))
        assert y.tobytes() == golden[f"{n}/{tag}/r{r}/y"].tobytes(), n


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_dropin_entry_points(cuda, golden, tag, dt, r):
    """core_SPC5_{r}rVc_Spmv_{T} over the reference's own converted arrays."""
    for n in names(golden)[:5]:
        nrows = int(golden[f"{n}/nrows"])
        args = (dev(golden[f"{n}/{tag}/r{r}/rowsSize"]), dev(golden[f"{n}/{tag}/r{r}/headers"]),
                dev(golden[f"{n}/{tag}/r{r}/values"]), dev(golden[f"{n}/x"].astype(dt)))
        for fn in (S.core_spmv, S.core_spmv_void):
            y = torch.zeros(nrows, dtype=TORCH[dt], device="cuda")
            fn(r, nrows, *args, y)
            torch.cuda.synchronize()
            assert y.cpu().numpy().tobytes() == golden[f"{n}/{tag}/r{r}/y"].tobytes(), (n, fn.__name__)


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_dropin_takes_either_kernel(cuda, tag, dt, r):
    """The drop-in symbols pick the row kernel or the group kernel on the
    device (a block-row of a dense 1500-column row does not fit the row
    kernel's buffers; the stencil's do): both give the oracle's bits, over
    three accumulating calls that reuse the library's scratch pool."""
    f = oracle.beta_spmv_f64 if dt == np.float64 else oracle.beta_spmv_f32
    for csr in (M.stencil27(14), M.dense(1500), M.powerlaw(30000, seed=13)):
        vals = csr.values.astype(dt)
        brptr, headers, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, vals)
        x = M.x_vector(csr.ncols, 8, dt)
        y0 = M.x_vector(csr.nrows, 9, dt)
        yo = y0.copy()
        args = (dev(brptr), dev(headers), dev(ov), dev(x))
        y = dev(y0)
        for _ in range(3):
            f(r, csr.nrows, brptr, headers, ov, x, yo)
            S.core_spmv_void(r, csr.nrows, *args, y)
        torch.cuda.synchronize()
        assert y.cpu().numpy().tobytes() == yo.tobytes(), csr.name


@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_handle_from_reference_arrays(cuda, golden, r):
    for n in names(golden)[:4]:
        nrows, ncols = int(golden[f"{n}/nrows"]), int(golden[f"{n}/ncols"])
        m = S.beta_matrix(r, nrows, ncols, golden[f"{n}/f64/r{r}/rowsSize"], golden[f"{n}/f64/r{r}/headers"],
                          golden[f"{n}/f64/r{r}/values"])
        y = gpu_spmv(m, golden[f"{n}/x"], np.zeros(nrows))
        assert y.tobytes() == golden[f"{n}/f64/r{r}/y"].tobytes()


def irregular_cases():
    yield M.random_csr(1000, 1200, 0.02, seed=1, empty_row_frac=0.2)
    yield M.random_csr(333, 64, 0.5, seed=2)
    yield M.powerlaw(20000, seed=7)
    yield M.banded(4099, 150, 0.1, seed=8)
    yield M.stencil27(9)
    yield M.from_coo(5, 3, [0, 2, 4], [2, 0, 1], [1.5, -2.0, 3.25])  # ncols < VS
    yield M.from_coo(7, 7, [], [], [])  # no entries at all
    yield M.dense(40)


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_spmv_accumulates_like_oracle(cuda, tag, dt, r):
    """y += A x on a nonzero y, repeated 16 times like the reference driver
    (load_mm_and_compare.cpp:505-507): bit-identical to the oracle."""
    f = oracle.beta_spmv_f64 if dt == np.float64 else oracle.beta_spmv_f32
    for csr in irregular_cases():
        vals = csr.values.astype(dt)
        brptr, headers, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, vals)
        m = converted(csr, dt, r)
        gb, gh, gv = m.arrays()
        assert np.array_equal(gb, brptr) and np.array_equal(gh, headers) and gv.tobytes() == ov.tobytes()
        x = M.x_vector(csr.ncols, 3, dt)
        y0 = M.x_vector(csr.nrows, 4, dt)
        yo = y0.copy()
        for _ in range(16):
            f(r, csr.nrows, brptr, headers, ov, x, yo)
        y = dev(y0)
        xd = dev(x)
        for _ in range(16):
            S.SPC5_Spmv(m, xd, y)
        torch.cuda.synchronize()
        assert y.cpu().numpy().tobytes() == yo.tobytes(), csr.name


def kernel_cases():
    yield from irregular_cases()
    yield M.stencil27(24)
    yield M.poisson2d(96)
    yield M.random_csr(4000, 4000, 0.003, seed=11, empty_row_frac=0.5)  # runs of empty rows


@pytest.mark.parametrize("tag,dt", DTYPES + [("mixed", np.float32)])
@pytest.mark.parametrize("r", [1, 2, 4, 8])
@pytest.mark.parametrize("kernel", [S.KERNEL_GROUPS, S.KERNEL_ROWS, S.KERNEL_SORTED])
def test_both_kernels_bit_exact(cuda, tag, dt, r, kernel):
    """The group kernel, the thread-per-sub-row kernel and the length-sorted
    plan each give the oracle's bits (y += A x on a nonzero y); the row
    kernel refuses a matrix with a block-row larger than its staging
    buffers."""
    for csr in kernel_cases():
        vals = csr.values.astype(dt)
        brptr, headers, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, vals)
        m = converted(csr, dt, r)
        if kernel == S.KERNEL_ROWS:
            nbr = len(brptr) - 1
            longest = int(np.diff(brptr).max()) if nbr else 0
            rp = csr.rowptr.astype(np.int64)
            vals_per = rp[np.minimum(np.arange(1, nbr + 1) * r, csr.nrows)] - rp[np.arange(nbr) * r]
            most = int(vals_per.max()) if nbr else 0
            vb, mb = (8, 1) if dt == np.float64 else (4, 2)
            fits = longest * (4 + r * mb) + 32 <= 2048 and (most + 2 * (16 // vb)) * vb <= 8192
            try:
                m.set_kernel(kernel)
            except S.SPC5Error as e:
                assert e.status == 5 and not fits, csr.name
                continue
            assert fits, csr.name
        else:
            m.set_kernel(kernel)
        assert m.kernel == kernel, csr.name
        x = M.x_vector(csr.ncols, 3, np.float32 if tag == "mixed" else dt)
        if tag == "mixed":
            y0 = M.x_vector(csr.nrows, 4)
            yo = oracle.beta_spmv_mixed(r, csr.nrows, brptr, headers, ov, x, y0.copy())
            y = dev(y0)
            S.SPC5_Spmv_mixed(m, dev(x), y)
        else:
            y0 = M.x_vector(csr.nrows, 4, dt)
            f = oracle.beta_spmv_f64 if dt == np.float64 else oracle.beta_spmv_f32
            yo = f(r, csr.nrows, brptr, headers, ov, x, y0.copy())
            y = dev(y0)
            S.SPC5_Spmv(m, dev(x), y)
        torch.cuda.synchronize()
        assert y.cpu().numpy().tobytes() == yo.tobytes(), (csr.name, kernel)


def test_kernel_selection(cuda):
    """AUTO picks the row kernel for a stencil (every r) and the sorted plan
    for a matrix with a block-row longer than the row kernel's buffers."""
    st = converted(M.stencil27(12), np.float64, 4)
    assert st.kernel == S.KERNEL_ROWS
    st.set_kernel(S.KERNEL_GROUPS)
    assert st.kernel == S.KERNEL_GROUPS
    st.set_kernel(S.KERNEL_AUTO)
    assert st.kernel == S.KERNEL_ROWS
    st8 = converted(M.stencil27(12), np.float64, 8)
    assert st8.kernel == S.KERNEL_ROWS  # r = 8: one lane per sub-row
    st8.set_kernel(S.KERNEL_GROUPS)
    assert st8.kernel == S.KERNEL_GROUPS
    d = converted(M.dense(4096), np.float64, 1)  # one block-row of 512 blocks: 2.5 KB of headers
    assert d.kernel == S.KERNEL_SORTED  # AUTO: a block-row does not fit the row kernel
    d.set_kernel(S.KERNEL_GROUPS)
    assert d.kernel == S.KERNEL_GROUPS
    with pytest.raises(S.SPC5Error) as e:
        d.set_kernel(S.KERNEL_ROWS)
    assert e.value.status == 5
    with pytest.raises(S.SPC5Error):
        d.set_kernel(7)
    pl = converted(M.powerlaw(20000, seed=7), np.float64, 2)
    assert pl.kernel == S.KERNEL_SORTED
    assert st.spmv_launches == 1 and pl.spmv_launches >= 2  # one launch per part of the plan
    before = pl.info().device_bytes
    pl.set_kernel(S.KERNEL_GROUPS)  # the reference order back, the sorted copy released
    assert pl.kernel == S.KERNEL_GROUPS
    pl.set_kernel(S.KERNEL_AUTO)  # builds it again, in place
    assert pl.kernel == S.KERNEL_SORTED and pl.info().device_bytes == before


@pytest.mark.parametrize("vt", [S.F64, S.F32, S.F32_V8])
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_sorted_plan_in_place(cuda, vt, r):
    """A handle served by the length-sorted plan keeps one copy of its
    headers and values (the sorted one): its device footprint is the beta
    arrays plus int32 offsets.  The reference order rebuilt from that copy
    (arrays(), decode_coo, a batch graph, the group kernel after set_kernel)
    is the oracle's conversion, byte for byte, and every path's SpMV is the
    oracle's."""
    dt = np.float64 if vt == S.F64 else np.float32
    mixed = vt == S.F32_V8
    for csr in (M.powerlaw(60_000, seed=21), M.dense(4096)):  # the dense rows run in segments
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols,
                         value_type=S.F32_V8 if mixed else None)
        m.set_kernel(S.KERNEL_SORTED)
        S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
        assert m.kernel == S.KERNEL_SORTED
        inf = m.info()
        nbr = (csr.nrows + r - 1) // r
        vbytes = 8 if vt == S.F64 else 4
        # headers + values once, int32 offsets (brptr, valptr, perm, sorted
        # offsets, partitions), and for the values of the chain part (the
        # largest block-rows) a 4-byte x index each plus, per chain, its
        # length and id (at most 8 bytes per value), and slice padding
        beta = inf.header_bytes + csr.nnz * vbytes
        assert inf.device_bytes <= 1.05 * beta + 12 * csr.nnz + 7 * 4 * (nbr + 1) + (1 << 20), \
            (csr.name, inf.device_bytes, inf.header_bytes, csr.nnz)
        conv = oracle.csr_to_beta_v8 if mixed else oracle.csr_to_beta
        ob, oh, ov = conv(r, csr.rowptr, csr.colidx, csr.values.astype(dt))
        gb, gh, gv = m.arrays()
        assert np.array_equal(gb, ob) and np.array_equal(gh, oh) and gv.tobytes() == ov.tobytes(), csr.name
        rows, cols, vals = (t.cpu().numpy() for t in S.decode_coo(m))
        if not mixed:
            orow, ocol, oval = oracle.beta_to_coo(r, csr.nrows, ob, oh, ov)
            assert np.array_equal(rows, orow) and np.array_equal(cols, ocol) and vals.tobytes() == oval.tobytes()
        order = np.lexsort((cols, rows))
        assert np.array_equal(cols[order], csr.colidx)
        assert vals[order].tobytes() == csr.values.astype(dt).tobytes()
        assert inf.device_bytes == m.info().device_bytes  # nothing kept by the rebuilds
        x = M.x_vector(csr.ncols, 5, dt)
        y0 = M.x_vector(csr.nrows, 6, np.float64 if mixed else dt)
        if mixed:
            yo = oracle.beta_spmv_mixed8(r, csr.nrows, ob, oh, ov, x, y0.copy())
        else:
            yo = oracle_spmv(dt, r, csr.nrows, ob, oh, ov, x, y0.copy())
        f = S.SPC5_Spmv_mixed if mixed else S.SPC5_Spmv
        y = dev(y0)
        f(m, dev(x), y)
        torch.cuda.synchronize()
        assert y.cpu().numpy().tobytes() == yo.tobytes(), (csr.name, "plan")
        m.set_kernel(S.KERNEL_GROUPS)  # runs on the rebuilt reference order
        y = dev(y0)
        f(m, dev(x), y)
        torch.cuda.synchronize()
        assert y.cpu().numpy().tobytes() == yo.tobytes(), (csr.name, "groups")
        m.set_kernel(S.KERNEL_SORTED)
        assert m.kernel == S.KERNEL_SORTED and m.info().device_bytes == inf.device_bytes
        # a batch graph reads the reference order: the handle keeps both copies
        Y = dev(y0[:, None].copy())
        b = S.Batch([m], [dev(x[:, None].copy())], [Y], mixed=mixed)
        b.launch()
        torch.cuda.synchronize()
        assert Y.cpu().numpy()[:, 0].tobytes() == yo.tobytes(), (csr.name, "batch")
        assert m.info().device_bytes > inf.device_bytes
        y = dev(y0)
        f(m, dev(x), y)
        torch.cuda.synchronize()
        assert y.cpu().numpy().tobytes() == yo.tobytes(), (csr.name, "plan after batch")


@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_mixed_precision(cuda, r):
    for csr in list(irregular_cases())[:5]:
        m = converted(csr, np.float32, r)
        brptr, headers, v32 = m.arrays()
        x = M.x_vector(csr.ncols, 5)
        x32 = x.astype(np.float32)
        y = torch.zeros(csr.nrows, dtype=torch.float64, device="cuda")
        S.SPC5_Spmv_mixed(m, dev(x32), y)
        torch.cuda.synchronize()
        y = y.cpu().numpy()
        yo = oracle.beta_spmv_mixed(r, csr.nrows, brptr, headers, v32, x32, np.zeros(csr.nrows))
        assert y.tobytes() == yo.tobytes(), csr.name
        y64, absrow = oracle.csr_spmv_f64(csr.rowptr, csr.colidx, csr.values, x, np.zeros(csr.nrows))
        if csr.nnz:
            assert np.abs(y - y64).max() / np.abs(y64).max() <= 1e-6
            assert (np.abs(y - y64) / np.maximum(absrow, 1e-300)).max() <= 2.5e-7


@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_mixed_precision_v8_layout(cuda, r):
    """F32_V8: float values in the 8-column layout.  Arrays equal the double
    conversion with values rounded to float; y equals the FP64 oracle on the
    widened values and x bit for bit (row kernel and sorted plan), and is
    within 1e-6 normwise of the FP64 CSR result on the unrounded inputs."""
    cases = list(irregular_cases()) + [M.powerlaw(60000, seed=5), M.stencil27(20)]
    for csr in cases:
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols, value_type=S.F32_V8)
        S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
        assert m.value_type == S.F32_V8 and m.info().vs == 8
        ob, oh, ov = oracle.csr_to_beta_v8(r, csr.rowptr, csr.colidx, csr.values)
        gb, gh, gv = m.arrays()
        assert np.array_equal(gb, ob) and np.array_equal(gh, oh) and gv.tobytes() == ov.tobytes(), csr.name
        x = M.x_vector(csr.ncols, 5)
        x32 = x.astype(np.float32)
        y0 = M.x_vector(csr.nrows, 6)
        y = dev(y0)
        for _ in range(3):
            S.SPC5_Spmv_mixed(m, dev(x32), y)
        torch.cuda.synchronize()
        yo = y0.copy()
        for _ in range(3):
            oracle.beta_spmv_mixed8(r, csr.nrows, ob, oh, ov, x32, yo)
        assert y.cpu().numpy().tobytes() == yo.tobytes(), csr.name
        if csr.nnz:
            y1 = torch.zeros(csr.nrows, dtype=torch.float64, device="cuda")
            S.SPC5_Spmv_mixed(m, dev(x32), y1)
            y1 = y1.cpu().numpy()
            y64, absrow = oracle.csr_spmv_f64(csr.rowptr, csr.colidx, csr.values, x, np.zeros(csr.nrows))
            assert np.abs(y1 - y64).max() / np.abs(y64).max() <= 1e-6
            assert (np.abs(y1 - y64) / np.maximum(absrow, 1e-300)).max() <= 2.5e-7
    # the plain calls reject the layout
    with pytest.raises(S.SPC5Error):
        S.SPC5_Spmv(m, dev(x32), dev(np.zeros(csr.nrows, np.float32)))


@pytest.mark.parametrize("r", [1, 4])
def test_mixed_v8_spmm_columns_equal_oracle(cuda, r):
    """Mixed SpMM on an F32_V8 matrix: every column equals the oracle's mixed
    SpMV of that column (staged SpMM and the sorted plan's SpMM)."""
    for csr in (M.banded(3000, 40, 0.2, seed=9), M.powerlaw(30000, seed=4)):
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols, value_type=S.F32_V8)
        S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
        ob, oh, ov = oracle.csr_to_beta_v8(r, csr.rowptr, csr.colidx, csr.values)
        k = 5
        X = np.stack([M.x_vector(csr.ncols, 20 + j).astype(np.float32) for j in range(k)], axis=1)
        Y = torch.zeros((csr.nrows, k), dtype=torch.float64, device="cuda")
        S.SPC5_Spmm_mixed(m, torch.from_numpy(np.ascontiguousarray(X)).cuda(), Y)
        torch.cuda.synchronize()
        Yh = Y.cpu().numpy()
        for j in range(k):
            yo = oracle.beta_spmv_mixed8(r, csr.nrows, ob, oh, ov, X[:, j].copy(), np.zeros(csr.nrows))
            assert Yh[:, j].tobytes() == yo.tobytes(), (csr.name, j)


def test_fp64_matches_csr_oracle_componentwise(cuda):
    csr = M.powerlaw(50000, seed=2)
    x = M.x_vector(csr.ncols, 6)
    y64, absrow = oracle.csr_spmv_f64(csr.rowptr, csr.colidx, csr.values, x, np.zeros(csr.nrows))
    for r in (1, 2, 4, 8):
        y = gpu_spmv(converted(csr, np.float64, r), x, np.zeros(csr.nrows))
        assert (np.abs(y - y64) / np.maximum(absrow, 1e-300)).max() <= 1e-13


def test_errors_are_status_codes(cuda):
    bad = M.CSR(2, 4, np.array([0, 2, 3], np.int32), np.array([3, 1, 0], np.int32), np.ones(3), "unsorted")
    with pytest.raises(S.SPC5Error) as e:
        S.csr_matrix(bad.rowptr, bad.colidx, bad.values, bad.ncols)
    assert e.value.status == 1
    out_of_range = M.CSR(1, 2, np.array([0, 1], np.int32), np.array([5], np.int32), np.ones(1), "oor")
    with pytest.raises(S.SPC5Error):
        S.csr_matrix(out_of_range.rowptr, out_of_range.colidx, out_of_range.values, out_of_range.ncols)
    a = M.poisson2d(8)
    m = S.csr_matrix(a.rowptr, a.colidx, a.values, a.ncols)
    with pytest.raises(S.SPC5Error) as e:
        S.CSR_to_SPC5(m, 9)
    assert e.value.status == 4
    with pytest.raises(S.SPC5Error):
        S.SPC5_Spmv(m, torch.zeros(64, dtype=torch.float64, device="cuda"),
                    torch.zeros(64, dtype=torch.float64, device="cuda"))
    S.CSR_to_SPC5(m, S.FORMAT_2rVc)
    with pytest.raises(S.SPC5Error):
        S.CSR_to_SPC5(m, S.FORMAT_4rVc)  # already converted
    with pytest.raises(S.SPC5Error):
        S.SPC5_Spmv_mixed(m, torch.zeros(64, dtype=torch.float32, device="cuda"),
                          torch.zeros(64, dtype=torch.float64, device="cuda"))
    with pytest.raises(S.SPC5Error):
        S.core_spmv(3, 64, *[torch.zeros(1, dtype=t, device="cuda") for t in
                             (torch.int32, torch.uint8, torch.float64, torch.float64, torch.float64)])


@pytest.mark.slow
@pytest.mark.parametrize("which", ["powerlaw", "stencil27"])
def test_full_size_bit_exact(cuda, which):
    """The full-size workloads: device conversion byte-identical and FP64 SpMV
    bit-identical to the oracle, for every r."""
    csr = M.powerlaw() if which == "powerlaw" else M.stencil27(160)
    x = M.x_vector(csr.ncols, 0)
    for r in (1, 2, 4, 8):
        brptr, headers, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, csr.values)
        m = converted(csr, np.float64, r)
        gb, gh, gv = m.arrays()
        assert np.array_equal(gb, brptr) and np.array_equal(gh, headers) and gv.tobytes() == ov.tobytes()
        yo = oracle.beta_spmv_f64(r, csr.nrows, brptr, headers, ov, x, np.zeros(csr.nrows))
        y = gpu_spmv(m, x, np.zeros(csr.nrows))
        assert y.tobytes() == yo.tobytes()
        del m


@pytest.mark.slow
def test_full_size_poisson_512(cuda):
    """The 5-point Poisson 512^2 workload (beta(2,8) is its headline format,
    every r is checked): conversion byte-identical and FP64 y bit-identical to
    the oracle's AVX-512 order, and componentwise within 1e-13 of the FP64
    scalar CSR product (CSR_Spmv_scalar, src/spc5.hpp:116-127)."""
    csr = M.poisson2d(512)
    x = M.x_vector(csr.ncols, 0)
    y64, absrow = oracle.csr_spmv_f64(csr.rowptr, csr.colidx, csr.values, x, np.zeros(csr.nrows))
    for r in (2, 1, 4, 8):
        brptr, headers, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, csr.values)
        m = converted(csr, np.float64, r)
        gb, gh, gv = m.arrays()
        assert np.array_equal(gb, brptr) and np.array_equal(gh, headers) and gv.tobytes() == ov.tobytes()
        y0 = M.x_vector(csr.nrows, 9)
        yo = oracle.beta_spmv_f64(r, csr.nrows, brptr, headers, ov, x, y0.copy())
        assert gpu_spmv(m, x, y0).tobytes() == yo.tobytes()
        y = gpu_spmv(m, x, np.zeros(csr.nrows))
        assert (np.abs(y - y64) / np.maximum(absrow, 1e-300)).max() <= 1e-13


@pytest.mark.slow
def test_full_size_stencil_f32_and_mixed(cuda):
    """The 27-point stencil 160^3 in the float layouts: FP32 (beta(r,16))
    and mixed bit-identical to the oracle, in the reference's float layout and
    in the 8-column layout; the mixed results within 1e-6 normwise and 2.5e-7
    per row (relative to sum_j |a_ij x_j|) of the FP64 CSR product."""
    csr = M.stencil27(160)
    x = M.x_vector(csr.ncols, 0)
    x32 = x.astype(np.float32)
    y64, absrow = oracle.csr_spmv_f64(csr.rowptr, csr.colidx, csr.values, x, np.zeros(csr.nrows))

    def close(y):
        assert np.abs(y - y64).max() / np.abs(y64).max() <= 1e-6
        assert (np.abs(y - y64) / np.maximum(absrow, 1e-300)).max() <= 2.5e-7

    r = 4
    v32 = csr.values.astype(np.float32)
    brptr, headers, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, v32)
    m = converted(csr, np.float32, r)
    gb, gh, gv = m.arrays()
    assert np.array_equal(gb, brptr) and np.array_equal(gh, headers) and gv.tobytes() == ov.tobytes()
    yf = dev(np.zeros(csr.nrows, np.float32))
    S.SPC5_Spmv(m, dev(x32), yf)
    yo = oracle.beta_spmv_f32(r, csr.nrows, brptr, headers, ov, x32, np.zeros(csr.nrows, np.float32))
    assert yf.cpu().numpy().tobytes() == yo.tobytes()
    ym = torch.zeros(csr.nrows, dtype=torch.float64, device="cuda")
    S.SPC5_Spmv_mixed(m, dev(x32), ym)
    torch.cuda.synchronize()
    ym = ym.cpu().numpy()
    assert ym.tobytes() == oracle.beta_spmv_mixed(r, csr.nrows, brptr, headers, ov, x32,
                                                  np.zeros(csr.nrows)).tobytes()
    close(ym)
    del m
    for r in (1, 4):
        b8, h8, v8 = oracle.csr_to_beta_v8(r, csr.rowptr, csr.colidx, csr.values)
        m8 = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols, value_type=S.F32_V8)
        S.CSR_to_SPC5(m8, S.FORMAT_OF_R[r])
        gb, gh, gv = m8.arrays()
        assert np.array_equal(gb, b8) and np.array_equal(gh, h8) and gv.tobytes() == v8.tobytes()
        y8 = torch.zeros(csr.nrows, dtype=torch.float64, device="cuda")
        S.SPC5_Spmv_mixed(m8, dev(x32), y8)
        torch.cuda.synchronize()
        y8 = y8.cpu().numpy()
        assert y8.tobytes() == oracle.beta_spmv_mixed8(r, csr.nrows, b8, h8, v8, x32, np.zeros(csr.nrows)).tobytes()
        close(y8)
        del m8


def oracle_spmv(dt, r, nrows, brptr, headers, vals, x, y):
    """The oracle's y += A x for the value type of the arrays."""
    f = oracle.beta_spmv_f64 if dt == np.float64 else oracle.beta_spmv_f32
    return f(r, nrows, brptr, headers, vals, x, y)


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("r", [1, 2, 4, 8])
@pytest.mark.parametrize("k", [1, 3, 4, 8, 16])
def test_spmm_columns_equal_spmv(cuda, tag, dt, r, k):
    """Every column of Y += A X equals an independent SpMV of that column,
    bit for bit (the request loop relies on it)."""
    for csr in list(irregular_cases())[:4]:
        m = converted(csr, dt, r)
        X = np.stack([M.x_vector(csr.ncols, 30 + j, dt) for j in range(k)], axis=1)
        Y0 = np.stack([M.x_vector(csr.nrows, 60 + j, dt) for j in range(k)], axis=1)
        Yd = dev(Y0)
        S.SPC5_Spmm(m, dev(X), Yd)
        torch.cuda.synchronize()
        Y = Yd.cpu().numpy()
        brptr, headers, ov = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, csr.values.astype(dt))
        for j in range(k):
            yj = oracle_spmv(dt, r, csr.nrows, brptr, headers, ov, np.ascontiguousarray(X[:, j]),
                             np.ascontiguousarray(Y0[:, j]))
            assert Y[:, j].tobytes() == yj.tobytes(), (csr.name, j)


@pytest.mark.parametrize("tag,dt", DTYPES + [("mixed", np.float32)])
@pytest.mark.parametrize("r", [1, 2, 4, 8])
def test_spmm_staged_and_group_bit_exact(cuda, tag, dt, r):
    """The staged SpMM (matrices whose block-rows fit the row kernels'
    buffers), the group SpMM (KERNEL_GROUPS) and the staged SpMM over the
    length-sorted plan (KERNEL_SORTED, and AUTO for block-rows too large,
    whose largest block-rows run in segments) give the oracle's SpMV bits in
    every column, for k = 1, 5 (passes of 4 + 1) and 16, with row-major X and
    Y of padded leading dimension."""
    mixed = tag == "mixed"
    f = oracle.beta_spmv_mixed if mixed else (oracle.beta_spmv_f64 if dt == np.float64 else oracle.beta_spmv_f32)
    ydt = np.float64 if mixed else dt
    for csr in kernel_cases():
        if csr.nnz > 400_000:
            continue
        for kernel in (S.KERNEL_AUTO, S.KERNEL_GROUPS, S.KERNEL_SORTED):
            m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols)
            m.set_kernel(kernel)
            S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
            brptr, headers, vals = m.arrays()
            for k in (1, 5, 16):
                X = np.zeros((csr.ncols, k + 3), dtype=dt)
                Y0 = np.zeros((csr.nrows, k + 2), dtype=ydt)
                for j in range(k):
                    X[:, j] = M.x_vector(csr.ncols, 70 + j, dt)
                    Y0[:, j] = M.x_vector(csr.nrows, 90 + j, ydt)
                Xd, Yd = dev(X), dev(Y0)
                (S.SPC5_Spmm_mixed if mixed else S.SPC5_Spmm)(m, Xd[:, :k], Yd[:, :k])
                torch.cuda.synchronize()
                Y = Yd.cpu().numpy()
                assert Y[:, k:].tobytes() == Y0[:, k:].tobytes()  # padding untouched
                for j in range(k):
                    yo = f(r, csr.nrows, brptr, headers, vals, np.ascontiguousarray(X[:, j]),
                           np.ascontiguousarray(Y0[:, j]))
                    assert Y[:, j].tobytes() == yo.tobytes(), (csr.name, kernel, k, j)


@pytest.mark.parametrize("r", [1, 4, 8])
def test_spmm_mixed_columns(cuda, r):
    csr = M.powerlaw(5000, seed=12)
    m = converted(csr, np.float32, r)
    k = 5
    X = np.stack([M.x_vector(csr.ncols, 40 + j, np.float32) for j in range(k)], axis=1)
    Yd = torch.zeros(csr.nrows, k, dtype=torch.float64, device="cuda")
    S.SPC5_Spmm_mixed(m, dev(X), Yd)
    torch.cuda.synchronize()
    brptr, headers, v32 = m.arrays()
    for j in range(k):
        yo = oracle.beta_spmv_mixed(r, csr.nrows, brptr, headers, v32, np.ascontiguousarray(X[:, j]),
                                    np.zeros(csr.nrows))
        assert Yd[:, j].cpu().numpy().tobytes() == yo.tobytes()


def test_find_best_matches_reference(cuda, golden):
    """SPC5_find_best on device block counts picks the reference's format."""
    for n in names(golden):
        csr = golden_csr(golden, n)
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
        r, est = S.SPC5_find_best(m)
        assert r == int(golden[f"{n}/find_best_r"]), n
        assert est == pytest.approx(float(golden[f"{n}/find_best_est"]), rel=1e-12), n


@pytest.mark.parametrize("mode", [S.TUNE_MODEL, S.TUNE_MEASURE])
def test_autotune(cuda, mode):
    for csr in (M.stencil27(20), M.powerlaw(30000, seed=4), M.banded(5000, 30, 0.2, seed=2)):
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
        t = S.autotune(m, mode)
        assert t["r"] in (1, 2, 4, 8)
        for r in (1, 2, 4, 8):
            assert t["blocks"][r] == oracle.block_count(r, csr.rowptr, csr.colidx)
            assert t["est_us"][r] > 0
        assert t["est_us"][t["r"]] == min(t["est_us"].values())
        assert m.format == S.FORMAT_CSR  # the autotuner leaves the handle untouched


@pytest.mark.parametrize("mixed", [False, True])
def test_batch_equals_independent_spmv(cuda, mixed):
    """One graph over matrices of uneven sizes, r and k: every column equals
    the oracle's SpMV bit for bit (mixed: F32 and F32_V8 matrices in one
    batch)."""
    rng = np.random.default_rng(5)
    mats, Xs, Ys, keep = [], [], [], []
    dt = np.float32 if mixed else np.float64
    for i in range(12):
        n = int(rng.integers(50, 6000))
        csr = M.banded(n, int(rng.integers(2, 60)), 0.3, seed=100 + i)
        r = (1, 2, 4, 8)[i % 4]
        k = (1, 4, 8, 16, 3)[i % 5]
        v8 = mixed and i % 2 == 1
        if v8:
            m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols, value_type=S.F32_V8)
            S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
        else:
            m = converted(csr, dt, r)
        X = dev(np.stack([M.x_vector(n, 200 + i * 20 + j, dt) for j in range(k)], axis=1))
        Y = torch.zeros(n, k, dtype=torch.float64 if mixed or dt == np.float64 else torch.float32,
                        device="cuda")
        mats.append(m); Xs.append(X); Ys.append(Y); keep.append((csr, r, v8))
    b = S.Batch(mats, Xs, Ys, mixed=mixed)
    nclasses, njobs = b.info()
    assert nclasses >= 4 and njobs >= 12
    for _ in range(2):  # y accumulates over two replays
        b.launch()
    torch.cuda.synchronize()
    for m, X, Y, (csr, r, v8) in zip(mats, Xs, Ys, keep):
        brptr, headers, vals = m.arrays()
        Xh, Yh = X.cpu().numpy(), Y.cpu().numpy()
        for j in range(X.shape[1]):
            xj = np.ascontiguousarray(Xh[:, j])
            y = np.zeros(csr.nrows, dtype=Yh.dtype)
            for _ in range(2):
                if v8:
                    oracle.beta_spmv_mixed8(r, csr.nrows, brptr, headers, vals, xj, y)
                elif mixed:
                    oracle.beta_spmv_mixed(r, csr.nrows, brptr, headers, vals, xj, y)
                else:
                    oracle_spmv(dt, r, csr.nrows, brptr, headers, vals, xj, y)
            assert Yh[:, j].tobytes() == y.tobytes(), (csr.name, r, j)
