"""The request loop: continuous batching over resident matrices.

Each request's result must be identical, bit for bit, whether it runs alone
or coalesced with other requests to the same matrix while other launches
overlap on the device; admission by HBM footprint must reject a matrix that
does not fit the budget.
"""
import numpy as np
import pytest
import torch

import spc5_b200 as S
from spc5_b200 import matrices as M

pytestmark = pytest.mark.gpu


def converted(csr, dt, r):
    m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols)
    S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
    return m


def solo(m, x, mixed):
    y = torch.zeros(m.numberOfRows, dtype=torch.float64, device="cuda")
    (S.SPC5_Spmv_mixed if mixed else S.SPC5_Spmv)(m, x, y)
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("vt", [S.F64, S.F32, S.F32_V8])
def test_results_same_alone_and_in_the_mix(cuda, vt):
    mixed = vt != S.F64
    dt = np.float32 if mixed else np.float64
    tdt = torch.float32 if mixed else torch.float64
    csrs = [M.powerlaw(20000, seed=3), M.stencil27(18), M.banded(7000, 40, 0.2, seed=5)]
    if vt == S.F32_V8:
        mats = []
        for c, r in zip(csrs, (1, 4, 2)):
            m = S.csr_matrix(c.rowptr, c.colidx, c.values, c.ncols, value_type=S.F32_V8)
            S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
            mats.append(m)
    else:
        mats = [converted(c, dt, r) for c, r in zip(csrs, (1, 4, 2))]
    srv = S.Server(slots=3, max_k=16, mixed=mixed)
    ids = [srv.add_matrix(m) for m in mats]
    rng = np.random.default_rng(0)
    work = []
    for q in range(300):
        i = int(rng.integers(0, len(mats)))
        x = torch.from_numpy(M.x_vector(csrs[i].ncols, 1000 + q, dt)).cuda()
        y = torch.full((csrs[i].nrows,), float("nan"), dtype=torch.float64, device="cuda")
        work.append((i, x, y))
    torch.cuda.synchronize()
    # a burst: requests arrive while earlier launches are still in flight
    reqs = [(i, x, y, srv.submit(ids[i], x, y)) for i, x, y in work]
    for _, _, _, rid in reqs:
        assert srv.wait(rid) >= 0.0
    for i, x, y, _ in reqs:
        assert y.cpu().numpy().tobytes() == solo(mats[i], x, mixed).cpu().numpy().tobytes()
    st = srv.stats()
    assert st["completed"] == 300 and st["launches"] < 300 and st["mean_k"] > 1.0
    assert st["p99_us"] >= st["p50_us"] > 0
    # alone: one request at a time
    for i, x, y, _ in reqs[:20]:
        y2 = torch.empty_like(y)
        srv.wait(srv.submit(ids[i], x, y2))
        assert y2.cpu().numpy().tobytes() == y.cpu().numpy().tobytes()
    srv.close()
    del tdt


def test_bounded_wait_times_out_then_drains(cuda):
    """wait() with a zero timeout on a request queued behind work returns
    SPC5CUDA_ERR_TIMEOUT (6) without touching the request; drain() then
    completes everything and the result equals a solo SpMV.  No device
    spin: the timeout is on the host's wait for the completion event."""
    csr = M.powerlaw(400_000, seed=12)
    m = converted(csr, np.float64, 1)
    srv = S.Server(slots=1, max_k=16)
    mid = srv.add_matrix(m)
    x = torch.from_numpy(M.x_vector(csr.ncols, 77)).cuda()
    timed_out = False
    for burst in (64, 256, 1024):
        ys = [torch.zeros(csr.nrows, dtype=torch.float64, device="cuda") for _ in range(burst)]
        torch.cuda.synchronize()
        rids = [srv.submit(mid, x, y) for y in ys]
        try:
            srv.wait(rids[-1], timeout_s=0.0)
        except S.SPC5Error as e:
            assert e.status == 6
            timed_out = True
        srv.drain(timeout_s=120.0)
        ref = solo(m, x, False).cpu().numpy().tobytes()
        assert ys[-1].cpu().numpy().tobytes() == ref and ys[0].cpu().numpy().tobytes() == ref
        del ys
        if timed_out:
            break
    assert timed_out
    srv.close()


def test_admission_by_hbm_footprint(cuda):
    csr = M.stencil27(20)
    m = converted(csr, np.float64, 4)
    small = S.Server(slots=2, max_k=4, hbm_budget=m.info().device_bytes // 2)
    with pytest.raises(S.SPC5Error) as e:
        small.add_matrix(m)
    assert e.value.status == 3
    ok = S.Server(slots=2, max_k=4, hbm_budget=1 << 30)
    assert ok.add_matrix(m) == 0
    assert ok.stats()["resident_bytes"] == m.info().device_bytes
    small.close()
    ok.close()


def test_wrong_value_type_rejected(cuda):
    m = converted(M.poisson2d(16), np.float64, 2)
    srv = S.Server(slots=1, max_k=2, hbm_budget=1 << 28, mixed=True)
    with pytest.raises(S.SPC5Error):
        srv.add_matrix(m)
    srv.close()


@pytest.mark.parametrize("r", [1, 4])
def test_shards_concatenate_to_full_spmv(cuda, r):
    """Block-row shards (as each rank of a multi-GPU run builds them), run one
    after the other on this GPU: the concatenated y equals the full SpMV."""
    from spc5_b200 import distributed as D
    csr = M.powerlaw(40000, seed=8)
    x = torch.from_numpy(M.x_vector(csr.ncols, 2)).cuda()
    full = converted(csr, np.float64, r)
    y_full = torch.zeros(csr.nrows, dtype=torch.float64, device="cuda")
    S.SPC5_Spmv(full, x, y_full)
    for world in (2, 3):
        parts = []
        for rank in range(world):
            sh = D.ShardedSpMV(csr, rank, world, r, device="cuda")
            y = torch.zeros(sh.r1 - sh.r0, dtype=torch.float64, device="cuda")
            parts.append(sh.spmv(x, y))
        torch.cuda.synchronize()
        assert torch.cat(parts).cpu().numpy().tobytes() == y_full.cpu().numpy().tobytes()


def test_multi_server_places_routes_and_matches_solo(cuda):
    """MultiServer over the GPUs of this run: the placement covers every
    matrix, and each request's result equals a solo SpMV bit for bit on
    whichever GPU the router picked."""
    from spc5_b200 import serving as SV
    n = torch.cuda.device_count()
    csrs = [M.powerlaw(20000, seed=3), M.stencil27(18), M.banded(7000, 40, 0.2, seed=5)]
    rs = (1, 4, 2)
    ms = SV.MultiServer(n_gpus=n, slots=2, max_k=8)
    ids = ms.add_matrices(csrs, [0.6, 0.3, 0.1], [S.FORMAT_OF_R[r] for r in rs])
    assert all(len(gs) >= 1 for gs in ms.placement)
    mats = [converted(c, np.float64, r) for c, r in zip(csrs, rs)]
    pending = []
    for q in range(24):
        i = q % 3
        x = torch.from_numpy(M.x_vector(csrs[i].ncols, 50 + q, np.float64)).cuda()
        y = torch.empty(csrs[i].nrows, dtype=torch.float64, device="cuda")
        pending.append((i, x, y, ms.submit(ids[i], x, y)))
    for i, x, y, rid in pending:
        assert ms.wait(rid) >= 0.0
        assert y.cpu().numpy().tobytes() == solo(mats[i], x, False).cpu().numpy().tobytes()
    assert all(v == 0 for v in ms.router.outstanding)
    ms.close()
