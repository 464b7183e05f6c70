"""Multi-rank sharding on CPU (gloo, world size 2).

The sharded path's host logic -- block-row aligned, nnz-balanced cuts, the x
all-gather and the y concatenation -- runs on two gloo ranks; each rank's
local SpMV is the oracle restatement of the reference kernel (CPU), so the
concatenated result must equal the single-matrix oracle result bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from spc5_b200 import distributed as D
from spc5_b200 import matrices as M


class OracleShard(D.ShardedSpMV):
    def _build(self, local):
        return oracle.csr_to_beta(self.r, local.rowptr, local.colidx, local.values)

    def local_spmv(self, x_full, y_local):
        brptr, headers, vals = self.mat
        y = y_local.numpy()
        oracle.beta_spmv_f64(self.r, self.local.nrows, brptr, headers, vals, x_full.numpy(), y)


def test_partition_properties():
    csr = M.powerlaw(30000, seed=2)
    for world in (1, 2, 3, 8):
        for r in (1, 2, 4, 8):
            cuts = D.partition_rows(csr.rowptr, world, r)
            assert cuts[0] == 0 and cuts[-1] == csr.nrows and len(cuts) == world + 1
            assert np.all(np.diff(cuts) >= 0)
            assert all(c % r == 0 or c == csr.nrows for c in cuts)
            loads = np.diff(csr.rowptr[cuts])
            if world > 1:
                assert loads.max() <= csr.nnz / world + csr.rowptr[min(csr.nrows, 8)] + 2000 * r


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_equal_cuts_properties():
    for n in (1, 7, 1000, 6001):
        for world in (1, 2, 3, 8):
            for r in (1, 4, 8):
                cuts = D.equal_cuts(n, world, r)
                counts = np.diff(cuts)
                assert cuts[0] == 0 and cuts[-1] == n and len(cuts) == world + 1
                assert np.all(counts >= 0) and all(c % r == 0 or c == n for c in cuts)
                width = counts.max()
                assert all(cuts[k] == min(n, k * width) for k in range(world))


def _worker(rank, world, port, r, out_path, cuts="nnz"):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        csr = M.powerlaw(6000, seed=11)
        x = torch.from_numpy(M.x_vector(csr.ncols, 3))
        sh = OracleShard(csr, rank, world, r, device="cpu", cuts=cuts)
        if cuts == "equal":
            assert sh.in_place
        # one-shot, replicated x
        y_local = torch.zeros(sh.r1 - sh.r0, dtype=torch.float64)
        sh.spmv(x, y_local)
        # iterative: sharded x, all-gathered each step
        x_local = x[sh.r0:sh.r1].clone()
        for _ in range(3):
            x_local = sh.iterate(x_local)
        parts = [None] * world
        dist.all_gather_object(parts, (y_local.numpy().tobytes(), x_local.numpy().tobytes()))
        if rank == 0:
            np.savez(out_path, y=np.frombuffer(b"".join(p[0] for p in parts), dtype=np.float64),
                     x=np.frombuffer(b"".join(p[1] for p in parts), dtype=np.float64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("r,cuts", [(1, "nnz"), (4, "nnz"), (1, "equal"), (8, "equal")])
def test_two_ranks_match_single_matrix(r, cuts, tmp_path):
    """The real ShardedSpMV host path on two gloo ranks -- the block-row
    aligned cuts, the x all-gather (in place for equal-width cuts, packed
    otherwise) and iterate -- with the oracle as each rank's local SpMV."""
    out = str(tmp_path / "ranks.npz")
    port = _free_port()
    mp.spawn(_worker, args=(2, port, r, out, cuts), nprocs=2, join=True)
    got = np.load(out)
    csr = M.powerlaw(6000, seed=11)
    x = M.x_vector(csr.ncols, 3)
    brptr, headers, vals = oracle.csr_to_beta(r, csr.rowptr, csr.colidx, csr.values)
    y_full = oracle.beta_spmv_f64(r, csr.nrows, brptr, headers, vals, x, np.zeros(csr.nrows))
    assert got["y"].tobytes() == y_full.tobytes()
    xi = x.copy()
    for _ in range(3):
        xi = oracle.beta_spmv_f64(r, csr.nrows, brptr, headers, vals, xi, np.zeros(csr.nrows))
    assert got["x"].tobytes() == xi.tobytes()
