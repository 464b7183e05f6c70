"""Multi-GPU SpMV: block-row sharding and the x all-gather.

One process per GPU (``torch.distributed``, NCCL over NVLink for CUDA
tensors).  Rank k owns a contiguous range of rows cut at a block-row
boundary (a multiple of r), so its block-rows -- and therefore the blocks,
headers, values and the FP64 result of every row -- are exactly those of the
single-GPU matrix: the concatenated y is bit-identical to one SpMV of the
whole matrix.  The cuts balance nnz (the GPU analogue of the reference's
block-balanced ``core_SPC5_rVc_threadsplit``, src/spc5.hpp:346-387; ``by``
selects "nnz" or "blocks").

* ``y = A x`` once: every rank holds the full x (replicated) and computes
  its y slice; no collective on the data path.
* iterative use (x_{t+1} = A x_t, square A): each rank holds only its x
  slice; ``iterate`` all-gathers the slices (one ``all_gather_into_tensor``
  of ~N * 8 bytes over NVLink), then runs its local SpMV.  With equal-width
  cuts (``cuts="equal"``: every rank but the last owns ``width`` rows, a
  multiple of r) the gathered buffer is x itself: NCCL writes every slice in
  place and the local SpMV reads a view of it, with no copy of x per
  iteration.  Other cuts gather into a padded buffer and pack it once.
"""
from __future__ import annotations

import numpy as np

from .matrices import CSR


def partition_rows(rowptr, world: int, r: int = 1, weights=None):
    """Contiguous row ranges [cut[k], cut[k+1]) for ``world`` ranks.  Every
    cut is a multiple of r (or nrows); the cuts balance the per-row
    ``weights`` (default: nnz per row)."""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    n = len(rowptr) - 1
    if weights is None:
        cum = rowptr
    else:
        w = np.asarray(weights, dtype=np.int64)
        cum = np.concatenate([[0], np.cumsum(w)])
    total = int(cum[-1])
    nbr = (n + r - 1) // r
    brow_cum = cum[np.minimum(np.arange(nbr + 1) * r, n)]  # weight before each block-row
    cuts = [0]
    for k in range(1, world):
        target = total * k / world
        br = int(np.searchsorted(brow_cum, target, side="left"))
        br = max(br, (cuts[-1] + r - 1) // r)
        cuts.append(min(n, br * r))
    cuts.append(n)
    return np.asarray(cuts, dtype=np.int64)


def equal_cuts(nrows: int, world: int, r: int = 1):
    """Cuts of equal width (a multiple of r) for ``world`` ranks; the last
    range is the remainder (possibly shorter or empty)."""
    per = (nrows + world - 1) // world
    width = ((per + r - 1) // r) * r
    return np.asarray([min(nrows, k * width) for k in range(world)] + [nrows], dtype=np.int64)


def row_slice(csr: CSR, r0: int, r1: int) -> CSR:
    """Rows [r0, r1) of a CSR matrix, all columns kept."""
    a, b = int(csr.rowptr[r0]), int(csr.rowptr[r1])
    return CSR(r1 - r0, csr.ncols, (csr.rowptr[r0:r1 + 1] - a).astype(np.int32), csr.colidx[a:b],
               csr.values[a:b], f"{csr.name}[{r0}:{r1}]")


class ShardedSpMV:
    """This rank's block-row shard of A in beta(r,VS) on its GPU."""

    def __init__(self, csr: CSR, rank: int, world: int, r: int, device, dtype=np.float64,
                 cuts=None):
        """``cuts``: None or "nnz" (nnz-balanced, block-row aligned), "equal"
        (equal widths: the zero-copy gather of ``iterate``), or an array of
        world + 1 row boundaries."""
        self.rank, self.world, self.r = rank, world, r
        if cuts is None or (isinstance(cuts, str) and cuts == "nnz"):
            self.cuts = partition_rows(csr.rowptr, world, r)
        elif isinstance(cuts, str) and cuts == "equal":
            self.cuts = equal_cuts(csr.nrows, world, r)
        else:
            self.cuts = np.asarray(cuts, dtype=np.int64)
        counts = np.diff(self.cuts)
        self.width = max(1, int(counts.max())) if len(counts) else 1
        # the gathered buffer is x itself when rank k's slice starts at
        # k * width (every slice but the trailing ones has the full width)
        self.in_place = bool(all(int(self.cuts[k]) == min(csr.nrows, k * self.width) for k in range(world)))
        self._xbuf = None
        self.r0, self.r1 = int(self.cuts[rank]), int(self.cuts[rank + 1])
        self.nrows, self.ncols = csr.nrows, csr.ncols
        self.local = row_slice(csr, self.r0, self.r1)
        self.device = device
        self.dtype = dtype
        self.mat = self._build(self.local)

    # The local compute; a CPU test may substitute another implementation.
    def _build(self, local: CSR):
        from . import CSR_to_SPC5, FORMAT_OF_R, csr_matrix
        m = csr_matrix(local.rowptr, local.colidx, local.values.astype(self.dtype), local.ncols)
        CSR_to_SPC5(m, FORMAT_OF_R[self.r])
        return m

    def local_spmv(self, x_full, y_local) -> None:
        """y_local += A[r0:r1, :] x_full."""
        from . import SPC5_Spmv
        SPC5_Spmv(self.mat, x_full, y_local)

    def spmv(self, x_full, y_local):
        """One-shot y = A x with replicated x: this rank's slice of y."""
        self.local_spmv(x_full, y_local)
        return y_local

    def gather_x(self, x_local, group=None):
        """All-gather the ranks' x slices into the full x (one collective).
        With equal-width cuts the result is a view of the gather buffer (no
        copy of x); otherwise the padded slices are packed once."""
        import torch
        import torch.distributed as dist
        if self.world == 1:
            return x_local
        w = self.width
        if self._xbuf is None or self._xbuf.dtype != x_local.dtype or self._xbuf.device != x_local.device:
            self._xbuf = torch.empty(w * self.world, dtype=x_local.dtype, device=x_local.device)
            self._xsend = torch.zeros(w, dtype=x_local.dtype, device=x_local.device)
        send = x_local
        if x_local.numel() != w:  # a shorter (last) slice: padded to the width
            self._xsend[: x_local.numel()].copy_(x_local)
            send = self._xsend
        dist.all_gather_into_tensor(self._xbuf, send, group=group)
        if self.in_place:
            return self._xbuf[: self.ncols]
        counts = np.diff(self.cuts)
        return torch.cat([self._xbuf[k * w: k * w + int(counts[k])] for k in range(self.world)])

    def iterate(self, x_local, group=None):
        """x_next slice = A[r0:r1, :] x for a square A whose x is sharded like y."""
        import torch
        if self.nrows != self.ncols:
            raise ValueError("iterate needs a square matrix")
        x_full = self.gather_x(x_local, group)
        y = torch.zeros(self.r1 - self.r0, dtype=x_local.dtype, device=x_local.device)
        self.local_spmv(x_full, y)
        return y
