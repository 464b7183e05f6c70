"""Serving on several GPUs: whole matrices placed per GPU, replicas for hot ones.

SpMV requests need no exchange between GPUs: a matrix lives whole on every
GPU that serves it, and a request runs where its matrix is.  This module
holds the host side of that:

* ``place_matrices`` -- which GPUs hold which matrix.  The expected load of a
  matrix is its share of the requests times its footprint (an SpMV's time
  grows with the bytes it reads).  A matrix whose load is above one GPU's
  fair share (total load / GPUs) gets enough replicas that each carries at
  most that share.  Replicas are placed greedily, heaviest per-replica load
  first, on the GPU with the least load that still has room and does not
  hold the matrix yet.
* ``Router`` -- a request goes to the replica with the fewest outstanding
  requests (ties: the lowest GPU index).
* ``MultiServer`` -- one ``Server`` (the request loop of ``csrc/serve.cu``) per
  GPU, the matrices converted on every GPU that holds them, and the router in
  front.  Every replica holds the same beta(r,VS) arrays, so a request's
  result is the same bits on whichever GPU it runs.
"""
from __future__ import annotations

import math

import numpy as np


def place_matrices(footprints, shares, n_gpus: int, capacity):
    """Placement of matrices on ``n_gpus`` GPUs.

    footprints: device bytes of each matrix (one replica); shares: expected
    fraction of the requests for each matrix (any non-negative weights, they
    are normalised); capacity: bytes each GPU may hold (a number, or one per
    GPU).  Returns ``(placement, load, used)``: ``placement[i]`` is the sorted
    list of GPUs holding matrix i, ``load[g]`` the expected load of GPU g
    (share x bytes, summed over its replicas, a replica carrying its matrix's
    load / replicas) and ``used[g]`` its bytes.  Raises ValueError when a
    matrix fits on no GPU; a hot matrix gets fewer replicas than it wants
    when room runs out, never fewer than one.
    """
    fp = np.asarray(footprints, dtype=np.float64)
    sh = np.asarray(shares, dtype=np.float64)
    if fp.shape != sh.shape:
        raise ValueError("footprints and shares differ in length")
    if n_gpus < 1:
        raise ValueError("n_gpus must be >= 1")
    if np.any(fp < 0) or np.any(sh < 0):
        raise ValueError("footprints and shares must be non-negative")
    cap = np.broadcast_to(np.asarray(capacity, dtype=np.float64), (n_gpus,)).copy()
    total = sh.sum()
    sh = sh / total if total > 0 else np.full_like(sh, 1.0 / max(1, len(sh)))
    load_of = sh * fp
    fair = load_of.sum() / n_gpus
    want = [1 if fair <= 0 else int(min(n_gpus, max(1, math.ceil(l / fair - 1e-9)))) for l in load_of]

    placement = [[] for _ in range(len(fp))]
    load = np.zeros(n_gpus)
    used = np.zeros(n_gpus)
    # every replica, heaviest per-replica load first (longest processing time
    # first: each goes to the least loaded GPU with room); a matrix's first
    # replica must find room, an extra one may not
    def put(i, per_replica):
        best = None
        for g in range(n_gpus):
            if g in placement[i] or used[g] + fp[i] > cap[g]:
                continue
            if best is None or load[g] < load[best]:
                best = g
        if best is None:
            return False
        placement[i].append(best)
        used[best] += fp[i]
        load[best] += per_replica
        return True

    items = sorted(((load_of[i] / want[i], i, k) for i in range(len(fp)) for k in range(want[i])),
                   key=lambda t: (-t[0], -fp[t[1]], t[1], t[2]))
    for per, i, k in items:
        if not put(i, per) and not placement[i]:
            raise ValueError(f"matrix {i} ({int(fp[i])} bytes) fits on no GPU")
    # a matrix that got fewer replicas than it wanted spreads its load over
    # those it has
    load = np.zeros(n_gpus)
    for i, gs in enumerate(placement):
        for g in gs:
            load[g] += load_of[i] / len(gs)
    return [sorted(gs) for gs in placement], load, used


class Router:
    """Picks, for each request, the replica with the fewest outstanding
    requests (ties: the lowest GPU index)."""

    def __init__(self, placement, n_gpus: int):
        self.placement = [list(gs) for gs in placement]
        self.outstanding = [0] * n_gpus

    def pick(self, mat: int) -> int:
        gs = self.placement[mat]
        if not gs:
            raise ValueError(f"matrix {mat} is not placed")
        g = min(gs, key=lambda g: (self.outstanding[g], g))
        self.outstanding[g] += 1
        return g

    def done(self, gpu: int) -> None:
        self.outstanding[gpu] -= 1


class MultiServer:
    """Request loop over several GPUs of one node (one ``Server`` per GPU).

    ``add_matrices(csrs, shares)`` places the matrices (``place_matrices``),
    converts each on every GPU that holds it and registers it with that GPU's
    server.  ``submit(mat, x, y)`` copies x to the chosen GPU, queues
    ``y = A x`` there and returns a request id; ``wait(rid)`` copies the result
    into y (any device) and returns the latency in microseconds seen by that
    GPU's request loop.  A wait that raises (a timeout, a device error) keeps
    the request outstanding, so the caller can wait on it again.

    The device work goes through the methods ``_device_count``, ``_device``,
    ``_free_bytes``, ``_new_server``, ``_convert``, ``_stage`` and
    ``_copy_out``, so that the placement, routing and bookkeeping can be
    exercised without GPUs.
    """

    def __init__(self, n_gpus=None, slots=4, max_k=16, mixed=False, hbm_fraction=0.9):
        self.slots, self.max_k = int(slots), int(max_k)
        self.n = self._device_count() if n_gpus is None else int(n_gpus)
        if self.n < 1:
            raise RuntimeError("MultiServer needs a CUDA device")
        self.mixed = bool(mixed)
        self.capacity = []
        self.servers = []
        for g in range(self.n):
            with self._device(g):
                free = self._free_bytes()
                self.capacity.append(int(free * hbm_fraction))
                self.servers.append(self._new_server(int(free * hbm_fraction)))
        self.placement = []
        self.ids = []      # per matrix: {gpu: id on that gpu's server}
        self.handles = []  # keeps the per-GPU handles alive
        self.router = None
        self._reqs = {}
        self._next = 1

    # ---- device hooks ---------------------------------------------------
    def _device_count(self) -> int:
        import torch
        return torch.cuda.device_count()

    def _device(self, g):
        import torch
        return torch.cuda.device(g)

    def _free_bytes(self) -> int:
        import torch
        free, _ = torch.cuda.mem_get_info()
        return int(free)

    def _new_server(self, budget: int):
        from . import Server
        return Server(slots=self.slots, max_k=self.max_k, mixed=self.mixed, hbm_budget=budget)

    def _convert(self, csr, fmt):
        """A converted handle of ``csr`` on the current device."""
        from . import CSR_to_SPC5, csr_matrix
        dt = np.float32 if self.mixed else np.float64
        m = csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols)
        CSR_to_SPC5(m, fmt)
        return m

    def _stage(self, g, x, nrows):
        """x on GPU g and a result vector there; the request loop's stream
        must see the copy of x."""
        import torch
        dev = torch.device("cuda", g)
        xg = x.to(dev, non_blocking=True)
        yg = torch.empty(nrows, dtype=torch.float64, device=dev)
        torch.cuda.current_stream(dev).synchronize()
        return xg, yg

    def _copy_out(self, y, yg) -> None:
        y.copy_(yg)

    # ---- requests ---------------------------------------------------------
    def add_matrices(self, csrs, shares, formats):
        """Places and registers ``csrs`` (``matrices.CSR``); ``formats[i]`` is
        the beta(r,VS) format of matrix i (``FORMAT_OF_R[r]``)."""
        # footprint of one replica: measured on the first GPU that converts it
        footprints = []
        for csr, fmt in zip(csrs, formats):
            with self._device(0):
                m = self._convert(csr, fmt)
                footprints.append(int(m.info().device_bytes))
                del m
        # every server also keeps its slots' staging blocks (max_k columns of
        # X and Y per slot, sized for the largest matrix it holds): reserve
        # them for the largest matrix of this batch
        xb = 4 if self.mixed else 8
        staging = self.slots * self.max_k * (max(c.ncols for c in csrs) * xb + max(c.nrows for c in csrs) * 8)
        room = [c - s.stats()["resident_bytes"] - staging for c, s in zip(self.capacity, self.servers)]
        placement, _, _ = place_matrices(footprints, shares, self.n, room)
        base = len(self.placement)
        for i, (csr, fmt) in enumerate(zip(csrs, formats)):
            ids = {}
            for g in placement[i]:
                with self._device(g):
                    m = self._convert(csr, fmt)
                    ids[g] = self.servers[g].add_matrix(m)
                    self.handles.append(m)
            self.placement.append(placement[i])
            self.ids.append(ids)
        if self.router is None:
            self.router = Router(self.placement, self.n)
        else:
            # keep the outstanding counts of requests already submitted
            self.router.placement = [list(gs) for gs in self.placement]
        return list(range(base, base + len(csrs)))

    def submit(self, mat: int, x, y) -> int:
        g = self.router.pick(mat)
        try:
            with self._device(g):
                xg, yg = self._stage(g, x, y.shape[0])
                rid = self.servers[g].submit(self.ids[mat][g], xg, yg)
        except BaseException:
            self.router.done(g)
            raise
        key = self._next
        self._next += 1
        self._reqs[key] = (g, rid, xg, yg, y)
        return key

    def wait(self, key: int, timeout_s: float = 60.0) -> float:
        g, rid, _, yg, y = self._reqs[key]
        lat = self.servers[g].wait(rid, timeout_s)  # raises: still outstanding
        self._copy_out(y, yg)
        del self._reqs[key]
        self.router.done(g)
        return lat

    def outstanding(self) -> list:
        """Requests submitted and not yet waited for, per GPU."""
        return list(self.router.outstanding) if self.router else [0] * self.n

    def gpu_of(self, key: int) -> int:
        return self._reqs[key][0]

    def close(self) -> None:
        for s in self.servers:
            s.close()
