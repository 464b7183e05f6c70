"""Placement of whole matrices on several GPUs and request routing (host
logic of spc5_b200.serving; no GPU)."""
import numpy as np
import pytest

from spc5_b200 import serving as SV


def zipf_shares(n, s=1.1):
    w = 1.0 / np.arange(1, n + 1) ** s
    return w / w.sum()


def check(placement, load, used, fp, cap, n_gpus):
    assert all(len(gs) >= 1 for gs in placement)
    assert all(len(set(gs)) == len(gs) and all(0 <= g < n_gpus for g in gs) for gs in placement)
    held = np.zeros(n_gpus)
    for i, gs in enumerate(placement):
        for g in gs:
            held[g] += fp[i]
    assert np.allclose(held, used) and np.all(used <= np.broadcast_to(cap, (n_gpus,)) + 1e-6)


def test_every_matrix_placed_within_capacity():
    rng = np.random.default_rng(0)
    fp = rng.integers(10**8, 2 * 10**9, size=64).astype(float)
    sh = zipf_shares(64)
    for n in (1, 2, 4, 8):
        cap = fp.sum() / n * 1.5 + 2e9
        placement, load, used = SV.place_matrices(fp, sh, n, cap)
        check(placement, load, used, fp, cap, n)
        assert np.isclose(load.sum(), (sh * fp).sum())


def test_hot_matrix_is_replicated_and_load_balanced():
    fp = np.full(16, 1e9)
    sh = np.full(16, 0.1 / 15)
    sh[0] = 0.9  # one matrix takes 90% of the requests
    placement, load, used = SV.place_matrices(fp, sh, 4, 40e9)
    check(placement, load, used, fp, 40e9, 4)
    assert len(placement[0]) == 4  # its load is 3.6 fair shares: a replica on every GPU
    fair = load.sum() / 4
    assert load.max() <= 1.2 * fair


def test_zipf_pool_balances_on_eight_gpus():
    # the serving bench's pool: 8 distinct sizes, each registered 8 times
    sizes = np.array([0.03, 0.6, 0.2, 1.4, 0.6, 2.7, 1.3, 5.5]) * 1e9
    fp = np.tile(sizes, 8)
    sh = zipf_shares(64)
    placement, load, used = SV.place_matrices(fp, sh, 8, 60e9)
    check(placement, load, used, fp, 60e9, 8)
    fair = load.sum() / 8
    assert load.max() <= 1.3 * fair


def test_room_limits_replicas_not_placement():
    fp = np.array([4e9, 1e9, 1e9])
    sh = np.array([0.98, 0.01, 0.01])
    # each GPU has room for the hot matrix and one small one: the hot one
    # still gets a replica wherever it fits
    placement, load, used = SV.place_matrices(fp, sh, 3, 5.5e9)
    check(placement, load, used, fp, 5.5e9, 3)
    assert len(placement[0]) >= 2
    with pytest.raises(ValueError):
        SV.place_matrices([8e9], [1.0], 2, 5e9)  # fits on no GPU
    with pytest.raises(ValueError):
        SV.place_matrices([1e9, 1e9], [1.0], 2, 5e9)  # lengths differ


def test_router_least_outstanding():
    rt = SV.Router([[0, 1], [1], [2, 0]], 3)
    assert rt.pick(0) == 0          # tie: lowest index
    assert rt.pick(0) == 1          # GPU 0 has one outstanding
    assert rt.pick(1) == 1
    assert rt.pick(2) == 2
    assert rt.pick(0) == 0          # 0 has 1, 1 has 2
    rt.done(1)
    rt.done(1)
    assert rt.pick(0) == 1          # 1 has 0 now
    with pytest.raises(ValueError):
        SV.Router([[]], 1).pick(0)


# ---- MultiServer bookkeeping over several (fake) GPUs ------------------------

class _FakeInfo:
    def __init__(self, n):
        self.device_bytes = n


class _FakeHandle:
    def __init__(self, csr):
        self.csr = csr

    def info(self):
        return _FakeInfo(int(self.csr.nnz) * 12 + 64)


class _FakeServer:
    """Stands in for one GPU's request loop: y = (matrix id + 1) * sum(x)."""

    def __init__(self):
        self.mats, self.reqs, self.next, self.fail_waits = [], {}, 1, 0

    def add_matrix(self, m):
        self.mats.append(m)
        return len(self.mats) - 1

    def submit(self, mid, x, y):
        rid = self.next
        self.next += 1
        self.reqs[rid] = (mid, x, y)
        return rid

    def wait(self, rid, timeout_s):
        if self.fail_waits:
            self.fail_waits -= 1
            raise TimeoutError("request not finished")
        mid, x, y = self.reqs.pop(rid)
        y[:] = (mid + 1) * float(np.sum(x))
        return 10.0

    def stats(self):
        return {"resident_bytes": sum(m.info().device_bytes for m in self.mats)}

    def close(self):
        pass


class _FakeMulti(SV.MultiServer):
    def _device_count(self):
        return 4

    def _device(self, g):
        import contextlib
        return contextlib.nullcontext()

    def _free_bytes(self):
        return 10**9

    def _new_server(self, budget):
        return _FakeServer()

    def _convert(self, csr, fmt):
        return _FakeHandle(csr)

    def _stage(self, g, x, nrows):
        return np.array(x, copy=True), np.zeros(nrows)

    def _copy_out(self, y, yg):
        y[:] = yg


def _pool(n):
    from spc5_b200 import matrices as M
    return [M.banded(200 + 10 * i, 5, 0.5, seed=i) for i in range(n)]


def test_multiserver_routes_hot_matrix_over_its_replicas():
    ms = _FakeMulti(n_gpus=4, slots=2, max_k=4)
    csrs = _pool(8)
    shares = np.full(8, 0.02)
    shares[0] = 0.86
    ms.add_matrices(csrs, shares / shares.sum(), [2] * 8)
    reps = ms.placement[0]
    assert len(reps) > 1  # the hot matrix is replicated
    keys = [ms.submit(0, np.ones(csrs[0].ncols), np.zeros(csrs[0].nrows)) for _ in range(4 * len(reps))]
    per = ms.outstanding()
    assert sorted(set(ms.gpu_of(k) for k in keys)) == sorted(reps)
    assert all(per[g] == 4 for g in reps) and sum(per) == len(keys)
    for k in keys:
        ms.wait(k)
    assert ms.outstanding() == [0, 0, 0, 0]


def test_multiserver_failed_wait_keeps_the_request():
    ms = _FakeMulti(n_gpus=4)
    csrs = _pool(4)
    ms.add_matrices(csrs, np.full(4, 0.25), [2] * 4)
    y = np.zeros(csrs[1].nrows)
    key = ms.submit(1, np.ones(csrs[1].ncols), y)
    g = ms.gpu_of(key)
    ms.servers[g].fail_waits = 1
    with pytest.raises(TimeoutError):
        ms.wait(key)
    assert ms.outstanding()[g] == 1  # still outstanding, still counted
    ms.wait(key)  # retry succeeds
    assert np.all(y == (ms.ids[1][g] + 1) * csrs[1].ncols) and ms.outstanding()[g] == 0


def test_multiserver_second_add_keeps_outstanding_counts():
    ms = _FakeMulti(n_gpus=4)
    first = _pool(4)
    ms.add_matrices(first, np.full(4, 0.25), [2] * 4)
    keys = [ms.submit(i, np.ones(c.ncols), np.zeros(c.nrows)) for i, c in enumerate(first)]
    before = ms.outstanding()
    ms.add_matrices(_pool(2), np.full(2, 0.5), [2] * 2)
    assert ms.outstanding() == before
    for k in keys:
        ms.wait(k)
    assert ms.outstanding() == [0, 0, 0, 0]
