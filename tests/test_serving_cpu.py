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
