"""Cell sort on the GPU: permutation bit-identical to a stable argsort of the
oracle's tile-major keys, dead particles dropped, tile starts exact."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from pic_b200 import _lib

pytestmark = pytest.mark.gpu
DEV = "cuda"


def run_sort(x, y, vx, vy, vz, m, nn, tile, capacity=None):
    n = len(x)
    cap = capacity or max(n, 1)
    s = _lib.C.c_void_p()
    _lib.call("pic_sorter_create", cap, m, nn, tile, _lib.C.byref(s))
    try:
        ins = [torch.zeros(cap, dtype=torch.float32, device=DEV) for _ in range(5)]
        for a, v in zip(ins, (x, y, vx, vy, vz)):
            a[:n] = torch.as_tensor(v, device=DEV)
        outs = [torch.full((cap,), -1.0, dtype=torch.float32, device=DEV) for _ in range(5)]
        perm = torch.zeros(cap, dtype=torch.int32, device=DEV)
        cnt = torch.zeros(1, dtype=torch.int32, device=DEV)
        ntiles = ((m - 1 + tile - 1) // tile) * ((nn - 1 + tile - 1) // tile)
        ts = torch.zeros(ntiles + 1, dtype=torch.int32, device=DEV)
        _lib.call("pic_sort", s, *[_lib.ptr(a) for a in ins], n, *[_lib.ptr(a) for a in outs], _lib.ptr(perm),
                  _lib.ptr(cnt), _lib.ptr(ts), _lib.stream_ptr())
        torch.cuda.synchronize()
        k = int(cnt.item())
        return k, perm[:k].cpu().numpy().astype(np.uint32), [a[:k].cpu().numpy() for a in outs], ts.cpu().numpy()
    finally:
        _lib.load().pic_sorter_destroy(s)


# key widths: 9 bits (one radix pass), 15 (two), 19 (two of 10 and 9 bits),
# 21 (three of 7), and a tile side that is not a power of two
@pytest.mark.parametrize("m,nn,n,tile", [(17, 17, 1000, 4), (129, 129, 300_000, 16), (513, 513, 3_000_000, 16),
                                         (65, 33, 50_000, 8), (1025, 1025, 2_000_000, 16), (200, 150, 100_000, 5)])
def test_sort_is_stable_argsort(m, nn, n, tile):
    rng = np.random.Generator(np.random.Philox(7))
    x = rng.uniform(0, m - 1, n).astype(np.float32)
    y = rng.uniform(0, nn - 1, n).astype(np.float32)
    x[:3] = [0.0, m - 1, m - 1]
    y[:3] = [nn - 1, 0.0, nn - 1]
    dead = rng.random(n) < 0.02
    x[dead] = np.nan
    y[dead] = np.nan
    vx, vy, vz = (rng.normal(0, 1, n).astype(np.float32) for _ in range(3))
    k, perm, outs, ts = run_sort(x, y, vx, vy, vz, m, nn, tile)
    keys = O.sort_keys(x, y, m, nn, tile)
    ref = np.argsort(keys, kind="stable")[: int((~dead).sum())].astype(np.uint32)
    assert k == int((~dead).sum())
    np.testing.assert_array_equal(perm, ref)
    np.testing.assert_array_equal(outs[0], x[ref])
    np.testing.assert_array_equal(outs[4], vz[ref])
    skeys = keys[ref]
    ntiles = len(ts) - 1
    np.testing.assert_array_equal(ts[:-1], np.searchsorted(skeys, np.arange(ntiles) * tile * tile, side="left"))
    assert ts[-1] == k


def test_sort_is_deterministic_and_handles_empty():
    rng = np.random.Generator(np.random.Philox(8))
    n, m = 200_000, 129
    x = rng.uniform(0, 8, n).astype(np.float32)  # heavy contention: few cells
    y = rng.uniform(0, 8, n).astype(np.float32)
    z = np.zeros(n, np.float32)
    a = run_sort(x, y, z, z, z, m, m, 16)
    b = run_sort(x, y, z, z, z, m, m, 16)
    np.testing.assert_array_equal(a[1], b[1])
    k, perm, _, ts = run_sort(np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32),
                              np.zeros(0, np.float32), np.zeros(0, np.float32), m, m, 16, capacity=16)
    assert k == 0 and np.all(ts == 0)


def test_permutation_only_writes_the_live_entries():
    """pic_sort with d_x_out NULL: the permutation alone, into a buffer sized
    for n (not for the sorter's larger capacity); nothing past the live count
    is written (a guard region after n keeps its fill)."""
    rng = np.random.Generator(np.random.Philox(12))
    m, tile, n, cap, guard = 129, 16, 50_000, 400_000, 4096
    x = rng.uniform(0, m - 1, n).astype(np.float32)
    y = rng.uniform(0, m - 1, n).astype(np.float32)
    dead = rng.random(n) < 0.05
    x[dead] = np.nan
    s = _lib.C.c_void_p()
    _lib.call("pic_sorter_create", cap, m, m, tile, _lib.C.byref(s))
    try:
        X, Y = torch.as_tensor(x, device=DEV), torch.as_tensor(y, device=DEV)
        perm = torch.full((n + guard,), -7, dtype=torch.int32, device=DEV)
        cnt = torch.zeros(1, dtype=torch.int32, device=DEV)
        _lib.call("pic_sort", s, _lib.ptr(X), _lib.ptr(Y), None, None, None, n, None, None, None, None, None,
                  _lib.ptr(perm), _lib.ptr(cnt), None, _lib.stream_ptr())
        torch.cuda.synchronize()
        k = int(cnt.item())
        got = perm.cpu().numpy()
    finally:
        _lib.load().pic_sorter_destroy(s)
    keys = O.sort_keys(x, y, m, m, tile)
    ref = np.argsort(keys, kind="stable")[: int((~dead).sum())]
    assert k == ref.size
    np.testing.assert_array_equal(got[:k], ref.astype(np.int32))
    assert np.all(got[k:] == -7)
