"""pic_sort_static (the cell sort with its scratch in a fixed device array)
against pic_sort (scratch from pic_sorter_create) through the C ABI: two
calls in a row, the second smaller and on another grid, so that whatever the
first call left in the shared scratch must not leak into the second.  The
sort is index work, so the comparison is exact."""
import numpy as np
import pytest
import torch

from pic_b200 import _lib

pytestmark = pytest.mark.gpu
DEV = "cuda"
STATIC_MAX = 1 << 20  # PIC_SORT_STATIC_MAX


def particles(n, m, nn, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    x = rng.uniform(0, m - 1, n).astype(np.float32)
    y = rng.uniform(0, nn - 1, n).astype(np.float32)
    dead = rng.random(n) < 0.03
    x[dead] = np.nan
    y[dead] = np.nan
    v = [rng.normal(0, 1e5, n).astype(np.float32) for _ in range(3)]
    return [torch.as_tensor(a, device=DEV) for a in (x, y, *v)]


def outputs(n, ntiles):
    outs = [torch.full((max(n, 1),), -1.0, dtype=torch.float32, device=DEV) for _ in range(5)]
    perm = torch.full((max(n, 1),), -1, dtype=torch.int32, device=DEV)
    cnt = torch.full((1,), -1, dtype=torch.int32, device=DEV)
    ts = torch.full((ntiles + 1,), -1, dtype=torch.int32, device=DEV)
    return outs, perm, cnt, ts


def ntiles_of(m, nn, tile):
    return ((m - 1 + tile - 1) // tile) * ((nn - 1 + tile - 1) // tile)


def sort_with_sorter(ins, n, m, nn, tile):
    s = _lib.C.c_void_p()
    _lib.call("pic_sorter_create", max(n, 1), m, nn, tile, _lib.C.byref(s))
    try:
        outs, perm, cnt, ts = outputs(n, ntiles_of(m, nn, tile))
        _lib.call("pic_sort", s, *[_lib.ptr(a) for a in ins], n, *[_lib.ptr(a) for a in outs], _lib.ptr(perm),
                  _lib.ptr(cnt), _lib.ptr(ts), _lib.stream_ptr())
        torch.cuda.synchronize()
    finally:
        _lib.load().pic_sorter_destroy(s)
    return outs, perm, cnt, ts


def sort_static(ins, n, m, nn, tile):
    outs, perm, cnt, ts = outputs(n, ntiles_of(m, nn, tile))
    _lib.call("pic_sort_static", *[_lib.ptr(a) for a in ins], n, m, nn, tile, *[_lib.ptr(a) for a in outs],
              _lib.ptr(perm), _lib.ptr(cnt), _lib.ptr(ts), _lib.stream_ptr())
    torch.cuda.synchronize()
    return outs, perm, cnt, ts


def assert_same(a, b):
    k = int(a[2].item())
    assert k == int(b[2].item())
    assert torch.equal(a[1][:k], b[1][:k])
    for u, v in zip(a[0], b[0]):
        assert torch.equal(u[:k], v[:k])
    assert torch.equal(a[3], b[3])
    return k


def test_static_sort_matches_sorter_on_two_calls_in_a_row():
    cases = [(513, 513, 16, 900_000, 11), (129, 65, 8, 250_000, 12)]
    for m, nn, tile, n, seed in cases:
        ins = particles(n, m, nn, seed)
        ref = sort_with_sorter(ins, n, m, nn, tile)
        got = sort_static(ins, n, m, nn, tile)
        k = assert_same(got, ref)
        assert 0 < k < n


def test_static_sort_limits():
    # the largest size it takes, then one past it (rejected before any work)
    n = STATIC_MAX
    ins = particles(n, 257, 257, 13)
    k = assert_same(sort_static(ins, n, 257, 257, 16), sort_with_sorter(ins, n, 257, 257, 16))
    assert k > 0
    with pytest.raises(_lib.PicError) as e:
        _lib.call("pic_sort_static", *[_lib.ptr(a) for a in ins], STATIC_MAX + 1, 257, 257, 16,
                  *[_lib.ptr(None)] * 5, _lib.ptr(None), _lib.ptr(None), _lib.ptr(None), _lib.stream_ptr())
    assert e.value.code == _lib.PIC_ERR_BAD_ARG and "fixed scratch" in str(e.value)
    # empty input: count 0, every tile start 0
    outs, perm, cnt, ts = sort_static(ins, 0, 257, 257, 16)
    assert int(cnt.item()) == 0 and bool((ts == 0).all())
