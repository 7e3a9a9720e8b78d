"""Particle and grid operators on the GPU against the CPU oracle.

Bit-exact: drift, absorption (positions, NaN set, absorbed count), gather +
kick, E = -grad(phi).  Deposit: FP32 atomics in any order; compared with the
exact sum of the same FP32 contributions, |drho| <= 2e-6 * sum|contrib| + 1e-30
per node (a handful of FP32 roundings of partial sums).
Against the FP64 reference arithmetic the stated FP32 error is
|drho| <= 3e-5 * sum|contrib| (FP32 weights from FP32 grid-unit positions).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from pic_b200 import _lib

pytestmark = pytest.mark.gpu
DEV = "cuda"


def rand_particles(rng, n, m, nn, dead_frac=0.01, edge=True):
    x = rng.uniform(0, m - 1, n).astype(np.float32)
    y = rng.uniform(0, nn - 1, n).astype(np.float32)
    if edge:
        x[:4] = [0.0, m - 1, 3.0, np.nextafter(np.float32(m - 1), np.float32(0))]
        y[:4] = [0.0, nn - 1, np.nextafter(np.float32(2.0), np.float32(3)), 5.0]
    dead = rng.random(n) < dead_frac
    dead[:4] = False
    x[dead] = np.nan
    y[dead] = np.nan
    return x, y


def t(a):
    return torch.as_tensor(np.ascontiguousarray(a), device=DEV)


def s():
    return _lib.stream_ptr()


@pytest.mark.parametrize("m,nn,n", [(17, 13, 5000), (129, 129, 200_000)])
def test_drift_and_absorb_bit_exact(m, nn, n):
    rng = np.random.Generator(np.random.Philox(1))
    x, y = rand_particles(rng, n, m, nn)
    vx = rng.normal(0, 3e5, n).astype(np.float32)
    vy = rng.normal(0, 3e5, n).astype(np.float32)
    dtdx, dtdy = np.float32(1e-11 / 1e-4), np.float32(1e-11 / 1.25e-4)
    X, Y, VX, VY = t(x), t(y), t(vx), t(vy)
    absorbed = torch.zeros(1, dtype=torch.int64, device=DEV)
    _lib.call("pic_update_R", _lib.ptr(X), _lib.ptr(Y), _lib.ptr(VX), _lib.ptr(VY), n, float(dtdx), float(dtdy), None,
              None, s())
    _lib.call("pic_absorb", _lib.ptr(X), _lib.ptr(Y), n, m, nn, _lib.ptr(absorbed), s())
    ox, oy = x.copy(), y.copy()
    k = O.drift_absorb_f32(ox, oy, vx, vy, dtdx, dtdy, m, nn)
    gx, gy = X.cpu().numpy(), Y.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(gx), np.isnan(ox))
    np.testing.assert_array_equal(gx.view(np.uint32)[~np.isnan(ox)], ox.view(np.uint32)[~np.isnan(ox)])
    np.testing.assert_array_equal(gy.view(np.uint32)[~np.isnan(oy)], oy.view(np.uint32)[~np.isnan(oy)])
    assert int(absorbed.item()) == k


def test_update_E_bit_exact():
    rng = np.random.Generator(np.random.Philox(2))
    m, nn, dx, dy = 65, 33, 1e-4, 2e-4
    phi = rng.normal(0, 30, m * nn)
    Ex = torch.zeros(m * nn, dtype=torch.float32, device=DEV)
    Ey = torch.zeros_like(Ex)
    PHI = t(phi)
    _lib.call("pic_update_E", _lib.ptr(PHI), _lib.ptr(Ex), _lib.ptr(Ey), m, nn, dx, dy, s())
    ox, oy = O.update_E_f32(phi, m, nn, dx, dy)
    np.testing.assert_array_equal(Ex.cpu().numpy(), ox)
    np.testing.assert_array_equal(Ey.cpu().numpy(), oy)
    fx, fy = O.update_E_f64(phi, m, nn, dx, dy)
    np.testing.assert_allclose(Ex.cpu().numpy(), fx, rtol=6e-8, atol=1e-30)


@pytest.mark.parametrize("m,nn,n", [(17, 13, 3000), (129, 129, 300_000)])
def test_gather_kick_bit_exact(m, nn, n):
    rng = np.random.Generator(np.random.Philox(3))
    x, y = rand_particles(rng, n, m, nn)
    ex = rng.normal(0, 1e4, m * nn).astype(np.float32)
    ey = rng.normal(0, 1e4, m * nn).astype(np.float32)
    vx = rng.normal(0, 1e5, n).astype(np.float32)
    vy = rng.normal(0, 1e5, n).astype(np.float32)
    kq = np.float32(-1.6e-19 / 9.10938356e-31 * 1e-11)
    X, Y, VX, VY, EX, EY = t(x), t(y), t(vx), t(vy), t(ex), t(ey)  # keep every buffer alive during the call
    _lib.call("pic_update_V", _lib.ptr(X), _lib.ptr(Y), _lib.ptr(VX), _lib.ptr(VY), n, _lib.ptr(EX), _lib.ptr(EY), m,
              nn, float(kq), s())
    ovx, ovy = vx.copy(), vy.copy()
    O.kick_f32(x, y, ovx, ovy, ex, ey, kq, m, nn)
    np.testing.assert_array_equal(VX.cpu().numpy().view(np.uint32), ovx.view(np.uint32))
    np.testing.assert_array_equal(VY.cpu().numpy().view(np.uint32), ovy.view(np.uint32))


@pytest.mark.parametrize("m,nn,n", [(17, 13, 20_000), (513, 513, 2_000_000)])
def test_deposit_against_oracle(m, nn, n):
    rng = np.random.Generator(np.random.Philox(4))
    x, y = rand_particles(rng, n, m, nn)
    scale = np.float32(-1.6e-19 * 6.55e4 / 1e-8)
    rho = torch.zeros(m * nn, dtype=torch.float32, device=DEV)
    X, Y = t(x), t(y)
    _lib.call("pic_deposit", _lib.ptr(X), _lib.ptr(Y), n, float(scale), _lib.ptr(rho), m, nn, s())
    exact, abs_sum = O.deposit_f32(x, y, scale, m, nn)
    got = rho.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(got - exact) <= 2e-6 * abs_sum + 1e-30)
    # total charge is conserved to FP32 summation accuracy
    live = ~np.isnan(x)
    assert abs(got.sum() - float(scale) * live.sum()) <= 1e-5 * abs(float(scale)) * live.sum()


def test_deposit_fp32_error_against_fp64_reference_arithmetic():
    rng = np.random.Generator(np.random.Philox(5))
    m, nn, n, dx, dy = 129, 129, 100_000, 1e-4, 1e-4
    x, y = rand_particles(rng, n, m, nn, dead_frac=0.0)
    q, np2c = -1.6e-19, 1.638e5
    scale = np.float32(q * np2c / (dx * dy))
    rho = torch.zeros(m * nn, dtype=torch.float32, device=DEV)
    X, Y = t(x), t(y)
    _lib.call("pic_deposit", _lib.ptr(X), _lib.ptr(Y), n, float(scale), _lib.ptr(rho), m, nn, s())
    ref = O.deposit_f64(x.astype(np.float64) * dx, y.astype(np.float64) * dy, q * np2c, dx, dy, m, nn,
                        floorf_quirk=False) / (dx * dy)
    _, abs_sum = O.deposit_f32(x, y, scale, m, nn)
    err = np.abs(rho.cpu().numpy() - ref)
    assert np.all(err <= 3e-5 * abs_sum + 1e-30)


def test_bad_arguments_raise():
    with pytest.raises(_lib.PicError) as e:
        _lib.call("pic_deposit", None, None, 10, 1.0, None, 17, 17, s())
    assert e.value.code == _lib.PIC_ERR_BAD_ARG
    assert "pic_deposit" in str(e.value)
