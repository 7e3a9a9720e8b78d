"""The r-z (axisymmetric) pieces of the oracle, on the CPU.

* The reference's cylindrical Laplacian builder (src/Solvers.py:100-166),
  restated, against its golden matrix lap.txt (tests/golden/
  lap_cylindrical_10x10.npz): every row off the axis agrees to the file's two
  decimals.  The file's axis rows (-2 on the diagonal, +2 towards row 1, no
  z neighbours) come from an earlier form of the builder than the source now
  holds (-4, z neighbours, +2), so the axis rows are checked against each
  form separately.
* The build's r-z operator: exact on quadratics, symmetric once weighted by
  the row volumes, and its direct solve reproduces an exact solution.  Where
  it differs from the reference's matrix is written out below.
* The r-z drift: a straight line in 3D (radius and angular momentum), the
  axis crossing, and the planar drift it reduces to without azimuthal motion.
* The node volumes: a load uniform in volume deposits a uniform density.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "lap_cylindrical_10x10.npz")


def golden_lap():
    z = np.load(GOLDEN)
    L = np.zeros(tuple(z["shape"]))
    L[z["rows"], z["cols"]] = z["vals"]
    return L


def test_reference_laplacian_against_golden_matrix():
    L = golden_lap()
    A = O.ref_cylindrical_laplacian(10, 10, 1, 1)
    np.testing.assert_array_equal(np.round(A[10:], 2), L[10:])
    # the axis rows: the file's form and the source's form
    for k in range(10):
        assert L[k, k] == -2.0 and L[k, k + 10] == 2.0 and np.count_nonzero(L[k]) == 2
        nz = {int(c): A[k, c] for c in np.flatnonzero(A[k])}
        assert nz[k] == -4.0 and nz[k + 10] == 2.0
        assert all(nz[c] == 1.0 for c in (k - 1, k + 1) if c in nz)


def test_build_operator_against_reference_matrix():
    """Where the build's operator (rows times dr^2, dr = dz = 1) departs from
    the reference's matrix: the upper r weight of row j is 1 + 1/2j (the
    reference takes 1 + 1/2(j+1)), the last interior row keeps its upper
    neighbour, and the axis row is 4 (phi_1 - phi_0) + the z terms (the
    reference: 2 (phi_1 - phi_0)).  The lower r weights agree."""
    m = n = 10
    A = O.ref_cylindrical_laplacian(m, n, 1, 1)
    wn, ws, dg = O.rz_rows(n, 1.0, 1.0)
    for j in range(1, n - 1):
        k = j * m + 4
        assert A[k, k - m] == ws[j]
        assert wn[j] == 1 + 0.5 / j
        assert A[k, k + m] == (1 + 0.5 / (j + 1) if j < n - 2 else 0.0)
        assert dg[j] == pytest.approx(-4.0, rel=1e-15)
    assert (wn[0], ws[0], dg[0]) == (4.0, 0.0, -6.0) and A[4, 4 + m] == 2.0


def test_operator_is_exact_on_quadratics():
    # phi = r^2 + z^2: (1/r) d/dr (r 2r) + 2 = 6, on every row including the axis
    m, n, dx, dy = 17, 9, 0.003, 0.002
    j, i = np.divmod(np.arange(m * n), m)
    phi = (i * dx) ** 2 + (j * dy) ** 2
    L = O.rz_apply(phi, m, n, dx, dy).reshape(n, m)
    np.testing.assert_allclose(L[:-1, 1:-1], 6.0, rtol=1e-9)


def test_operator_is_symmetric_with_row_volumes():
    m, n, dx, dy = 7, 9, 1.0, 1.0
    size = m * n
    A = np.zeros((size, size))
    for k in range(size):
        e = np.zeros(size)
        e[k] = 1.0
        A[:, k] = O.rz_apply(e, m, n, dx, dy)
    j = np.arange(size) // m
    D = np.where(j == 0, 0.125, j.astype(float))
    inner = np.flatnonzero((np.arange(size) % m > 0) & (np.arange(size) % m < m - 1) & (j < n - 1))
    S = (D[:, None] * A)[np.ix_(inner, inner)]
    np.testing.assert_allclose(S, S.T, atol=1e-12)


def test_direct_solve_reproduces_the_quadratic():
    m, n, dx, dy = 33, 17, 0.01, 0.01
    j, i = np.divmod(np.arange(m * n), m)
    exact = (i * dx) ** 2 + (j * dy) ** 2
    mask = np.zeros(m * n, np.uint8)
    mask[(j == 5) & (i > 10) & (i < 20)] = 1  # an internal electrode at its exact potential
    phi = O.rz_solve(np.full(m * n, 6.0), exact, mask, m, n, dx, dy)
    np.testing.assert_allclose(phi, exact, rtol=1e-10, atol=1e-14)
    assert O.rz_residual(phi, np.full(m * n, 6.0), mask, m, n, dx, dy) < 1e-12


def test_drift_is_a_straight_line_in_3d():
    rng = np.random.default_rng(1)
    k = 2000
    y = rng.uniform(0.0, 50.0, k).astype(np.float32)
    x = rng.uniform(10.0, 50.0, k).astype(np.float32)
    vx, vy, vz = (rng.normal(0, 1e5, k).astype(np.float32) for _ in range(3))
    dt = np.float32(2e-6)  # dt/dy: displacements of a fraction of a cell
    gx, gy, wy, wz = x.copy(), y.copy(), vy.copy(), vz.copy()
    a, c = O.drift_rz_absorb_f32(gx, gy, vx, wy, wz, dt, dt, 64, 64)
    assert a == 0 and c == 0
    # FP64 straight line from (y, 0) with velocity (vy, vz) in the plane normal to the axis
    Y = y.astype(np.float64) + vy.astype(np.float64) * np.float64(dt)
    T = vz.astype(np.float64) * np.float64(dt)
    R = np.hypot(Y, T)
    np.testing.assert_allclose(gy, R, rtol=3e-6, atol=3e-6)
    np.testing.assert_allclose(gx, x.astype(np.float64) + vx.astype(np.float64) * np.float64(dt), rtol=1e-6)
    # speed and angular momentum about the axis are kept
    np.testing.assert_allclose(np.hypot(wy, wz), np.hypot(vy, vz), rtol=2e-6)
    np.testing.assert_allclose(gy.astype(np.float64) * wz, y.astype(np.float64) * vz, rtol=1e-5, atol=1e-3)


def test_drift_through_the_axis_and_without_azimuthal_motion():
    # inward through the axis: comes out at r = |y + vy dt| moving outwards
    gx = np.array([5.0], np.float32)
    gy = np.array([0.25], np.float32)
    vy = np.array([-1.0], np.float32)
    vz = np.array([0.0], np.float32)
    O.drift_rz_absorb_f32(gx, gy, np.zeros(1, np.float32), vy, vz, np.float32(0.5), np.float32(0.5), 16, 16)
    assert gy[0] == np.float32(0.25) and vy[0] == np.float32(1.0) and vz[0] == 0.0
    # no azimuthal velocity and no axis crossing: bit-identical to the planar drift
    rng = np.random.default_rng(2)
    k = 1000
    x = rng.uniform(1, 30, k).astype(np.float32)
    y = rng.uniform(1, 30, k).astype(np.float32)
    vx, vy = (rng.normal(0, 1, k).astype(np.float32) for _ in range(2))
    a1, a2 = (x.copy(), y.copy()), (x.copy(), y.copy())
    O.drift_rz_absorb_f32(a1[0], a1[1], vx, vy.copy(), np.zeros(k, np.float32), np.float32(0.3), np.float32(0.3),
                          32, 32)
    O.drift_absorb_f32(a2[0], a2[1], vx, vy, np.float32(0.3), np.float32(0.3), 32, 32)
    np.testing.assert_array_equal(a1[0].view(np.uint32), a2[0].view(np.uint32))
    np.testing.assert_array_equal(a1[1].view(np.uint32), a2[1].view(np.uint32))


def test_node_volumes_make_a_uniform_load_uniform():
    n, dy = 17, 1.0
    rng = np.random.default_rng(3)
    N = 2_000_000
    r = np.sqrt(rng.uniform(0.0, (n - 1) ** 2, N))  # uniform in volume, grid units
    j0 = np.minimum(np.floor(r).astype(int), n - 2)
    w1 = r - j0
    q = np.bincount(j0, 1.0 - w1, n) + np.bincount(j0 + 1, w1, n)
    dens = q / O.rz_row_volume(np.arange(n), n, dy)
    expect = N / (np.pi * (n - 1) ** 2)  # particles per unit volume (per unit length of the axis)
    np.testing.assert_allclose(dens, expect, rtol=0.02)
