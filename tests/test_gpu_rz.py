"""Axisymmetric r-z geometry on the GPU (x axial, y radial, row 0 the axis).

* Multigrid: the exact discrete solution phi = r^2 + z^2 of L phi = 6 (the
  operator is exact on quadratics), in both precisions and every launch mode
  (the persistent and cluster modes fall back to the graph loop); a
  two-electrode problem against the oracle's direct sparse solve; the
  reported residual against the oracle's FP64 recomputation.
* The drop-in operators (pic_update_R_rz, pic_update_E_rz, pic_rz_density)
  against the oracle, bit for bit where the arithmetic is the same.
* The fused step in r-z: every particle pass bit-exact against the oracle's
  FP32 drift_rz given the same E; the density within the deposit tolerance
  of the Cartesian tests divided by the node volumes; the diagnostics
  against numpy.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from pic_b200 import Consts, _lib, workloads
from pic_b200.Boundaries import Boundaries
from pic_b200.Grid import Grid2D
from pic_b200.multigrid import MultigridSolver
from pic_b200.Particles import Particles2D
from pic_b200.simulation import PICSimulation
from pic_b200.Solvers import Solver

pytestmark = pytest.mark.gpu
DEV = "cuda"


def rz_mask(m, n):
    mk = np.zeros((n, m), np.uint8)
    mk[-1, :] = mk[:, 0] = mk[:, -1] = 1
    return mk.reshape(-1)


def quadratic(m, n, dx, dy):
    j, i = np.divmod(np.arange(m * n), m)
    return (i * dx) ** 2 + (j * dy) ** 2


@pytest.mark.parametrize("launch", ["graph", "host", "persistent", "cluster"])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("shape", [(17, 17), (65, 33), (129, 129), (257, 257), (513, 257)])
def test_exact_quadratic(launch, precision, shape):
    m, n = shape
    h = 1e-3
    mask = rz_mask(m, n)
    exact = quadratic(m, n, h, h)
    f = np.full(m * n, 6.0)
    f[mask == 1] = 0.0
    mg = MultigridSolver(mask, m, n, h, precision=precision, launch=launch, hy=h, geometry="rz")
    assert mg.effective_launch() in ("graph", "host")
    phi0 = np.where(mask == 1, exact, 0.0)
    phi = torch.as_tensor(phi0, device=DEV)
    # phi ~ 0.1 against 1/h^2 = 1e6: the FP64 residual of this problem bottoms out near 2e-12
    phi, (cycles, rel) = mg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-10, max_cycles=40)
    assert rel < 1e-10 and cycles <= 16, (cycles, rel)
    np.testing.assert_allclose(phi.cpu().numpy(), exact, rtol=0, atol=1e-8 * exact.max())


def electrode_problem(m, n, h, cols=None):
    """Two disk electrodes on the axis at -10 V and +10 V, a Gaussian charge cloud."""
    j, i = np.divmod(np.arange(m * n), m)
    mask = rz_mask(m, n)
    phi_bc = np.zeros(m * n)
    for col, v in zip(cols or (m // 4, 3 * m // 4), (-10.0, 10.0)):
        sel = (i == col) & (j <= n // 2)
        mask[sel] = 1
        phi_bc[sel] = v
    x, r = i * h, j * h
    rho = 1e-6 * np.exp(-(((x - 0.5 * (m - 1) * h) / (0.15 * m * h)) ** 2) - (r / (0.3 * n * h)) ** 2)
    f = -rho / Consts.eps0
    f[mask == 1] = 0.0
    return mask, phi_bc, f


@pytest.mark.parametrize("cols", [(32, 96), (43, 85)])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_electrodes_against_direct_solve(precision, cols):
    """Electrodes on lines that coarsen exactly (32, 96) and on odd lines (43,
    85), which the coarse grids keep as two-line bands (slower: about 35
    cycles to 1e-10 instead of under 20)."""
    m, n, h = 129, 65, 2e-4
    mask, phi_bc, f = electrode_problem(m, n, h, cols)
    direct = O.rz_solve(f, phi_bc, mask, m, n, h, h)
    mg = MultigridSolver(mask, m, n, h, precision=precision, hy=h, geometry="rz")
    phi = torch.as_tensor(phi_bc.copy(), device=DEV)
    phi, (cycles, rel) = mg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-10, max_cycles=60)
    got = phi.cpu().numpy()
    assert rel < 1e-10 and cycles <= (20 if cols[0] % 2 == 0 else 45), (cycles, rel)
    np.testing.assert_allclose(got, direct, rtol=0, atol=1e-8 * np.abs(direct).max())
    # the reported residual is the oracle's FP64 residual (to 2 %, above the FP64 floor)
    cpu = O.rz_residual(got, f, mask, m, n, h, h)
    assert abs(rel - cpu) <= 2e-2 * cpu + 1e-12, (rel, cpu)
    # the axis nodes between the electrodes are unknowns, not boundary values
    assert -10.0 < got[m // 2] < 10.0 and got[m // 2] != 0.0


def test_drop_in_operators_bit_exact():
    rng = np.random.default_rng(5)
    m, n, h, k = 65, 33, 1e-3, 50_000
    x = rng.uniform(5, m - 6, k).astype(np.float32)  # at least 5 cells from the walls: no absorption
    y = rng.uniform(0, n - 7, k).astype(np.float32)
    vx, vy, vz = (rng.normal(0, 1e4, k).astype(np.float32) for _ in range(3))
    dt = np.float32(5e-8 / h)
    d = [torch.as_tensor(a.copy(), device=DEV) for a in (x, y, vx, vy, vz)]
    _lib.call("pic_update_R_rz", *[_lib.ptr(t) for t in d], k, float(dt), float(dt), _lib.stream_ptr())
    ref = [a.copy() for a in (x, y, vx, vy, vz)]
    a, _ = O.drift_rz_absorb_f32(ref[0], ref[1], ref[2], ref[3], ref[4], dt, dt, m, n)
    assert a == 0
    for t, r in zip(d, ref):
        np.testing.assert_array_equal(t.cpu().numpy().view(np.uint32), r.view(np.uint32))
    # E with E_r = 0 on the axis
    phi = rng.normal(0, 1, m * n)
    ex = torch.zeros(m * n, dtype=torch.float32, device=DEV)
    ey = torch.zeros_like(ex)
    _lib.call("pic_update_E_rz", _lib.ptr(torch.as_tensor(phi, device=DEV)), _lib.ptr(ex), _lib.ptr(ey), m, n, h, h,
              _lib.stream_ptr())
    rx, ry = O.update_E_f32(phi, m, n, h, h)
    ry[:m] = 0.0
    np.testing.assert_array_equal(ex.cpu().numpy(), rx)
    np.testing.assert_array_equal(ey.cpu().numpy(), ry)
    # deposit -> density with the node volumes
    rho = rng.uniform(-1, 1, m * n).astype(np.float32)
    t = torch.as_tensor(rho.copy(), device=DEV)
    _lib.call("pic_rz_density", _lib.ptr(t), m, n, h, _lib.stream_ptr())
    want = (rho.astype(np.float64) / np.repeat(O.rz_row_volume(np.arange(n), n, h), m)).astype(np.float32)
    np.testing.assert_allclose(t.cpu().numpy(), want, rtol=2e-7)


def make_rz_sim(w, seed=0, push_kernel="ring", mcc=None, sort_interval=0, use_graph=False):
    m = w.nodes
    mask = rz_mask(m, m)
    phi_bc = np.zeros(m * m)
    j, i = np.divmod(np.arange(m * m), m)
    sel = (i == m // 3) & (j <= m // 4)  # a disk electrode on the axis
    mask[sel] = 1
    phi_bc[sel] = -w.left_V if w.left_V else -20.0
    sp_ = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=5e3, capacity=2 * w.n_e),
           dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=5e3, capacity=2 * w.n_i)]
    sim = PICSimulation(m, m, w.dx, w.dx, w.dt, sp_, mask, phi_bc, tol=w.tol, max_cycles=60,
                        sort_interval=sort_interval, seed=seed, geometry="rz", push_kernel=push_kernel, mcc=mcc,
                        use_graph=use_graph)
    rng = np.random.Generator(np.random.Philox(w.seed))
    arrays = [list(workloads.species_arrays(w, "e", rng)), list(workloads.species_arrays(w, "i", rng))]
    for s, a in enumerate(arrays):
        # radii uniform in volume (the Maxwellian vz is the azimuthal velocity)
        a[1] = np.sqrt(rng.uniform(0.0, (m - 2) ** 2, a[1].size)).astype(np.float32)
        sim.load(s, *a)
    return sim, [[c.copy() for c in a] for a in arrays], mask


def assert_bits(a, b):
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_array_equal(a[~np.isnan(a)].view(np.uint32), b[~np.isnan(b)].view(np.uint32))


@pytest.mark.parametrize("push_kernel", ["ring", "warp", "warp_agg", "pipe"])
def test_fused_rz_step_bit_exact(push_kernel):
    w = workloads.scaled(workloads.SMALL, n=30_000)
    sim, ref, mask = make_rz_sim(w, push_kernel=push_kernel)
    m = w.nodes
    kqs = [np.float32(-Consts.qe / Consts.me * w.dt), np.float32(Consts.qe / workloads.ION_MASS * w.dt)]
    dtdx = np.float32(w.dt / w.dx)
    vb, hb = O.electrode_bits(mask, m, m)
    sim.init()
    phi, rho, Ex, Ey = (f.cpu().numpy().copy() for f in sim.fields())
    ex, ey = O.update_E_f32(phi, m, m, w.dx, w.dx)
    ey[:m] = 0.0
    np.testing.assert_array_equal(Ex, ex)
    np.testing.assert_array_equal(Ey, ey)
    # density: the Cartesian deposit tolerance, times dx*dy / V_j
    exact = np.zeros(m * m)
    absum = np.zeros(m * m)
    fixed = np.zeros(m * m)
    for s, a in enumerate(ref):
        scale = np.float32(sim.species[s]["charge"] * sim.species[s]["np2c"] / (w.dx * w.dx))
        O.deposit_f32(a[0], a[1], scale, m, m, exact, absum)
        fixed += O.deposit_counts(a[0], a[1], m, m) * 2.0**-20 * abs(float(scale))
    g = 1.0 / np.repeat(O.rz_row_volume(np.arange(m), m, w.dx), m)
    assert np.all(np.abs(rho - exact * g) <= (2e-6 * absum + fixed) * g + 1e-7 * np.abs(exact * g) + 1e-30)
    # the solve: FP64 residual of the stored (float32) density
    f = -rho.astype(np.float64) / Consts.eps0
    f[mask == 1] = 0.0
    assert O.rz_residual(phi, f, mask, m, m, w.dx, w.dx) < 1e-6
    for s, a in enumerate(ref):
        O.kick_f32(a[0], a[1], a[2], a[3], ex, ey, np.float32(np.float64(kqs[s]) * -0.5), m, m)
        got = [t.cpu().numpy() for t in sim.species_arrays(s)]
        for k in range(5):
            assert_bits(got[k], a[k])
    sim.step(1)
    absorbed, collected = [0, 0], [0, 0]
    for s in range(2):
        a = ref[s]
        absorbed[s], collected[s] = O.drift_rz_absorb_f32(a[0], a[1], a[2], a[3], a[4], dtdx, dtdx, m, m, vb, hb)
        got = [t.cpu().numpy() for t in sim.species_arrays(s)]
        for k in range(5):
            assert_bits(got[k], a[k])
    c = sim.counters()
    assert c["absorbed"] == absorbed and c["electrode_absorbed"] == collected
    _, _, Ex1, Ey1 = (f.cpu().numpy().copy() for f in sim.fields())
    assert np.all(Ey1[:m] == 0.0)
    sim.step(1)
    for s in range(2):
        a = ref[s]
        O.kick_f32(a[0], a[1], a[2], a[3], Ex1, Ey1, kqs[s], m, m)
        O.drift_rz_absorb_f32(a[0], a[1], a[2], a[3], a[4], dtdx, dtdx, m, m, vb, hb)
        got = [t.cpu().numpy() for t in sim.species_arrays(s)]
        for k in range(5):
            assert_bits(got[k], a[k])
    live = [np.isfinite(t.cpu().numpy()) for t in (sim.species_arrays(0)[0], sim.species_arrays(1)[0])]
    ys = [sim.species_arrays(s)[1].cpu().numpy()[live[s]] for s in range(2)]
    assert min(y.min() for y in ys) >= 0.0
    sim.close()


@pytest.mark.parametrize("push_kernel", ["ring", "warp"])
def test_rz_step_with_mcc_bookkeeping(push_kernel):
    """r-z geometry with null-collision MCC in a dense gas (the disk electrode
    on the axis collecting too): the candidates keep their azimuthal velocity
    through the pass and take the r-z drift after their collision, the
    ionisation products too.  Every particle is accounted for, no live radius
    is negative, and the azimuthal velocities stay finite."""
    w = workloads.scaled(workloads.MCC, nodes=129, n=60_000, gas_density=3e22)
    sim, _, _ = make_rz_sim(w, seed=5, push_kernel=push_kernel, mcc=workloads.mcc_tables(w), sort_interval=4,
                            use_graph=True)
    sim.init()
    sim.step(10)
    sim.sync()
    c = sim.counters()
    assert sum(c["collisions"][0]) > 0 and c["born"][0] > 0 and c["dropped_births"] == 0
    for s, n0 in enumerate((w.n_e, w.n_i)):
        x, y, vx, vy, vz = (t.cpu().numpy() for t in sim.species_arrays(s))
        live = np.isfinite(x)
        assert int(live.sum()) == n0 - c["absorbed"][s] - c["electrode_absorbed"][s] + c["born"][s]
        assert y[live].min() >= 0.0
        assert np.all(np.isfinite(vz[live]))
    sim.close()


def test_rz_diagnostics_match_numpy():
    w = workloads.scaled(workloads.SMALL, n=20_000)
    sim, _, _ = make_rz_sim(w, seed=2)
    sim.init()
    sim.step(3)
    sim.sync()
    d = sim.diagnostics()
    m, dx = w.nodes, w.dx
    phi, rho, E0, E1 = (f.cpu().numpy().astype(np.float64) for f in sim.fields())
    v = np.repeat(O.rz_row_volume(np.arange(m), m, dx), m)  # V_j / (dx dy)
    assert d["field_energy"] == pytest.approx(0.5 * np.sum(rho * phi * v) * dx * dx, rel=1e-12)
    assert d["gauss_charge"] == pytest.approx(np.sum(rho * v) * dx * dx / Consts.eps0, rel=1e-12)
    Ex, Ey = E0.reshape(m, m), E1.reshape(m, m)
    vv = v.reshape(m, m)
    R = (m - 1) * dx
    flux = np.sum(Ex[:, -1] * dx * vv[:, -1]) - np.sum(Ex[:, 0] * dx * vv[:, 0]) + np.sum(Ey[-1, :]) * dx * 2 * np.pi * R
    assert d["gauss_flux"] == pytest.approx(flux, rel=1e-9, abs=1e-12 * abs(flux) + 1e-30)
    for s in range(2):
        vx, vy, vz = (t.cpu().numpy().astype(np.float64) for t in sim.species_arrays(s)[2:])
        live = np.isfinite(sim.species_arrays(s)[0].cpu().numpy())
        sp_ = sim.species[s]
        ke = 0.5 * sp_["mass"] * sp_["np2c"] * np.sum(vx[live] ** 2 + vy[live] ** 2 + vz[live] ** 2)
        assert d["kinetic"][s] == pytest.approx(ke, rel=1e-12)
    sim.close()


def test_drop_in_classes_cylindrical():
    m, n, X, Y = 65, 33, 0.032, 0.016
    grid = Grid2D(m, n, X, Y, cylindrical=True)
    parts = Particles2D(200_000, cylindrical=True)
    parts.add_species("electrons", Consts.me, -Consts.qe, 0)
    parts.grid = grid
    parts.np2c = 1e4
    parts.maxwellian_species_load(0.004, 0.0, 0.028, 0.012, 200_000, "electrons", 2.0, seed=3, grid=grid)
    bounds = [((m // 4, 0, m // 4, n // 3), -5.0), ((0, n - 1, m - 1, n - 1), 0.0)]
    bnd = Boundaries(bounds, grid)
    solver = Solver("multigrid", grid, cylindrical=True, boundaries=bnd, tol=1e-10)
    grid.update_density(parts)
    solver.solve(grid)
    grid.update_E()
    # the solve against the oracle's direct r-z solve of the same density
    mask = solver.dirichlet.cpu().numpy()
    f = -grid.rho.cpu().numpy().astype(np.float64) / Consts.eps0
    f[mask == 1] = 0.0
    direct = O.rz_solve(f, bnd.phi_bc_host, mask, m, n, grid.dx, grid.dy)
    phi = grid.phi.cpu().numpy()
    np.testing.assert_allclose(phi, direct, rtol=0, atol=1e-7 * np.abs(direct).max())
    assert np.all(grid.E[1][:m].cpu().numpy() == 0.0)
    # the density of a uniform-in-volume load is flat in r inside the load (statistically)
    rho = grid.rho.cpu().numpy().reshape(n, m)
    band = rho[1:8, 16:48]
    assert np.std(band.mean(axis=1)) < 0.1 * abs(band.mean())
    # the drift keeps r >= 0
    s = parts.species[0]
    parts.update_R(1e-9)
    assert float(s.y[: s.n][torch.isfinite(s.x[: s.n])].min()) >= 0.0
