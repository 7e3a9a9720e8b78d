"""The Cartesian drop-in classes driven in the reference's step order.

SimulationManager._init_step / _step (src/simulation.py:622-660) call
  update_density -> solve -> update_E -> update_V(-dt/2)            (init)
  update_R -> update_axis -> update_density -> solve -> update_E
  -> update_V(dt) -> null_collision_method                          (step)
on Particles2D, Grid2D, Solver and MCC.  This test makes those calls on
pic_b200's classes, exactly as a caller that switched its imports would, and
checks every stage against the oracle: the deposit within the FP32-atomics
tolerance of the exact sum, phi through its FP64 residual and its Dirichlet
values, E, the kick, the drift and the wall absorption bit for bit, and the
null-collision step against the oracle's replay of the same Philox counters
(candidate and per-process counts exact, velocities of the particles that did
not collide bit for bit).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from pic_b200 import MCC, Consts, workloads
from pic_b200.Boundaries import Boundaries, walls_box
from pic_b200.Grid import Grid2D
from pic_b200.Particles import Particles2D
from pic_b200.Solvers import Solver

pytestmark = pytest.mark.gpu


def species_host(parts, k):
    s = parts.species[k]
    return [a[: s.n].cpu().numpy().copy() for a in s.arrays()]


def assert_bits(got, want, what):
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want), err_msg=what)
    live = ~np.isnan(want)
    np.testing.assert_array_equal(got[live].view(np.uint32), want[live].view(np.uint32), err_msg=what)


def check_density(grid, parts, what):
    m = grid.m
    exact, absum = np.zeros(m * m), np.zeros(m * m)
    for k, s in enumerate(parts.species):
        a = species_host(parts, k)
        live = ~np.isnan(a[0])
        scale = np.float32(s.charge * parts.species_np2c(s) / (grid.dx * grid.dy))
        O.deposit_f32(a[0][live], a[1][live], scale, m, m, exact, absum)
    rho = grid.rho.cpu().numpy()
    assert np.all(np.abs(rho - exact) <= 2e-6 * absum + 1e-30), what


def check_solve(grid, solver, bnd, tol, what):
    m = grid.m
    mask = solver.dirichlet.cpu().numpy()
    phi = grid.phi.cpu().numpy()
    f = -grid.rho.cpu().numpy().astype(np.float64) / Consts.eps0
    f[mask == 1] = 0
    rel = np.sqrt(O.residual_f64(phi, f, mask, m, m, grid.dx, grid.dy) / np.sum(f * f))
    assert rel < tol, f"{what}: residual {rel}"
    on = bnd.bc_lookup_host == 1
    np.testing.assert_array_equal(phi[on], bnd.phi_bc_host[on])
    return phi


def check_E(grid, phi, what):
    ex, ey = O.update_E_f32(phi, grid.m, grid.n, grid.dx, grid.dy)
    np.testing.assert_array_equal(grid.E[0].cpu().numpy(), ex, err_msg=what)
    np.testing.assert_array_equal(grid.E[1].cpu().numpy(), ey, err_msg=what)
    return ex, ey


def test_cartesian_dropin_classes_in_step_order():
    m, n_per = 129, 60_000
    dx = 1e-4
    L = dx * (m - 1)
    dt = 1e-11
    tol = 1e-8
    # 10 eV electrons: a tail above the 15.8 eV ionisation threshold, so that
    # the products are exercised too
    w = workloads.scaled(workloads.SMALL, n=n_per, left_V=20.0, Te=10.0)
    grid = Grid2D(m, m, L, L)
    parts = Particles2D(2 * n_per)
    parts.add_species("electrons", Consts.me, -Consts.qe, 0)  # collision model 0: takes part in MCC
    parts.add_species("ions", workloads.ION_MASS, Consts.qe, 1)
    parts.grid = grid
    parts.np2c = w.np2c(n_per)
    rng = np.random.Generator(np.random.Philox(5))
    for k, which in enumerate(("e", "i")):
        x, y, vx, vy, vz = workloads.species_arrays(w, which, rng)
        parts.load_species_arrays(k + 1, x.astype(np.float64) * dx, y.astype(np.float64) * dx, vx, vy, vz)
    bnd = Boundaries(walls_box(grid, left=20.0), grid)
    solver = Solver("multigrid", grid, boundaries=bnd, tol=tol)
    E_grid, sig_el, _, sig_ion, _ = workloads.cross_sections()
    xs = ((E_grid, sig_el), (E_grid, sig_ion))
    density, seed = 3e22, 99
    kq = [np.float32(s.charge / s.mass * dt) for s in parts.species]
    dtdx = np.float32(dt / dx)

    # _init_step (src/simulation.py:622-637)
    grid.update_density(parts)
    check_density(grid, parts, "init deposit")
    solver.solve(grid)
    phi = check_solve(grid, solver, bnd, tol, "init solve")
    grid.update_E()
    ex, ey = check_E(grid, phi, "init E")
    ref = [species_host(parts, k) for k in range(2)]
    parts.update_V(grid, -dt / 2)
    for k in range(2):
        O.kick_f32(ref[k][0], ref[k][1], ref[k][2], ref[k][3], ex, ey, np.float32(np.float64(kq[k]) * -0.5), m, m)
        got = species_host(parts, k)
        for c in range(4):
            assert_bits(got[c], ref[k][c], f"init kick species {k} array {c}")

    absorbed = candidates = 0
    collisions = np.zeros(4, np.int64)
    MCC._operators.clear()
    for step in range(2):
        # _step (src/simulation.py:640-660)
        ref = [species_host(parts, k) for k in range(2)]
        parts.update_R(dt)
        parts.update_axis(dt)
        for k in range(2):
            absorbed += O.drift_absorb_f32(ref[k][0], ref[k][1], ref[k][2], ref[k][3], dtdx, dtdx, m, m)
            got = species_host(parts, k)
            for c in range(4):
                assert_bits(got[c], ref[k][c], f"step {step} drift species {k} array {c}")
        assert int(parts.absorbed.item()) == absorbed
        grid.update_density(parts)
        check_density(grid, parts, f"step {step} deposit")
        solver.solve(grid)
        phi = check_solve(grid, solver, bnd, tol, f"step {step} solve")
        grid.update_E()
        ex, ey = check_E(grid, phi, f"step {step} E")
        parts.update_V(grid, dt)
        for k in range(2):
            O.kick_f32(ref[k][0], ref[k][1], ref[k][2], ref[k][3], ex, ey, kq[k], m, m)
            got = species_host(parts, k)
            for c in range(4):
                assert_bits(got[c], ref[k][c], f"step {step} kick species {k} array {c}")
        # null_collision_method: elastic and ionisation on the electrons
        n_e = parts.species[0].n
        n_i = parts.species[1].n
        MCC.null_collision_method(parts, density, xs, dt, 2 * n_per, IONIZATION=True, seed=seed)
        op = next(iter(MCC._operators.values()))
        nu, _, inv = op.query(0)
        procs = op.tables.species[0]
        S, keep = O.mcc_species(op.tables.energy, [p[2] for p in procs], [p[0] for p in procs],
                                [p[1] for p in procs], op.tables.gas_density, Consts.me, op.tables.gas_mass,
                                op.tables.gas_temperature, nu, inv, 0)
        mark = O.mcc_candidates(S, n_e, step, seed)
        mark[np.isnan(ref[0][0])] = 0
        e = ref[0]
        collided = np.zeros(n_e, bool)
        births = 0
        for i in np.flatnonzero(mark):
            v = [e[2][i], e[3][i], e[4][i]]
            proc, _, _ = O.mcc_collide(S, int(i), step, seed, v)
            if proc >= 0:
                collisions[proc] += 1
                collided[i] = True
                births += procs[proc][0] == MCC.IONIZATION
        candidates += int(mark.sum())
        ctr = op.counters.cpu().numpy()  # cumulative over the calls
        assert int(ctr[16]) == candidates
        np.testing.assert_array_equal(ctr[0:2], collisions[0:2])
        got = species_host(parts, 0)
        for c in range(5):
            assert_bits(got[c][:n_e][~collided], e[c][~collided], f"step {step} MCC species 0 array {c}")
        # the products join the electrons and the ions
        assert parts.species[0].n == n_e + births
        assert parts.species[1].n == n_i + births
        del keep
    assert collisions[0] > 100 and collisions[1] > 0
    MCC._operators.clear()
