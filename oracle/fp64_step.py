"""The reference's time step in FP64 on the CPU (test infrastructure only).

SimulationManager._init_step / _step (src/simulation.py:622-660) with the
reference's own kernel arithmetic in FP64 (oracle/pic_oracle.c: the CIC
deposit of src/Grid.py:96-154, E of :157-196, the kick of
src/Particles.py:117-180 and the drift of :251-264), wall absorption on all
four walls in place of the axis reflection, and the Poisson equation solved
exactly by a sparse LU of the 5-point operator with its Dirichlet rows
(the reference's 'direct' branch, src/Solvers.py:59-96,169-195,269-299,
without the dx^2 double count).  Positions are carried in metres.

The tests use it as the FP64 yardstick for the FP32 build: trajectories,
densities, potentials and fields after N steps.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import oracle as O

QE, ME, EPS0 = 1.6e-19, 9.10938356e-31, 8.85418782e-12


class Fp64Run:
    """A two-species collisionless run.

    arrays: per species (x, y, vx, vy, ...) with positions in grid units
    (float32, as loaded into the build); charges, masses and np2c per species;
    mask / phi_bc: Dirichlet node mask and values (m*m, node-major)."""

    def __init__(self, m, dx, dt, arrays, charges, masses, np2c, mask, phi_bc):
        self.m, self.dx, self.dt = int(m), float(dx), float(dt)
        self.q, self.mass, self.np2c = list(charges), list(masses), list(np2c)
        self.mask, self.phi_bc = np.asarray(mask), np.asarray(phi_bc, np.float64)
        m = self.m
        size = m * m
        off = np.ones(size)
        off[m - 1::m] = 0
        A = sp.diags([np.full(size, -4.0), off[:-1], off[:-1], np.ones(size - m), np.ones(size - m)],
                     [0, 1, -1, m, -m], (size, size), format="lil") / dx**2
        A = A.tolil()
        for k in np.flatnonzero(self.mask):
            A.rows[k] = [k]
            A.data[k] = [1.0]
        self.lu = spla.splu(A.tocsc())
        self.P = [[a[0].astype(np.float64) * dx, a[1].astype(np.float64) * dx, a[2].astype(np.float64),
                   a[3].astype(np.float64)] for a in arrays]
        self.L = dx * (m - 1)
        self.absorbed = [0] * len(self.P)
        self.rho = self.phi = self.E = None

    def solve(self):
        """Deposit (C/m^3), direct solve, E; stores rho, phi and E (the grid state after the solve)."""
        m, dx = self.m, self.dx
        rho = np.zeros(m * m)
        for s, P in enumerate(self.P):
            live = ~np.isnan(P[0])
            O.deposit_f64(P[0][live], P[1][live], self.q[s] * self.np2c[s], dx, dx, m, m, rho=rho,
                          floorf_quirk=False)
        b = -rho / (dx * dx) / EPS0
        b[self.mask == 1] = self.phi_bc[self.mask == 1]
        self.rho = rho / (dx * dx)
        self.phi = self.lu.solve(b)
        self.E = O.update_E_f64(self.phi, m, m, dx, dx)
        return self.E

    def kick(self, factor):
        ex, ey = self.E
        for s, P in enumerate(self.P):
            live = ~np.isnan(P[0])
            vx, vy = P[2][live].copy(), P[3][live].copy()
            O.lib().or_update_V_f64(P[0][live].copy(), P[1][live].copy(), vx, vy, int(live.sum()), ex, ey,
                                    self.dt * factor * self.q[s] / self.mass[s], self.dx, self.dx, self.m, self.m, 0)
            P[2][live], P[3][live] = vx, vy

    def init(self):
        """_init_step: deposit, solve, E, v(-dt/2)."""
        self.solve()
        self.kick(-0.5)

    def step(self):
        """One _step: drift, absorb, deposit, solve, E, kick."""
        for s, P in enumerate(self.P):
            live = ~np.isnan(P[0])
            x, y = P[0][live].copy(), P[1][live].copy()
            O.lib().or_update_R_f64(x, y, P[2][live].copy(), P[3][live].copy(), len(x), self.dt)
            self.absorbed[s] += int(O.lib().or_absorb_f64(x, y, len(x), self.L, self.L))
            P[0][live], P[1][live] = x, y
        self.solve()
        self.kick(1.0)


def fp64_reference_run(w, arrays, steps, charges, masses):
    """Init plus `steps` steps of workload w; returns the Fp64Run."""
    from pic_b200 import workloads

    mask, phi_bc = workloads.dirichlet(w)
    run = Fp64Run(w.nodes, w.dx, w.dt, arrays, charges, masses, [w.np2c(w.n_e), w.np2c(w.n_i)], mask, phi_bc)
    run.init()
    for _ in range(steps):
        run.step()
    return run
