"""FP64 CPU restatement of the differentiable collisionless step (test
infrastructure only: the GPU adjoint's checker).

Forward model, in the reference's step order (src/simulation.py:622-660):
  init:  rho_0 = D(x_0) (CIC, src/Grid.py:96-154), phi_0 = P(rho_0; V),
         E_0 = -grad phi_0 (src/Grid.py:167-194), u_0 = v_0 + A dv - (k/2) I(x_0; E_0)
  step:  x += (dt/dx) u (src/Particles.py:251-264); a particle outside
         [0, n-1]^2 is absorbed; rho, phi, E at the new positions;
         u += k I(x; E) (src/Particles.py:117-180)
  loss:  mean over nodes of (n_s(x_N) - target)^2
P solves the 5-point Laplacian with f = -rho/eps0 on free nodes and the
electrode potentials on Dirichlet nodes, directly (scipy sparse LU: the
reference's `direct` formulation, src/Solvers.py:59-96,169-195, with the RHS
scaled once by 1/h^2 through the operator).  Gradients here are central
finite differences of this forward model: the FP64 reference gradient.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class RefDifferentiable:
    def __init__(self, nx, ny, dx, dy, dt, eps0, species, mask, segment, nseg, steps, loss_species, target,
                 phi_fixed=None):
        """species: list of dicts with charge, mass, np2c and arrays x, y, vx, vy (grid units, m/s), dvx, dvy."""
        self.nx, self.ny, self.dx, self.dy, self.dt, self.eps0 = nx, ny, dx, dy, dt, eps0
        self.species = species
        self.steps = steps
        self.loss_species = loss_species
        self.target = np.asarray(target, np.float64).reshape(-1)
        self.nseg = nseg
        G = nx * ny
        m = np.asarray(mask, np.uint8).reshape(ny, nx).copy()
        m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = 1
        self.mask = m.reshape(-1).astype(bool)
        self.seg = np.asarray(segment, np.int64).reshape(-1)
        self.fixed = np.zeros(G) if phi_fixed is None else np.asarray(phi_fixed, np.float64).reshape(-1)
        # interior operator
        free = np.flatnonzero(~self.mask)
        self.free = free
        where = -np.ones(G, np.int64)
        where[free] = np.arange(free.size)
        cx, cy = 1.0 / dx ** 2, 1.0 / dy ** 2
        rows, cols, vals = [], [], []
        brow, bcol, bval = [], [], []
        for a, k in enumerate(free):
            rows.append(a)
            cols.append(a)
            vals.append(-2.0 * (cx + cy))
            for nb, c in ((k - 1, cx), (k + 1, cx), (k - nx, cy), (k + nx, cy)):
                if where[nb] >= 0:
                    rows.append(a)
                    cols.append(where[nb])
                    vals.append(c)
                else:
                    brow.append(a)
                    bcol.append(nb)
                    bval.append(c)
        A = sp.csc_matrix((vals, (rows, cols)), shape=(free.size, free.size))
        self.lu = spla.splu(A)
        self.B = sp.csr_matrix((bval, (brow, bcol)), shape=(free.size, G))

    # ---- pieces ----
    def _cell(self, x, y):
        i = np.clip(np.floor(x).astype(np.int64), 0, self.nx - 2)
        j = np.clip(np.floor(y).astype(np.int64), 0, self.ny - 2)
        return i, j, x - i, y - j

    def _deposit(self, x, y, w):
        i, j, fx, fy = self._cell(x, y)
        rho = np.zeros(self.nx * self.ny)
        k = j * self.nx + i
        np.add.at(rho, k, (1 - fx) * (1 - fy) * w)
        np.add.at(rho, k + 1, fx * (1 - fy) * w)
        np.add.at(rho, k + self.nx, (1 - fx) * fy * w)
        np.add.at(rho, k + self.nx + 1, fx * fy * w)
        return rho

    def _interp(self, F, x, y):
        i, j, fx, fy = self._cell(x, y)
        k = j * self.nx + i
        return ((1 - fx) * (1 - fy) * F[k] + fx * (1 - fy) * F[k + 1] + (1 - fx) * fy * F[k + self.nx]
                + fx * fy * F[k + self.nx + 1])

    def _solve(self, rho, phiB):
        f = -rho[self.free] / self.eps0 - self.B @ phiB
        phi = phiB.copy()
        phi[self.free] = self.lu.solve(f)
        return phi

    def _efield(self, phi):
        p = phi.reshape(self.ny, self.nx)
        ex = np.empty_like(p)
        ey = np.empty_like(p)
        ex[:, 1:-1] = -(p[:, 2:] - p[:, :-2]) / (2 * self.dx)
        ex[:, 0] = -(p[:, 1] - p[:, 0]) / self.dx
        ex[:, -1] = -(p[:, -1] - p[:, -2]) / self.dx
        ey[1:-1, :] = -(p[2:, :] - p[:-2, :]) / (2 * self.dy)
        ey[0, :] = -(p[1, :] - p[0, :]) / self.dy
        ey[-1, :] = -(p[-1, :] - p[-2, :]) / self.dy
        return ex.reshape(-1), ey.reshape(-1)

    # ---- forward ----
    def run(self, V, A):
        """(loss, final positions per species, final alive masks)."""
        phiB = np.where(self.mask, self.fixed, 0.0)
        for q in range(self.nseg):
            phiB[self.mask & (self.seg == q)] = V[q]
        st = []
        for s in self.species:
            st.append(dict(x=np.array(s["x"], np.float64), y=np.array(s["y"], np.float64),
                           ux=np.array(s["vx"], np.float64) + A * np.asarray(s.get("dvx", 0.0)),
                           uy=np.array(s["vy"], np.float64) + A * np.asarray(s.get("dvy", 0.0)),
                           alive=np.ones(len(s["x"]), bool),
                           k=s["charge"] * self.dt / s["mass"], w=s["charge"] * s["np2c"] / (self.dx * self.dy)))

        def fields():
            rho = np.zeros(self.nx * self.ny)
            for p in st:
                a = p["alive"]
                rho += self._deposit(p["x"][a], p["y"][a], p["w"])
            return self._efield(self._solve(rho, phiB))

        ex, ey = fields()
        for p in st:
            a = p["alive"]
            p["ux"][a] -= 0.5 * p["k"] * self._interp(ex, p["x"][a], p["y"][a])
            p["uy"][a] -= 0.5 * p["k"] * self._interp(ey, p["x"][a], p["y"][a])
        cx, cy = self.dt / self.dx, self.dt / self.dy
        for _ in range(self.steps):
            for p in st:
                a = p["alive"]
                p["x"][a] += cx * p["ux"][a]
                p["y"][a] += cy * p["uy"][a]
                out = ~((p["x"] >= 0) & (p["x"] <= self.nx - 1) & (p["y"] >= 0) & (p["y"] <= self.ny - 1))
                p["alive"] &= ~out
            ex, ey = fields()
            for p in st:
                a = p["alive"]
                p["ux"][a] += p["k"] * self._interp(ex, p["x"][a], p["y"][a])
                p["uy"][a] += p["k"] * self._interp(ey, p["x"][a], p["y"][a])
        L = self.species[self.loss_species]
        p = st[self.loss_species]
        a = p["alive"]
        dens = self._deposit(p["x"][a], p["y"][a], L["np2c"] / (self.dx * self.dy))
        loss = float(np.mean((dens - self.target) ** 2))
        return loss, [(q["x"], q["y"]) for q in st], [q["alive"] for q in st]

    def loss(self, V, A):
        return self.run(V, A)[0]

    def gradient_fd(self, V, A, hV=1e-3, hA=1.0):
        """Central differences: (dL/dV[nseg], dL/dA)."""
        V = np.asarray(V, np.float64)
        dV = np.zeros(self.nseg)
        for q in range(self.nseg):
            e = np.zeros(self.nseg)
            e[q] = hV
            dV[q] = (self.loss(V + e, A) - self.loss(V - e, A)) / (2 * hV)
        dA = (self.loss(V, A + hA) - self.loss(V, A - hA)) / (2 * hA)
        return dV, dA
