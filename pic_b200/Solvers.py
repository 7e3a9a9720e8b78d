"""Solver: drop-in for src/Solvers.py:198-299, Cartesian or r-z.

``solve(grid)`` forms b = -rho/eps0 on free nodes (without the reference's
extra dx^2, src/Solvers.py:271, which its multigrid then applies a second
time), keeps the Dirichlet values in phi, and solves on the GPU: the
multigrid; for 'cg' and 'gmres' (cupyx library solvers in the reference),
conjugate gradients preconditioned by a V-cycle; for 'direct' and 'inverse'
(a sparse LU and a dense inverse there), an exact solve.

cylindrical=True solves the axisymmetric equation (the operator the
reference builds in Laplacian_cylindrical_csr, src/Solvers.py:100-166, and
hands only to its cupyx solvers; its multigrid stays Cartesian): row 0 is the
axis, a free row, and the r-weights are (1 +- 1/2j) / dr^2, with 4 / dr^2 on
the axis.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Consts, _lib
from .multigrid import ConjugateGradientSolver, MultigridSolver

SOLVER_TYPES = ("multigrid", "cg", "gmres", "direct", "inverse")


class Solver:
    """solver_type (src/Solvers.py:219-258): 'multigrid'; 'cg' and 'gmres',
    preconditioned conjugate gradients (ConjugateGradientSolver; Cartesian);
    'direct' and 'inverse', an exact solve: the sine-transform solve where its
    grid qualifies (Cartesian, edge-only Dirichlet nodes, 2^q + 1 nodes), else
    the multigrid to min(tol, 1e-12)."""

    def __init__(self, solver_type, grid, cylindrical=False, boundaries=None, tol=1e-5, precision="mixed",
                 max_cycles=50):
        if solver_type not in SOLVER_TYPES:
            raise NotImplementedError(f"solver_type={solver_type!r}: one of {SOLVER_TYPES}")
        if cylindrical and solver_type in ("cg", "gmres"):
            raise NotImplementedError("the conjugate-gradient solve is Cartesian; use 'multigrid' in r-z")
        self.solver_type = solver_type
        self.m, self.n = grid.m, grid.n
        self.dx, self.dy = grid.dx, grid.dy
        self.cylindrical = bool(cylindrical)
        self.tol = tol
        self.max_cycles = max_cycles
        self.boundaries = boundaries
        if boundaries is not None:
            mask = boundaries.bc_lookup_host.astype(np.uint8)
            self.phi_bc = torch.as_tensor(boundaries.phi_bc_host, device=grid.phi.device)
        else:
            mask = np.zeros(grid.m * grid.n, np.uint8)
            self.phi_bc = None
        # the grid edges are always Dirichlet nodes of the 5-point operator
        # (in r-z all but the axis row)
        m2 = mask.reshape(grid.n, grid.m)
        self._edge_mask = m2.copy()
        self._edge_mask[-1, :] = self._edge_mask[:, 0] = self._edge_mask[:, -1] = 1
        if not self.cylindrical:
            self._edge_mask[0, :] = 1
        self.dirichlet = torch.as_tensor(self._edge_mask.reshape(-1), device=grid.phi.device)
        exact = solver_type in ("direct", "inverse")
        self.multigrid = MultigridSolver(self._edge_mask.reshape(-1), grid.m, grid.n, grid.dx, omega=1.15,
                                         precision=precision, hy=grid.dy,
                                         geometry="rz" if self.cylindrical else "cartesian",
                                         launch="dst" if exact else "graph")
        if exact:
            self.tol = min(float(tol), 1e-12) if self.multigrid.effective_launch() != "dst" else float(tol)
        self.cg = (ConjugateGradientSolver(self._edge_mask.reshape(-1), grid.m, grid.n, grid.dx, hy=grid.dy,
                                           precond=self.multigrid) if solver_type in ("cg", "gmres") else None)
        self.last_info = None
        if self.phi_bc is not None:
            bc = torch.as_tensor(boundaries.bc_lookup_host, device=grid.phi.device).bool()
            grid.phi[bc] = self.phi_bc[bc]

    def solve(self, grid):
        _lib.call("pic_form_rhs", _lib.ptr(grid.rho), _lib.ptr(self.dirichlet), Consts.eps0, _lib.ptr(grid.b),
                  grid.m, grid.n, _lib.stream_ptr())
        if self.cg is not None:
            grid.phi, info = self.cg.solve(grid.phi, grid.b, tol=self.tol, max_iter=max(self.max_cycles, 100))
            self.last_info = self.cg.last_info
            return info
        grid.phi, info = self.multigrid.solve(grid.phi, grid.b, tol=self.tol, max_cycles=self.max_cycles)
        self.last_info = self.multigrid.last_info
        return info
