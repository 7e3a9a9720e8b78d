"""The solver branches of the drop-in Solver (src/Solvers.py:198-299) on the GPU.

* Preconditioned conjugate gradients (pic_cg, the 'cg' and 'gmres' branches)
  against the reference's direct formulation (5-point CSR with Dirichlet
  rows, scipy's sparse LU), with electrodes on odd grid lines, with and
  without the V-cycle preconditioner, to 1e-9 of the solution.
* Every branch of Solver ('multigrid', 'cg', 'gmres', 'direct', 'inverse')
  gives the same potential for the same deposited charge; 'direct' uses the
  sine-transform solve where the grid qualifies.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from pic_b200 import Consts
from pic_b200.Boundaries import Boundaries, walls_box
from pic_b200.Grid import Grid2D
from pic_b200.multigrid import ConjugateGradientSolver, MultigridSolver
from pic_b200.Particles import Particles2D
from pic_b200.Solvers import Solver

pytestmark = pytest.mark.gpu
DEV = "cuda"


def direct(m, n, h, mask, phi_bc, f):
    size = m * n
    A = sp.lil_matrix((size, size))
    b = f.copy()
    for k in range(size):
        j, i = divmod(k, m)
        if mask[k] or i in (0, m - 1) or j in (0, n - 1):
            A[k, k] = 1.0
            b[k] = phi_bc[k]
        else:
            A[k, k] = -4.0 / h**2
            for q in (k - 1, k + 1, k - m, k + m):
                A[k, q] = 1.0 / h**2
    return spla.spsolve(A.tocsr(), b)


def problem(m, n, h, seed=4):
    rng = np.random.default_rng(seed)
    mask = np.zeros(m * n, np.uint8)
    e = np.zeros((n, m), np.uint8)
    e[0, :] = e[-1, :] = e[:, 0] = e[:, -1] = 1
    mask = e.reshape(-1).copy()
    phi_bc = np.zeros(m * n)
    phi_bc.reshape(n, m)[1:-1, 0] = 25.0
    j, i = np.divmod(np.arange(m * n), m)
    el = (i == 43) & (j > 10) & (j < 50)
    mask[el] = 1
    phi_bc[el] = -30.0
    f = rng.normal(0, 1e6, m * n)
    f[mask == 1] = 0.0
    return mask, phi_bc, f


@pytest.mark.parametrize("precond", [True, False])
def test_conjugate_gradients_against_direct_solve(precond):
    m, n, h = 129, 65, 1e-4
    mask, phi_bc, f = problem(m, n, h)
    ref = direct(m, n, h, mask, phi_bc, f)
    mg = MultigridSolver(mask, m, n, h) if precond else None
    cg = ConjugateGradientSolver(mask, m, n, h, precond=mg)
    phi = torch.as_tensor(phi_bc.copy(), device=DEV)
    phi, (iters, rel) = cg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-10, max_iter=2000, raise_on_fail=True)
    assert rel < 1e-10
    # a V-cycle preconditioner takes a handful of iterations; plain CG hundreds
    assert (iters <= 25) if precond else (iters > 50), iters
    np.testing.assert_allclose(phi.cpu().numpy(), ref, rtol=0, atol=1e-9 * np.abs(ref).max())


def test_every_solver_branch_gives_the_same_potential():
    m = n = 129
    X = Y = 0.0128
    grid = Grid2D(m, n, X, Y)
    parts = Particles2D(100_000)
    parts.add_species("electrons", Consts.me, -Consts.qe, 0)
    parts.add_species("ions", 40 * 1.66e-27, Consts.qe, 1)
    parts.grid = grid
    parts.np2c = 1e5
    for s in ("electrons", "ions"):
        parts.maxwellian_species_load(0.002, 0.002, 0.011, 0.011, 50_000, s, 1.0, seed=7 if s == "ions" else 8,
                                      grid=grid)
    bnd = Boundaries(walls_box(grid, left=40.0), grid)
    grid.update_density(parts)
    out = {}
    for kind in ("multigrid", "cg", "gmres", "direct", "inverse"):
        grid.phi.zero_()
        solver = Solver(kind, grid, boundaries=bnd, tol=1e-11, precision="fp64")
        solver.solve(grid)
        assert solver.last_info.converged, kind
        out[kind] = grid.phi.cpu().numpy().copy()
        if kind == "direct":
            assert solver.multigrid.effective_launch() == "dst"
    ref = out["direct"]
    for kind, phi in out.items():
        np.testing.assert_allclose(phi, ref, rtol=0, atol=1e-8 * np.abs(ref).max(), err_msg=kind)


def test_cg_refuses_rz():
    grid = Grid2D(65, 33, 0.01, 0.005, cylindrical=True)
    with pytest.raises(NotImplementedError):
        Solver("cg", grid, cylindrical=True)
