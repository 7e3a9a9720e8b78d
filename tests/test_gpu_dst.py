"""The sine-transform Poisson solve (PIC_MG_DST) on the GPU.

* The exact discrete eigenmode solution (FP64 round-off, ~1e-14 of its
  maximum) from 17^2 to 2049^2 nodes.
* Edge values and unequal spacings against the oracle's direct sparse solve,
  and square grids against the oracle's restatement of the reference's
  poisson_fft_dirichlet (src/FFT.py:10-64), to 1e-11 of the solution.
* The reported residual against the oracle's FP64 recomputation.
* Grids it does not apply to (internal electrodes, r-z, node counts other
  than 2^q + 1) fall back to the graph-loop multigrid.
* The fused step with the DST solve: the same potential as with the
  multigrid, to the multigrid's tolerance.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from oracle import oracle as O
from pic_b200 import Consts, workloads
from pic_b200.multigrid import MultigridSolver
from pic_b200.simulation import PICSimulation

pytestmark = pytest.mark.gpu
DEV = "cuda"


def edge_mask(m, n):
    mk = np.zeros((n, m), np.uint8)
    mk[0, :] = mk[-1, :] = mk[:, 0] = mk[:, -1] = 1
    return mk.reshape(-1)


@pytest.mark.parametrize("n", [17, 129, 513, 2049])
def test_eigenmode_exact(n):
    h = 1.0 / (n - 1)
    x = np.linspace(0, 1, n)
    X, Y = np.meshgrid(x, x)
    f = (-np.sin(np.pi * X) * np.sin(np.pi * Y)).reshape(-1)
    exact = (np.sin(np.pi * X) * np.sin(np.pi * Y)).reshape(-1) / ((8 / h**2) * np.sin(np.pi * h / 2) ** 2)
    mask = edge_mask(n, n)
    f[mask == 1] = 0.0
    mg = MultigridSolver(mask, n, n, h, launch="dst")
    assert mg.effective_launch() == "dst"
    phi = torch.zeros(n * n, dtype=torch.float64, device=DEV)
    phi, (cycles, rel) = mg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-9)
    # the FP64 residual of the exact solution is round-off of terms ~ phi / h^2: it grows as n^2 eps
    assert cycles == 0 and rel < 2e-16 * n * n, rel
    np.testing.assert_allclose(phi.cpu().numpy(), exact, rtol=0, atol=2e-14 * np.abs(exact).max() * np.log2(n))


@pytest.mark.parametrize("shape,dx,dy", [((65, 65), 1e-3, 1e-3), ((129, 33), 2e-4, 5e-4), ((33, 257), 1.0, 0.25)])
def test_edge_values_against_direct_solve(shape, dx, dy):
    m, n = shape
    rng = np.random.default_rng(11)
    f = rng.normal(0, 1e3, m * n)
    g = rng.normal(0, 10.0, m * n)
    mask = edge_mask(m, n)
    f[mask == 1] = 0.0
    phi_bc = np.where(mask == 1, g, 0.0)
    # direct sparse solve of the Cartesian 5-point system
    size = m * n
    A = sp.lil_matrix((size, size))
    b = f.copy()
    for k in range(size):
        j, i = divmod(k, m)
        if mask[k]:
            A[k, k] = 1.0
            b[k] = phi_bc[k]
        else:
            A[k, k] = -2.0 / dx**2 - 2.0 / dy**2
            A[k, k - 1] = A[k, k + 1] = 1.0 / dx**2
            A[k, k - m] = A[k, k + m] = 1.0 / dy**2
    direct = spla.spsolve(A.tocsr(), b)
    mg = MultigridSolver(mask, m, n, dx, hy=dy, launch="dst")
    phi = torch.as_tensor(phi_bc, device=DEV)
    phi, (cycles, rel) = mg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-10)
    got = phi.cpu().numpy()
    np.testing.assert_allclose(got, direct, rtol=0, atol=1e-11 * np.abs(direct).max())
    # the residual of an exact solve is round-off: both the reported and the recomputed one are tiny
    cpu = np.sqrt(O.residual_f64(got, f, mask, m, n, dx, dy) / np.sum(f * f))
    assert rel < 1e-9 and cpu < 1e-9, (rel, cpu)


@pytest.mark.parametrize("n", [33, 257])
def test_matches_the_reference_restatement(n):
    rng = np.random.default_rng(3)
    h = 1e-3
    f2 = rng.normal(0, 1e4, (n, n))
    g2 = rng.normal(0, 5.0, (n, n))
    want = O.poisson_fft_dirichlet(f2, g2, h)
    mask = edge_mask(n, n)
    f = f2.reshape(-1).copy()
    f[mask == 1] = 0.0
    phi = torch.as_tensor(np.where(mask == 1, g2.reshape(-1), 0.0), device=DEV)
    mg = MultigridSolver(mask, n, n, h, launch="dst")
    phi, _ = mg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-10)
    np.testing.assert_allclose(phi.cpu().numpy(), want.reshape(-1), rtol=0, atol=1e-11 * np.abs(want).max())


def test_falls_back_where_it_does_not_apply():
    n = 129
    mask = edge_mask(n, n)
    mask[40 * n + 30: 40 * n + 60] = 1  # an internal electrode
    assert MultigridSolver(mask, n, n, 1e-3, launch="dst").effective_launch() == "graph"
    assert MultigridSolver(edge_mask(n, n), n, n, 1e-3, launch="dst", geometry="rz").effective_launch() == "graph"
    m = 97  # 3 * 32 + 1: a multigrid grid, not a power of two
    assert MultigridSolver(edge_mask(m, m), m, m, 1e-3, launch="dst").effective_launch() == "graph"


def test_fused_step_with_the_dst_solve():
    w = workloads.scaled(workloads.SMALL, n=40_000, left_V=50.0)
    mask, phi_bc = workloads.dirichlet(w)
    sims = []
    for launch, tol in (("dst", 1e-8), ("graph", 1e-11)):
        sp_ = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
               dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
        sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp_, mask, phi_bc, tol=tol, max_cycles=80,
                            sort_interval=0, mg_launch=launch, use_graph=True)
        rng = np.random.Generator(np.random.Philox(w.seed))
        for s, which in enumerate("ei"):
            sim.load(s, *workloads.species_arrays(w, which, rng))
        sim.init()
        sims.append(sim)
    phi_d, rho_d = (t.cpu().numpy() for t in sims[0].fields()[:2])
    phi_m = sims[1].fields()[0].cpu().numpy()
    assert sims[0].counters()["last_cycles"] == 0
    # the same deposit, so the same potential: DST exact, multigrid to 1e-11
    np.testing.assert_allclose(phi_d, phi_m, rtol=0, atol=1e-8 * np.abs(phi_m).max())
    f = -rho_d.astype(np.float64) / Consts.eps0
    f[mask == 1] = 0.0
    m = w.nodes
    assert np.sqrt(O.residual_f64(phi_d, f, mask, m, m, w.dx, w.dx) / np.sum(f * f)) < 1e-11
    for sim in sims:
        sim.step(5)
        sim.sync()
        assert sim.counters()["steps"] == 5
        sim.close()
