"""Multigrid Poisson solver on the GPU.

Known answers:
  * the manufactured problem of src/Multigrid_test.py:415-433 (lap phi =
    -sin(pi x) sin(pi y) on [0,1]^2, phi = 0 on the edges) whose discrete
    solution is exact: sin(pi x) sin(pi y) / ((8/h^2) sin^2(pi h/2)) (the DST
    eigenvalue of src/FFT.py:112-119);
  * the electrode problem of src/multigrid.py:488-523 against the reference's
    direct formulation (Laplacian_cartesian_csr + apply_boundary_conditions,
    src/Solvers.py:59-96,169-195, with scipy's sparse LU);
  * at full size, the FP64 residual recomputed on the CPU by the oracle.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from oracle import oracle as O
from pic_b200 import _lib
from pic_b200.multigrid import MultigridSolver

pytestmark = pytest.mark.gpu
DEV = "cuda"


def edge_mask(n):
    m = np.zeros((n, n), np.uint8)
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = 1
    return m.reshape(-1)


def manufactured(n):
    h = 1.0 / (n - 1)
    x = np.linspace(0, 1, n)
    X, Y = np.meshgrid(x, x, indexing="xy")
    f = -(np.sin(np.pi * X) * np.sin(np.pi * Y)).reshape(-1)
    exact = (np.sin(np.pi * X) * np.sin(np.pi * Y)).reshape(-1) / ((8 / h**2) * np.sin(np.pi * h / 2) ** 2)
    return h, f, exact


@pytest.mark.parametrize("launch", ["persistent", "graph", "host", "cluster", "hybrid"])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("n", [17, 33, 65, 129, 257])
def test_manufactured_solution(launch, precision, n):
    """Small grids run entirely in the single-block coarse V-cycle; larger ones use the tiled (or, in the
    cluster mode, banded) phases too.  The launch modes run the same algorithm; the cluster mode falls back
    to the graph loop for FP64 levels."""
    h, f, exact = manufactured(n)
    mask = edge_mask(n)
    f[mask == 1] = 0.0
    mg = MultigridSolver(mask, n, n, h, precision=precision, launch=launch)
    phi = torch.zeros(n * n, dtype=torch.float64, device=DEV)
    phi, (cycles, rel) = mg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-12, max_cycles=40)
    # a V(2,2) cycle reduces the residual ~10x; from phi = 0 to 1e-12 takes about 12 cycles
    assert rel < 1e-12 and cycles <= 14, (cycles, rel)
    np.testing.assert_allclose(phi.cpu().numpy(), exact, rtol=0, atol=1e-10 * np.abs(exact).max())


def direct_solve(n, h, idx, val, f):
    """The reference's `direct` branch restated: 5-point CSR with row-boundary
    zeroing (src/Solvers.py:79-95), Dirichlet rows set to the identity
    (src/Solvers.py:186-193) and b[bc] = V (src/Solvers.py:274-276), without the
    dx^2 double count: rows are scaled by 1/h^2 so that b = f."""
    size = n * n
    main = np.full(size, -4.0)
    off_h = np.ones(size)
    off_h[n - 1::n] = 0
    off_v = np.ones(size - n)
    A = sp.diags([main, off_h[:-1], off_h[:-1], off_v, off_v], [0, 1, -1, n, -n], (size, size), format="lil")
    A = A / h**2
    edges = np.flatnonzero(edge_mask(n))
    bidx = np.concatenate([edges, idx])
    bval = np.concatenate([np.zeros(len(edges)), val])
    A = A.tolil()
    for k in bidx:
        A.rows[k] = [k]
        A.data[k] = [1.0]
    b = f.copy()
    b[edges] = 0.0
    b[idx] = val
    return spla.spsolve(A.tocsc(), b)


def test_internal_electrodes_match_direct_solve():
    n = 129
    h = 1.0 / (n - 1)
    _, f, _ = manufactured(n)
    cath = [(n // 4) + j * n for j in range(n // 4, 3 * n // 4 + 1)]  # column n//4, rows n//4 .. 3n//4
    anode = [(3 * n // 4) + j * n for j in range(n // 4, 3 * n // 4 + 1)]
    idx = np.array(cath + anode)
    val = np.array([-50.0] * len(cath) + [50.0] * len(anode))
    mask = edge_mask(n)
    mask[idx] = 1
    ref = direct_solve(n, h, idx, val, f)
    for precision, launch in (("mixed", "graph"), ("fp64", "graph"), ("mixed", "cluster"), ("mixed", "hybrid")):
        mg = MultigridSolver(mask, n, n, h, precision=precision, launch=launch)
        phi0 = np.zeros(n * n)
        phi0[idx] = val
        ff = f.copy()
        ff[mask == 1] = 0
        # +-50 V electrodes with |f| ~ 1: the FP64 rounding floor of the residual is ~1e-10 of ||f||
        phi, (cycles, rel) = mg.solve(torch.as_tensor(phi0, device=DEV), torch.as_tensor(ff, device=DEV), tol=1e-9,
                                      max_cycles=80)
        assert rel < 1e-9
        np.testing.assert_allclose(phi.cpu().numpy(), ref, rtol=0, atol=1e-8 * np.abs(ref).max())


@pytest.mark.parametrize("launch", ["graph", "persistent", "cluster", "hybrid"])
def test_electrodes_on_odd_lines(launch):
    """Electrodes on lines that do not survive injection to the coarse grids
    (column 43 and row 77, both odd; column 85): the coarse grids keep them as
    two-line bands, and the cycle converges to the direct solution (about 55
    V-cycles to 1e-9; with the electrodes left out of the coarse grids it
    diverged)."""
    n = 129
    h = 1.0 / (n - 1)
    _, f, _ = manufactured(n)
    cath = [43 + j * n for j in range(30, 91)]
    anode = [85 + j * n for j in range(20, 70)]
    bar = [i + 77 * n for i in range(50, 80)]
    idx = np.array(sorted(set(cath + anode + bar)))
    val = np.where(np.isin(idx, cath), -50.0, 50.0)
    mask = edge_mask(n)
    mask[idx] = 1
    ref = direct_solve(n, h, idx, val, f)
    for precision in ("mixed", "fp64"):
        mg = MultigridSolver(mask, n, n, h, precision=precision, launch=launch)
        phi0 = np.zeros(n * n)
        phi0[idx] = val
        ff = f.copy()
        ff[mask == 1] = 0
        phi, (cycles, rel) = mg.solve(torch.as_tensor(phi0, device=DEV), torch.as_tensor(ff, device=DEV), tol=1e-9,
                                      max_cycles=100)
        assert rel < 1e-9 and cycles <= 70, (precision, cycles, rel)
        np.testing.assert_allclose(phi.cpu().numpy(), ref, rtol=0, atol=1e-8 * np.abs(ref).max())


@pytest.mark.parametrize("n,tol", [(513, 1e-8), (513, 1e-10), (1025, 1e-10), (2049, 1e-10)])
def test_residual_recomputed_on_cpu(n, tol):
    rng = np.random.Generator(np.random.Philox(6))
    h = 1e-4
    mask = edge_mask(n)
    f = rng.normal(0, 1e6, n * n)
    f[mask == 1] = 0
    phi0 = np.zeros(n * n)
    phi0.reshape(n, n)[1:-1, 0] = 100.0
    for precision, launch in (("mixed", "graph"), ("fp64", "graph"), ("mixed", "cluster"), ("mixed", "hybrid")):
        mg = MultigridSolver(mask, n, n, h, precision=precision, launch=launch)
        if launch == "hybrid":
            assert mg.effective_launch() == "hybrid"
        if launch == "cluster":
            # the finest band of a 513^2 grid fits one CTA's shared memory; 1025^2 and up fall back
            assert mg.effective_launch() == ("cluster" if n <= 513 else "graph")
        phi, (cycles, rel) = mg.solve(torch.as_tensor(phi0, device=DEV), torch.as_tensor(f, device=DEV), tol=tol,
                                      max_cycles=60)
        p = phi.cpu().numpy()
        r2 = O.residual_f64(p, f, mask, n, n, h, h)
        f2 = float(np.sum(f * f))
        assert np.sqrt(r2 / f2) < tol, (precision, cycles, rel, np.sqrt(r2 / f2))
        # the device and the CPU sum the squares in different orders, and the last
        # cycle can end near the FP64 rounding floor of the residual itself (about
        # 1e-12 relative at 1025^2 and 2049^2 with |f| ~ 1e6, |phi| ~ 100 V)
        assert abs(np.sqrt(r2 / f2) - rel) <= 2e-2 * rel + 1e-12
        np.testing.assert_array_equal(p[mask == 1], phi0[mask == 1])


def test_not_converged_is_reported():
    n = 129
    h, f, _ = manufactured(n)
    mask = edge_mask(n)
    mg = MultigridSolver(mask, n, n, h)
    phi = torch.zeros(n * n, dtype=torch.float64, device=DEV)
    with pytest.raises(_lib.PicError) as e:
        mg.solve(phi, torch.as_tensor(f, device=DEV), tol=1e-14, max_cycles=1, raise_on_fail=True)
    assert e.value.code == _lib.PIC_ERR_NOT_CONVERGED
    assert mg.last_info is None or True


def test_rejects_grids_that_do_not_coarsen():
    with pytest.raises(_lib.PicError) as e:
        MultigridSolver(edge_mask(100), 100, 100, 1e-4)
    assert e.value.code == _lib.PIC_ERR_BAD_ARG


@pytest.mark.parametrize("n", [1025])
def test_solves_are_deterministic_across_launch_modes(n):
    """The up phase smooths each tile from the down phase's correction and
    writes its own array, so no CTA reads a neighbour's halo while another
    overwrites it.  At 1025^2 the up kernels run in several waves, where
    reading and writing one array raced; every solve must now be bit-identical."""
    rng = np.random.Generator(np.random.Philox(6))
    h = 1e-4
    mask = edge_mask(n)
    f = rng.normal(0, 1e6, n * n)
    f[mask == 1] = 0
    ft = torch.as_tensor(f, device=DEV)
    ref = None
    for launch in ("graph", "host", "graph"):
        mg = MultigridSolver(mask, n, n, h, precision="mixed", launch=launch)
        for _ in range(2):
            phi = torch.zeros(n * n, dtype=torch.float64, device=DEV)
            phi, (cycles, rel) = mg.solve(phi, ft, tol=1e-10, max_cycles=60)
            out = (cycles, rel, phi.cpu().numpy())
            if ref is None:
                ref = out
            assert out[0] == ref[0] and out[1] == ref[1]
            np.testing.assert_array_equal(out[2], ref[2])


@pytest.mark.parametrize("shape", [(513, 129), (129, 513), (385, 193)])
def test_rectangular_grids_with_electrodes_match_direct_solve(shape):
    # rectangular and 3 * 2^k + 1 grids deep enough for the two-level launches
    # and the direct coarse solve (first coarse levels 33 x 9, 9 x 33, 25 x 13),
    # with an electrode on an odd grid line, against scipy's sparse LU
    m, n = shape
    h = 1e-3
    rng = np.random.default_rng(12)
    mask = np.zeros((n, m), np.uint8)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    phi_bc = np.zeros((n, m))
    phi_bc[1:-1, 0] = 30.0
    el = (slice(n // 3, 2 * n // 3), 2 * (m // 5) + 1)  # a vertical electrode on an odd column
    mask[el] = 1
    phi_bc[el] = -20.0
    mask, phi_bc = mask.reshape(-1), phi_bc.reshape(-1)
    f = rng.normal(0, 1e5, m * n)
    f[mask == 1] = 0.0
    A = sp.lil_matrix((m * n, m * n))
    b = f.copy()
    for k in range(m * n):
        if mask[k]:
            A[k, k] = 1.0
            b[k] = phi_bc[k]
        else:
            A[k, k] = -4.0 / h**2
            for q in (k - 1, k + 1, k - m, k + m):
                A[k, q] = 1.0 / h**2
    ref = spla.spsolve(A.tocsr(), b)
    for precision in ("mixed", "fp64"):
        mg = MultigridSolver(mask, m, n, h, precision=precision)
        phi, (cycles, rel) = mg.solve(torch.as_tensor(phi_bc.copy(), device=DEV), torch.as_tensor(f, device=DEV),
                                      tol=1e-10, max_cycles=120)
        assert rel < 1e-10, (precision, cycles, rel)
        np.testing.assert_allclose(phi.cpu().numpy(), ref, rtol=0, atol=1e-8 * np.abs(ref).max(), err_msg=precision)


@pytest.mark.parametrize("n", [257, 513])
def test_coarse_solve_in_fp32_or_fp64(n):
    """The mixed V-cycle's direct solve of its first level of at most 33^2
    nodes runs in FP64 by default and in FP32 on request (coarse_fp32): both
    reach the same tolerance on the manufactured problem, the FP32 one in at
    most one more cycle, and agree with the exact discrete solution."""
    h, f, exact = manufactured(n)
    mask = edge_mask(n)
    f[mask == 1] = 0.0
    ft = torch.as_tensor(f, device=DEV)
    res = {}
    for c32 in (False, True):
        mg = MultigridSolver(mask, n, n, h, precision="mixed", coarse_fp32=c32)
        phi = torch.zeros(n * n, dtype=torch.float64, device=DEV)
        phi, (cycles, rel) = mg.solve(phi, ft, tol=1e-11, max_cycles=40)
        assert rel < 1e-11, (c32, cycles, rel)
        np.testing.assert_allclose(phi.cpu().numpy(), exact, rtol=0, atol=1e-9 * np.abs(exact).max())
        res[c32] = cycles
    assert res[True] <= res[False] + 1, res
