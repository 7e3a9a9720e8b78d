"""The oracle's restatement of the reference's sine-transform Poisson solve
(src/FFT.py:10-64) on the CPU: it reproduces the exact discrete eigenmode
solution and agrees with a direct sparse solve of the 5-point system with
Dirichlet edge values."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import oracle as O


def direct(f, g, h):
    n, m = f.shape
    size = n * m
    A = sp.lil_matrix((size, size))
    b = f.reshape(-1).copy()
    for j in range(n):
        for i in range(m):
            k = j * m + i
            if i in (0, m - 1) or j in (0, n - 1):
                A[k, k] = 1.0
                b[k] = g[j, i]
            else:
                A[k, k] = -4.0 / h**2
                for q in (k - 1, k + 1, k - m, k + m):
                    A[k, q] = 1.0 / h**2
    return spla.spsolve(A.tocsr(), b).reshape(n, m)


def test_eigenmode_is_exact():
    n = 33
    h = 1.0 / (n - 1)
    x = np.linspace(0, 1, n)
    X, Y = np.meshgrid(x, x)
    f = -np.sin(np.pi * X) * np.sin(np.pi * Y)
    exact = np.sin(np.pi * X) * np.sin(np.pi * Y) / ((8 / h**2) * np.sin(np.pi * h / 2) ** 2)
    phi = O.poisson_fft_dirichlet(f, np.zeros_like(f), h)
    np.testing.assert_allclose(phi, exact, rtol=0, atol=1e-13 * np.abs(exact).max())


def test_edge_values_against_direct_solve():
    rng = np.random.default_rng(7)
    n, m, h = 17, 25, 0.1
    f = rng.normal(size=(n, m))
    g = rng.normal(size=(n, m)) * 10
    phi = O.poisson_fft_dirichlet(f, g, h)
    np.testing.assert_allclose(phi, direct(f, g, h), rtol=0, atol=1e-10 * np.abs(phi).max())
