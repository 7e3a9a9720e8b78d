"""The band-LU inverse behind the multigrid's direct coarse solve, on the CPU.

pic_b200/csrc/band_inverse.h is built with g++ into a small shared library
and checked against numpy.linalg.inv on the level operators the solver
inverts: the Cartesian 5-point operator on a grid's free nodes (edges and
internal electrodes Dirichlet) and the r-z operator (axis row free, rows
weighted 1 +- 1/2j), at the sizes of a 33^2 coarse level and of smaller and
rectangular ones.  A singular matrix is reported, not inverted.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("bi") / "libbi.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(ROOT, "pic_b200", "csrc"),
                    os.path.join(ROOT, "tests", "band_inverse_harness.cpp"), "-o", str(out)], check=True,
                   capture_output=True)
    lib = C.CDLL(str(out))
    lib.band_inverse_c.argtypes = [C.c_void_p, C.c_int, C.c_int]
    return lib


def level_operator(nx, ny, mask, hx, hy, rz):
    """The dense operator on the free nodes, as pic_mg_create builds it; returns (A, bandwidth)."""
    where = -np.ones(nx * ny, int)
    idx = []
    for j in range(0 if rz else 1, ny - 1):
        for i in range(1, nx - 1):
            if not mask[j * nx + i]:
                where[j * nx + i] = len(idx)
                idx.append(j * nx + i)
    n = len(idx)
    A = np.zeros((n, n))
    cx, cy = 1 / hx**2, 1 / hy**2
    bw = 0
    for a, k in enumerate(idx):
        j = k // nx
        if rz:
            wn = 4 * cy if j == 0 else cy * (1 + 0.5 / j)
            ws = 0.0 if j == 0 else cy * (1 - 0.5 / j)
        else:
            wn = ws = cy
        A[a, a] = -(2 * cx + wn + ws)
        for nb, w in ((k - 1, cx), (k + 1, cx), (k - nx if j > 0 else -1, ws), (k + nx, wn)):
            if nb >= 0 and where[nb] >= 0:
                A[a, where[nb]] += w
                bw = max(bw, abs(int(where[nb]) - a))
    return A, bw


@pytest.mark.parametrize("nx,ny,rz,electrodes", [(33, 33, False, False), (33, 33, True, False), (33, 9, False, True),
                                                 (9, 33, True, True), (25, 13, False, True), (17, 17, False, False)])
def test_band_inverse_matches_numpy(lib, nx, ny, rz, electrodes):
    rng = np.random.default_rng(nx * 100 + ny)
    mask = np.zeros(nx * ny, np.uint8)
    if electrodes:
        mask[rng.integers(0, nx * ny, nx * ny // 20)] = 1
    A, bw = level_operator(nx, ny, mask, 2e-3, 3e-3, rz)
    M = np.ascontiguousarray(A.copy())
    assert lib.band_inverse_c(M.ctypes.data, M.shape[0], bw) == 0
    ref = np.linalg.inv(A)
    np.testing.assert_allclose(M, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # and it is an inverse: A A^-1 = I to FP64 round-off
    np.testing.assert_allclose(A @ M, np.eye(A.shape[0]), rtol=0, atol=1e-11)


def test_singular_matrix_is_reported(lib):
    A = np.array([[1.0, 1.0], [1.0, 1.0]])
    assert lib.band_inverse_c(np.ascontiguousarray(A).ctypes.data, 2, 1) == 1
