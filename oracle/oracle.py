"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker.  It wraps

* ``libpic_oracle.so`` -- the C restatement in pic_oracle.c (FP64 reference
  arithmetic and the build's FP32 arithmetic), and
* ``_ref/libpicref.so`` -- the reference's own RawKernel sources compiled by
  ref_build.py (present only where it was built from the reference tree).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libpic_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpicref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build_oracle(force: bool = False) -> str:
    """Compile pic_oracle.c (no contraction, so FP32 op order is exact)."""
    src = os.path.join(HERE, "pic_oracle.c")
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(
            ["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", ORACLE_SO, src, "-lm"],
            check=True,
        )
    return ORACLE_SO


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_oracle())
        L = _lib
        L.or_deposit_f64.argtypes = [_dp, _dp, _dp, C.c_long, C.c_double, C.c_double, C.c_double, C.c_int,
                                     C.c_int, C.c_int]
        L.or_update_E_f64.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double]
        L.or_update_V_f64.argtypes = [_dp, _dp, _dp, _dp, C.c_long, _dp, _dp, C.c_double, C.c_double,
                                      C.c_double, C.c_int, C.c_int, C.c_int]
        L.or_update_R_f64.argtypes = [_dp, _dp, _dp, _dp, C.c_long, C.c_double]
        L.or_absorb_f64.argtypes = [_dp, _dp, C.c_long, C.c_double, C.c_double]
        L.or_absorb_f64.restype = C.c_long
        L.or_residual_f64.argtypes = [_dp, _dp, _bp, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double]
        L.or_residual_f64.restype = C.c_double
        L.or_update_E_f32.argtypes = [_dp, _fp, _fp, C.c_int, C.c_int, C.c_double, C.c_double]
        L.or_deposit_f32.argtypes = [_dp, C.c_void_p, _fp, _fp, C.c_long, C.c_float, C.c_int, C.c_int]
        L.or_kick_f32.argtypes = [_fp, _fp, _fp, _fp, C.c_long, _fp, _fp, C.c_float, C.c_int, C.c_int]
        L.or_drift_absorb_f32.argtypes = [_fp, _fp, _fp, _fp, C.c_long, C.c_float, C.c_float, C.c_int, C.c_int]
        L.or_drift_absorb_f32.restype = C.c_long
        L.or_hits_electrode.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, _up, _up]
        L.or_hits_electrode.restype = C.c_int
        L.or_drift_absorb_electrodes_f32.argtypes = [_fp, _fp, _fp, _fp, C.c_long, C.c_float, C.c_float, C.c_int,
                                                     C.c_int, _up, _up, C.POINTER(C.c_long)]
        L.or_drift_absorb_electrodes_f32.restype = C.c_long
        L.or_drift_rz_absorb_f32.argtypes = [_fp, _fp, _fp, _fp, _fp, C.c_long, C.c_float, C.c_float, C.c_int,
                                             C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_long)]
        L.or_drift_rz_absorb_f32.restype = C.c_long
        L.or_sort_keys.argtypes = [_fp, _fp, C.c_long, C.c_int, C.c_int, C.c_int, _up]
        L.or_counting_sort.argtypes = [_up, C.c_long, C.c_uint32, _up]
        L.or_philox4x32_10.argtypes = [_up, _up, _up]
        L.or_mcc_candidates.argtypes = [C.c_void_p, C.c_long, C.c_uint32, C.c_uint32, C.c_uint32, _bp]
        L.or_mcc_collide.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                     C.c_void_p, C.c_void_p]
        L.or_mcc_collide.restype = C.c_int
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference's kernels compiled for the CPU (oracle/_ref/libpicref.so)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_SO} not built (python oracle/ref_build.py)")
        _ref = C.CDLL(REF_SO)
        R = _ref
        R.ref_set_parallel.argtypes = [C.c_int, C.c_int]
        R.ref_max_threads.restype = C.c_int
        R.ref_update_density.argtypes = [_dp, _dp, _ip, _dp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                         C.c_int]
        R.ref_update_E.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double]
        R.ref_update_V.argtypes = [_dp, _dp, C.c_void_p, C.c_void_p, _ip, _dp, _dp, C.c_double, C.c_double,
                                   C.c_double, C.c_int, C.c_int, C.c_int]
        R.ref_update_R.argtypes = [_dp, _dp, _dp, C.c_double, C.c_int]
        R.ref_update_axis.argtypes = [_dp, _dp, C.c_int]
        R.ref_sort_scatter.argtypes = [_ip, _ip, _ip, _ip, _ip, C.c_int]
        R.ref_gauss_seidel.argtypes = [_dp, _dp, _ip, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
        R.ref_residual.argtypes = [_dp, _dp, _dp, _ip, C.c_double, C.c_int, C.c_int]
        R.ref_restrict.argtypes = [_dp, _dp, _ip, C.c_int, C.c_int]
        R.ref_prolong.argtypes = [_dp, _dp, _ip, C.c_int, C.c_int]
        R.ref_coarsen_bc_mask.argtypes = [_ip, _ip, C.c_int, C.c_int, C.c_int, C.c_int]
        R.ref_speeds_energies.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _dp, _dp, _ip, _dp, C.c_int]
        R.ref_interp_cross_sections.argtypes = [_dp, _dp, _dp, _bp, _dp, C.c_int, C.c_int]
        R.ref_mg_create.argtypes = [_ip, C.c_int, C.c_double, C.c_int, C.c_double]
        R.ref_mg_create.restype = C.c_void_p
        R.ref_mg_destroy.argtypes = [C.c_void_p]
        R.ref_mg_solve.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_double)]
        R.ref_mg_solve.restype = C.c_int
        R.ref_step.argtypes = [C.c_void_p]
    return _ref


# ---------------------------------------------------------------------------
# numpy-level helpers
# ---------------------------------------------------------------------------

def philox4x32_10(ctr, key) -> np.ndarray:
    out = np.zeros(4, np.uint32)
    lib().or_philox4x32_10(np.ascontiguousarray(ctr, np.uint32), np.ascontiguousarray(key, np.uint32), out)
    return out


def deposit_f64(x, y, charge, dx, dy, m, n, rho=None, floorf_quirk=True):
    rho = np.zeros(m * n) if rho is None else rho
    lib().or_deposit_f64(rho, np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64), len(x),
                         charge, dx, dy, m, n, int(floorf_quirk))
    return rho


def update_E_f64(phi, m, n, dx, dy):
    ex, ey = np.zeros(m * n), np.zeros(m * n)
    lib().or_update_E_f64(np.ascontiguousarray(phi, np.float64), ex, ey, m, n, dx, dy)
    return ex, ey


def update_E_f32(phi, m, n, dx, dy):
    ex, ey = np.zeros(m * n, np.float32), np.zeros(m * n, np.float32)
    lib().or_update_E_f32(np.ascontiguousarray(phi, np.float64), ex, ey, m, n, dx, dy)
    return ex, ey


def deposit_f32(gx, gy, scale, m, n, rho=None, abs_sum=None):
    """Exact (FP64) sum of the FP32 per-particle contributions; returns (rho, abs_sum)."""
    rho = np.zeros(m * n) if rho is None else rho
    abs_sum = np.zeros(m * n) if abs_sum is None else abs_sum
    lib().or_deposit_f32(rho, abs_sum.ctypes.data, np.ascontiguousarray(gx, np.float32),
                         np.ascontiguousarray(gy, np.float32), len(gx), np.float32(scale), m, n)
    return rho, abs_sum


def deposit_counts(gx, gy, m, n):
    """Number of particles contributing to each node (CIC: the four nodes around each live particle)."""
    gx = np.asarray(gx, np.float32)
    gy = np.asarray(gy, np.float32)
    live = ~np.isnan(gx)
    cx = np.minimum(np.maximum(gx[live], 0), np.float32(m - 1))
    cy = np.minimum(np.maximum(gy[live], 0), np.float32(n - 1))
    i0 = np.floor(cx).astype(np.int64)
    j0 = np.floor(cy).astype(np.int64)
    i1 = np.minimum(i0 + 1, m - 1)
    j1 = np.minimum(j0 + 1, n - 1)
    cnt = np.zeros(m * n, np.int64)
    for a, b in ((i0, j0), (i1, j0), (i0, j1), (i1, j1)):
        np.add.at(cnt, b * m + a, 1)
    return cnt


def kick_f32(gx, gy, vx, vy, ex, ey, kq, m, n):
    lib().or_kick_f32(gx, gy, vx, vy, len(gx), ex, ey, np.float32(kq), m, n)


def drift_absorb_f32(gx, gy, vx, vy, dtdx, dtdy, m, n) -> int:
    return int(lib().or_drift_absorb_f32(gx, gy, vx, vy, len(gx), np.float32(dtdx), np.float32(dtdy), m, n))


def electrode_bits(mask, m, n):
    """Edge bit arrays (vertical, horizontal) of the internal electrodes of a
    node mask: grid-line segments between two Dirichlet nodes, at least one of
    them internal (an electrode that reaches the domain boundary keeps its end
    segment); segments on the boundary lines themselves are not included."""
    mk = np.asarray(mask).reshape(n, m).astype(bool)
    inner = np.zeros_like(mk)
    inner[1:-1, 1:-1] = mk[1:-1, 1:-1]
    vb = np.zeros((m * (n - 1) + 31) // 32, np.uint32)
    hb = np.zeros(((m - 1) * n + 31) // 32, np.uint32)

    def end(j, i, boundary_ok):
        return inner[j, i] or (boundary_ok and mk[j, i])

    for X in range(1, m - 1):
        for j in range(n - 1):
            a, b = end(j, X, j == 0), end(j + 1, X, j + 1 == n - 1)
            if a and b and (inner[j, X] or inner[j + 1, X]):
                k = X * (n - 1) + j
                vb[k >> 5] |= np.uint32(1 << (k & 31))
    for Y in range(1, n - 1):
        for i in range(m - 1):
            a, b = end(Y, i, i == 0), end(Y, i + 1, i + 1 == m - 1)
            if a and b and (inner[Y, i] or inner[Y, i + 1]):
                k = Y * (m - 1) + i
                hb[k >> 5] |= np.uint32(1 << (k & 31))
    return vb, hb


def hits_electrode(x0, y0, x1, y1, m, n, vb, hb) -> bool:
    return bool(lib().or_hits_electrode(np.float32(x0), np.float32(y0), np.float32(x1), np.float32(y1), m, n, vb, hb))


def drift_absorb_electrodes_f32(gx, gy, vx, vy, dtdx, dtdy, m, n, vb, hb):
    """(wall-absorbed, electrode-collected) counts; gx, gy updated in place."""
    c = C.c_long()
    a = lib().or_drift_absorb_electrodes_f32(gx, gy, vx, vy, len(gx), np.float32(dtdx), np.float32(dtdy), m, n, vb,
                                             hb, C.byref(c))
    return int(a), int(c.value)


def drift_rz_absorb_f32(gx, gy, vx, vy, vz, dtdx, dtdy, m, n, vb=None, hb=None):
    """r-z drift (pic_oracle.c or_drift_rz_absorb_f32) in place; (wall, electrode) counts."""
    c = C.c_long()
    a = lib().or_drift_rz_absorb_f32(gx, gy, vx, vy, vz, len(gx), np.float32(dtdx), np.float32(dtdy), m, n,
                                     None if vb is None else vb.ctypes.data, None if hb is None else hb.ctypes.data,
                                     C.byref(c))
    return int(a), int(c.value)


# ---- r-z operator (FP64, numpy / scipy) --------------------------------------------

def rz_row_volume(j, n, dy):
    """Node volume of row j of an r-z grid per dx*dy (m): the integral of 2 pi r
    times the row's linear weighting function (2 pi r_j inside, pi dy/3 on the
    axis, pi (r_top - dy/3) on the outer row)."""
    j = np.asarray(j)
    r = 2.0 * np.pi * j * dy
    r = np.where(j == 0, np.pi * dy / 3.0, r)
    return np.where(j == n - 1, np.pi * (j * dy - dy / 3.0), r)


def rz_rows(n, dx, dy):
    """(wN, wS, diag) per row of the build's r-z operator: conservative
    differences of (1/r) d/dr (r dphi/dr) + d2phi/dz2, with the axis limit
    2 d2phi/dr2 -> 4 (phi_1 - phi_0)/dy^2 on row 0."""
    cx, cy = 1.0 / dx ** 2, 1.0 / dy ** 2
    j = np.arange(n, dtype=np.float64)
    with np.errstate(divide="ignore"):
        wn = np.where(j == 0, 4.0 * cy, cy * (1.0 + 0.5 / j))
        ws = np.where(j == 0, 0.0, cy * (1.0 - 0.5 / j))
    return wn, ws, -(2.0 * cx + wn + ws)


def rz_free(mask, m, n):
    """Free nodes of an r-z grid: not masked, not on the x edges or the outer row (the axis row is free)."""
    mk = np.asarray(mask).reshape(n, m).astype(bool).copy()
    mk[:, 0] = mk[:, -1] = mk[-1, :] = True
    return ~mk


def rz_apply(phi, m, n, dx, dy):
    """The r-z operator applied at every node with an in-grid stencil (rows
    0..n-2, columns 1..m-2); zero elsewhere."""
    p = np.asarray(phi, np.float64).reshape(n, m)
    wn, ws, dg = rz_rows(n, dx, dy)
    out = np.zeros_like(p)
    c = p[:-1, 1:-1]
    south = np.vstack([np.zeros((1, m - 2)), p[:-2, 1:-1]])
    out[:-1, 1:-1] = ((p[:-1, :-2] + p[:-1, 2:]) / dx ** 2 + wn[:-1, None] * p[1:, 1:-1] + ws[:-1, None] * south
                      + dg[:-1, None] * c)
    return out.reshape(-1)


def rz_residual(phi, f, mask, m, n, dx, dy):
    """||f - L phi|| / ||f|| over the free nodes (the build's convergence measure)."""
    free = rz_free(mask, m, n).reshape(-1)
    r = (np.asarray(f, np.float64) - rz_apply(phi, m, n, dx, dy))[free]
    fn = np.linalg.norm(np.asarray(f, np.float64)[free])
    return float(np.linalg.norm(r) / (fn if fn > 0 else 1.0))


def rz_solve(f, phi_bc, mask, m, n, dx, dy):
    """Direct sparse solve of L phi = f on the free nodes of an r-z grid,
    phi = phi_bc elsewhere."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    free = rz_free(mask, m, n).reshape(-1)
    wn, ws, dg = rz_rows(n, dx, dy)
    idx = np.full(m * n, -1)
    fi = np.flatnonzero(free)
    idx[fi] = np.arange(fi.size)
    phi = np.asarray(phi_bc, np.float64).reshape(-1).copy()
    rows, cols, vals = [], [], []
    rhs = np.asarray(f, np.float64).reshape(-1)[fi].copy()
    for a, k in enumerate(fi):
        j, i = divmod(int(k), m)
        rows.append(a); cols.append(a); vals.append(dg[j])
        nb = [(k - 1, 1.0 / dx ** 2), (k + 1, 1.0 / dx ** 2), (k + m, wn[j])]
        if j > 0:
            nb.append((k - m, ws[j]))
        for q, w in nb:
            if idx[q] >= 0:
                rows.append(a); cols.append(int(idx[q])); vals.append(w)
            else:
                rhs[a] -= w * phi[q]
    A = sp.csr_matrix((vals, (rows, cols)), shape=(fi.size, fi.size))
    phi[fi] = spl.spsolve(A, rhs)
    return phi


def ref_cylindrical_laplacian(m, n, dz, dr):
    """Dense restatement of the reference's Laplacian_cylindrical_csr
    (src/Solvers.py:100-166) as its source reads: m nodes in z (fast index), n
    in r; main diagonal -4; z neighbours 1 except across rows; lower r
    neighbour of row r 1 - 1/(2 r/dr); upper r neighbour of row r set from the
    next row's index, 1 + 1/(2 (r+1)/dr), and left 0 for row n-2; axis rows
    -4 with z neighbours and 2 towards row 1."""
    size = m * n
    A = np.zeros((size, size))
    for k in range(size):
        A[k, k] = -4.0
        if (k + 1) % m != 0 and k + 1 < size:
            A[k, k + 1] = 1.0
            A[k + 1, k] = 1.0
    for i, r in enumerate(range(1, n)):
        lo = i * m
        for k in range(lo, lo + m):
            if i + 1 < n - 1:
                A[k, k + m] = 1.0 + 1.0 / (2 * r / dr)
            A[k + m, k] = 1.0 - 1.0 / (2 * r / dr)
    for k in range(m):
        A[k, k + m] = 2.0
    return A


def poisson_fft_dirichlet(f, g, dx):
    """The reference's poisson_fft_dirichlet (src/FFT.py:10-64) restated in
    numpy/scipy: lap(phi) = f on a square-celled grid, phi = g on the four
    edges.  The edge values enter through f - lap(phi_g) (phi_g = g on the
    edges, 0 inside), the interior is solved with orthonormal DST-I in both
    directions and the 5-point eigenvalues.  f, g: 2D arrays [rows, columns]."""
    from scipy.fft import dstn, idstn

    f = np.asarray(f, np.float64)
    g = np.asarray(g, np.float64)
    phi_g = np.zeros_like(f)
    phi_g[0, :], phi_g[-1, :], phi_g[:, 0], phi_g[:, -1] = g[0, :], g[-1, :], g[:, 0], g[:, -1]
    lap = np.zeros_like(f)
    lap[1:-1, 1:-1] = (-4 * phi_g[1:-1, 1:-1] + phi_g[2:, 1:-1] + phi_g[:-2, 1:-1] + phi_g[1:-1, 2:]
                       + phi_g[1:-1, :-2]) / dx ** 2
    f_hat = dstn((f - lap)[1:-1, 1:-1], type=1, norm="ortho")
    nx, ny = f_hat.shape
    i = np.arange(1, nx + 1).reshape(-1, 1)
    j = np.arange(1, ny + 1).reshape(1, -1)
    denom = (2 * (np.cos(np.pi * i / (nx + 1)) - 1) + 2 * (np.cos(np.pi * j / (ny + 1)) - 1)) / dx ** 2
    phi = phi_g.copy()
    phi[1:-1, 1:-1] += idstn(f_hat / denom, type=1, norm="ortho")
    return phi


def residual_f64(phi, f, dirichlet, m, n, dx, dy, want_r=False):
    r = np.zeros(m * n) if want_r else None
    s = lib().or_residual_f64(np.ascontiguousarray(phi, np.float64), np.ascontiguousarray(f, np.float64),
                              np.ascontiguousarray(dirichlet, np.uint8), None if r is None else r.ctypes.data,
                              m, n, dx, dy)
    return (s, r) if want_r else s


def sort_keys(gx, gy, m, n, ts):
    keys = np.zeros(len(gx), np.uint32)
    lib().or_sort_keys(np.ascontiguousarray(gx, np.float32), np.ascontiguousarray(gy, np.float32), len(gx), m, n,
                       ts, keys)
    return keys


def counting_sort(keys, nkeys):
    perm = np.zeros(len(keys), np.uint32)
    lib().or_counting_sort(np.ascontiguousarray(keys, np.uint32), len(keys), nkeys, perm)
    return perm


class OrMccSpecies(C.Structure):
    _fields_ = [
        ("nproc", C.c_int),
        ("type", C.c_int * 4),
        ("threshold", C.c_float * 4),
        ("sigma", C.c_void_p * 4),
        ("ne", C.c_int),
        ("energy", C.c_void_p),
        ("inv_log_ratio", C.c_float),
        ("log_e0", C.c_float),
        ("gas_density", C.c_float),
        ("half_m_over_q", C.c_float),
        ("mass_ratio2", C.c_float),
        ("gas_vth", C.c_float),
        ("nu_max", C.c_float),
        ("inv_log1m_p", C.c_double),
        ("species", C.c_uint32),
        ("seg", C.c_uint32),
    ]


# ---------------------------------------------------------------------------
# numpy restatements of the reference's multigrid and MCC kernels, operation
# for operation (pinned bit-exact against tests/golden/*.npz)
# ---------------------------------------------------------------------------

def rb_sor_color(phi, rho, bc_mask, h2, omega, nx, ny, is_red):
    """One colour of gauss_seidel_red_black (src/multigrid.py:26-47), in place."""
    P = phi.reshape(ny, nx)
    Rr = rho.reshape(ny, nx)
    B = bc_mask.reshape(ny, nx)
    j, i = np.mgrid[0:ny, 0:nx]
    sel = (i > 0) & (i < nx - 1) & (j > 0) & (j < ny - 1) & (B == 0) & ((i + j) % 2 == is_red)
    jj, ii = j[sel], i[sel]
    upd = 0.25 * (P[jj + 1, ii] + P[jj - 1, ii] + P[jj, ii + 1] + P[jj, ii - 1] - h2 * Rr[jj, ii])
    P[jj, ii] = (1.0 - omega) * P[jj, ii] + omega * upd
    return phi


def residual_ref(phi, rho, bc_mask, inv_h2, nx, ny):
    """residual_kernel (src/multigrid.py:64-79): 0 on edges and mask == 1."""
    P = phi.reshape(ny, nx)
    out = np.zeros((ny, nx))
    B = bc_mask.reshape(ny, nx)
    core = (B[1:-1, 1:-1] == 0)
    lap = (P[:-2, 1:-1] + P[2:, 1:-1] + P[1:-1, :-2] + P[1:-1, 2:] - 4.0 * P[1:-1, 1:-1]) * inv_h2
    inner = rho.reshape(ny, nx)[1:-1, 1:-1] - lap
    out[1:-1, 1:-1] = np.where(core, inner, 0.0)
    return out.reshape(-1)


def restrict_ref(fine, nx, ny):
    """restriction_kernel (src/multigrid.py:94-132): full weighting renormalised by the in-bounds weights."""
    nxc, nyc = (nx + 1) // 2, (ny + 1) // 2
    F = fine.reshape(ny, nx)
    out = np.zeros((nyc, nxc))
    for i in range(nyc):
        for j in range(nxc):
            s = 0.0
            w = 0.0
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    a, b = 2 * i + di, 2 * j + dj
                    if 0 <= a < ny and 0 <= b < nx:
                        wt = 0.25 if (di == 0 and dj == 0) else (0.125 if (di == 0 or dj == 0) else 0.0625)
                        s += wt * F[a, b]
                        w += wt
            out[i, j] = s / w if w > 0.0 else 0.0
    return out.reshape(-1)


def prolong_ref(fine, coarse, mask_fine, nxc, nyc):
    """prolong_kernel (src/multigrid.py:148-194): adds the bilinear coarse value where mask_fine != 0."""
    nxf = 2 * (nxc - 1) + 1
    nyf = 2 * (nyc - 1) + 1
    Fo = fine.reshape(nyf, nxf)
    Cc = coarse.reshape(nyc, nxc)
    M = mask_fine.reshape(nyf, nxf)
    for i in range(nyf):
        for j in range(nxf):
            if M[i, j] == 0:
                continue
            ic, jc = i // 2, j // 2
            io, jo = i % 2, j % 2
            v = 0.0
            if not io and not jo:
                v = Cc[ic, jc]
            elif io and not jo:
                if ic + 1 < nyc:
                    v = 0.5 * (Cc[ic, jc] + Cc[ic + 1, jc])
            elif not io and jo:
                if jc + 1 < nxc:
                    v = 0.5 * (Cc[ic, jc] + Cc[ic, jc + 1])
            else:
                if ic + 1 < nyc and jc + 1 < nxc:
                    v = 0.25 * (Cc[ic, jc] + Cc[ic + 1, jc] + Cc[ic, jc + 1] + Cc[ic + 1, jc + 1])
            Fo[i, j] += v
    return fine


def coarsen_mask_ref(fine, nxf, nyf, nxc, nyc):
    """coarsen_bc_mask (src/multigrid.py:248-271): 1 iff all 3x3 fine neighbours are in bounds and != 0."""
    F = fine.reshape(nyf, nxf)
    out = np.zeros((nyc, nxc), np.int32)
    for i in range(nyc):
        for j in range(nxc):
            ok = 1
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    a, b = 2 * i + di, 2 * j + dj
                    if not (0 <= a < nyf and 0 <= b < nxf) or F[a, b] == 0:
                        ok = 0
            out[i, j] = ok
    return out.reshape(-1)


def speeds_energies_ref(V, part_type, m_type):
    """compute_speeds_and_energies as called at src/MCC.py:118-121 on an (N,3) V:
    the kernel reads V.flat[i], V.flat[3+i], V.flat[6+i] and takes sqrtf of a double."""
    flat = np.ascontiguousarray(V).reshape(-1)
    n = len(part_type)
    vx, vy, vz = flat[0:n], flat[3:3 + n], flat[6:6 + n]
    s = vx * vx + vy * vy + vz * vz
    speed = np.sqrt(s.astype(np.float32)).astype(np.float64)
    energy = 0.5 * m_type[part_type] * speed * speed
    return speed, energy


def interp_ref(e, xs_e, xs_s, mask):
    """interpolate_cross_sections (src/MCC.py:43-81)."""
    out = np.zeros(len(e))
    for i, E in enumerate(e):
        if not mask[i]:
            out[i] = 0.0
        elif E <= xs_e[0]:
            out[i] = xs_s[0]
        elif E >= xs_e[-1]:
            out[i] = xs_s[-1]
        else:
            j = int(np.searchsorted(xs_e, E, side="right")) - 1
            t = (E - xs_e[j]) / (xs_e[j + 1] - xs_e[j])
            out[i] = xs_s[j] + t * (xs_s[j + 1] - xs_s[j])
    return out


def mcc_species(tables_energy, sigmas, types, thresholds, gas_density, mass, gas_mass, gas_temperature, nu_max,
                inv_log1m_p, species, seg=256):
    """An or_mcc_species for or_mcc_candidates / or_mcc_collide; returns (struct, keep-alive list)."""
    from math import log, sqrt

    qe, kb = 1.6e-19, 1.380649e-23
    E = np.ascontiguousarray(tables_energy, np.float32)
    S = OrMccSpecies()
    S.nproc = len(sigmas)
    keep = [E]
    for k, sig in enumerate(sigmas):
        a = np.ascontiguousarray(sig, np.float32)
        keep.append(a)
        S.type[k] = types[k]
        S.threshold[k] = thresholds[k]
        S.sigma[k] = a.ctypes.data
    S.ne = len(E)
    S.energy = E.ctypes.data
    S.log_e0 = np.float32(np.log(np.float32(E[0])))
    S.inv_log_ratio = np.float32((len(E) - 1) / log(float(E[-1]) / float(E[0])))
    S.gas_density = np.float32(gas_density)
    S.half_m_over_q = np.float32(0.5 * mass / qe)
    S.mass_ratio2 = np.float32(2.0 * mass / gas_mass)
    S.gas_vth = np.float32(sqrt(kb * gas_temperature / gas_mass))
    S.nu_max = np.float32(nu_max)
    S.inv_log1m_p = inv_log1m_p
    S.species = species
    S.seg = seg
    return S, keep


def mcc_candidates(S, n, step, seed):
    mark = np.zeros(n, np.uint8)
    lib().or_mcc_candidates(C.byref(S), n, step, seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, mark)
    return mark


def mcc_collide(S, idx, step, seed, v):
    """One candidate; v = [vx, vy, vz] float32 (updated).  Returns (proc, born_e, born_i)."""
    vx, vy, vz = C.c_float(v[0]), C.c_float(v[1]), C.c_float(v[2])
    be = np.zeros(3, np.float32)
    bi = np.zeros(3, np.float32)
    proc = lib().or_mcc_collide(C.byref(S), idx, step, seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, C.byref(vx),
                                C.byref(vy), C.byref(vz), be.ctypes.data, bi.ctypes.data)
    v[0], v[1], v[2] = vx.value, vy.value, vz.value
    return proc, be, bi
