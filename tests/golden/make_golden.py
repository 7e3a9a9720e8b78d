"""Generate the golden vectors in this folder from the reference's own kernels.

Runs the reference's CuPy RawKernel sources, compiled for the CPU by
oracle/ref_build.py (oracle/_ref/libpicref.so), serially (deterministic
atomics) on small seeded inputs, and stores inputs and outputs as .npz files
here.  The reference itself cannot be imported in this container (no CuPy, no
GPU, case-mismatched module names), so this is how its behaviour is captured.

    python oracle/ref_build.py && python tests/golden/make_golden.py

Each fixture names the reference function it exercises.  The files are small
(tens of KB) and are committed; the -m "not gpu" tests read them to pin the
oracle, and never need /root/reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle import oracle as O  # noqa: E402

QE, ME, AMU = 1.6e-19, 9.10938356e-31, 1.66e-27


def particles(rng, n, m, nn, dx, dy):
    """Positions in metres with edge cases: exact walls, exact nodes, near-node values."""
    X, Y = dx * (m - 1), dy * (nn - 1)
    x = rng.uniform(0, X, n)
    y = rng.uniform(0, Y, n)
    x[:6] = [0.0, X, X * 0.5, dx * 3, dx * 3 * (1 - 1e-12), np.nextafter(X, 0)]
    y[:6] = [0.0, Y, dy * 2, dy * 2 * (1 + 1e-12), Y * 0.25, 0.0]
    return x, y


def gen_particle_fixtures(rng):
    m, nn, dx, dy = 17, 13, 1e-4, 1.25e-4
    n = 600
    x, y = particles(rng, n, m, nn, dx, dy)
    R = np.ascontiguousarray(np.stack([x, y], 1))
    V = np.ascontiguousarray(np.stack([rng.normal(0, 5e5, n), rng.normal(0, 5e5, n), rng.normal(0, 5e5, n)], 1))
    part_type = np.where(np.arange(n) % 3 == 0, 2, 1).astype(np.int32)
    q_type = np.array([0.0, -QE, QE])
    m_type = np.array([0.0, ME, 40 * AMU])
    m_type_inv = np.array([0.0, 1 / ME, 1 / (40 * AMU)])
    np2c = 12345.0
    lib = O.ref()
    lib.ref_set_parallel(0, 0)

    rho = np.zeros(m * nn)
    lib.ref_update_density(rho, R.ravel(), part_type, q_type, np2c, dx, dy, m, nn, n)

    phi = rng.normal(0, 10, m * nn)
    E = np.zeros(2 * m * nn)
    lib.ref_update_E(phi, E, m, nn, dx, dy)

    Vk = V.copy().ravel()
    dt = 1e-11
    lib.ref_update_V(Vk, R.ravel(), E.ctypes.data, E.ctypes.data + 8 * m * nn, part_type, q_type, m_type_inv, dt, dx,
                     dy, m, nn, n)

    Rr, Rold, Vr = R.copy().ravel(), np.zeros(2 * n), V.copy().ravel()
    Vr[1::3] -= 3e6  # push some particles through y < 0 for the axis kernel
    lib.ref_update_R(Rold, Rr, Vr, 1e-10, n)
    Ra, Va = Rr.copy(), Vr.copy()
    lib.ref_update_axis(Ra, Va, n)

    np.savez_compressed(
        os.path.join(HERE, "particles_17x13.npz"),
        m=m, n=nn, dx=dx, dy=dy, np2c=np2c, dt=dt, R=R, V=V, part_type=part_type, q_type=q_type,
        m_type=m_type, m_type_inv=m_type_inv, rho=rho, phi=phi, E=E, V_kicked=Vk.reshape(n, 3),
        V_drift_in=Vr.reshape(n, 3), R_drift=Rr.reshape(n, 2), R_old=Rold.reshape(n, 2),
        R_axis=Ra.reshape(n, 2), V_axis=Va.reshape(n, 3),
    )


def gen_multigrid_fixtures(rng):
    n = 17
    h = 1.0 / (n - 1)
    bc = np.zeros(n * n, np.int32)
    idx = np.arange(n * n).reshape(n, n)
    bc[idx[0, :]] = bc[idx[-1, :]] = bc[idx[:, 0]] = bc[idx[:, -1]] = 1
    bc[idx[5, 4:9]] = 1  # an internal electrode
    phi = rng.normal(0, 1, n * n)
    rhs = rng.normal(0, 50, n * n)
    lib = O.ref()
    lib.ref_set_parallel(0, 0)
    red = phi.copy()
    lib.ref_gauss_seidel(red, rhs, bc, h * h, 1.9, n, n, 1)
    black = red.copy()
    lib.ref_gauss_seidel(black, rhs, bc, h * h, 1.9, n, n, 0)
    res = np.full(n * n, 7.0)
    lib.ref_residual(phi, rhs, res, bc, 1.0 / (h * h), n, n)
    nc = (n + 1) // 2
    coarse = np.zeros(nc * nc)
    lib.ref_restrict(rhs, coarse, bc, n, n)
    coarse_in = rng.normal(0, 1, nc * nc)
    free = (1 - bc).astype(np.int32)
    fine = phi.copy()
    lib.ref_prolong(fine, coarse_in, free, nc, nc)
    cmask = np.zeros(nc * nc, np.int32)
    lib.ref_coarsen_bc_mask(free, cmask, n, n, nc, nc)
    np.savez_compressed(
        os.path.join(HERE, "multigrid_17.npz"), n=n, h=h, bc=bc, phi=phi, rhs=rhs, omega=1.9, gs_red=red,
        gs_black=black, residual=res, restricted=coarse, coarse_in=coarse_in, prolonged=fine, coarse_free=cmask,
    )


def gen_mcc_fixtures(rng):
    n = 300
    V = rng.normal(0, 2e6, (n, 3))
    V[:4] = 0.0
    part_type = np.where(np.arange(n) % 4 == 0, 2, 1).astype(np.int32)
    m_type = np.array([0.0, ME, 40 * AMU])
    lib = O.ref()
    lib.ref_set_parallel(0, 0)
    speeds, energies = np.zeros(n), np.zeros(n)
    # the reference passes V[0], V[1], V[2] of the (N, 3) array (src/MCC.py:120)
    base = V.ctypes.data
    lib.ref_speeds_energies(base, base + 24, base + 48, speeds, energies, part_type, m_type, n)
    # an eV table in the H.txt two-column format, and energies spanning below / inside / above it
    xs_e = np.array([0.0, 0.1, 0.5, 1.0, 1.5, 2.0, 3.0, 5.0, 9.0, 15.0, 30.0, 100.0, 1000.0])
    xs_s = 4e-19 / (1.0 + xs_e) ** 0.7
    e_ev = np.concatenate([[0.0, -1.0, 1000.0, 5000.0, 0.1, 1.0, 100.0], rng.uniform(0, 1200, n - 7)])
    mask = (np.arange(n) % 5 != 0).astype(np.uint8)
    out = np.full(n, -1.0)
    lib.ref_interp_cross_sections(e_ev, xs_e, xs_s, mask, out, len(xs_e), n)
    np.savez_compressed(
        os.path.join(HERE, "mcc.npz"), V=V, part_type=part_type, m_type=m_type, speeds=speeds, energies=energies,
        xs_e=xs_e, xs_s=xs_s, e_ev=e_ev, mcc_mask=mask, sigma=out,
    )


def gen_sort_fixture(rng):
    n, ncells = 2000, 300
    cells = rng.integers(0, ncells, n).astype(np.int32)
    # host part of sort_particles_sparse (src/Particles.py:572-586) restated in numpy
    counts = np.bincount(cells, minlength=ncells)
    active = np.nonzero(counts)[0]
    starts = np.zeros(len(active), np.int32)
    starts[1:] = np.cumsum(counts[active])[:-1]
    to_active = -np.ones(ncells, np.int32)
    to_active[active] = np.arange(len(active))
    temp = np.zeros(len(active), np.int32)
    out = np.zeros(n, np.int32)
    lib = O.ref()
    lib.ref_set_parallel(0, 0)
    lib.ref_sort_scatter(cells, to_active, starts, temp, out, n)
    np.savez_compressed(os.path.join(HERE, "sort.npz"), cells=cells, ncells=ncells, sorted_indices=out)


def main():
    rng = np.random.Generator(np.random.Philox(20261203))
    gen_particle_fixtures(rng)
    gen_multigrid_fixtures(rng)
    gen_mcc_fixtures(rng)
    gen_sort_fixture(rng)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
