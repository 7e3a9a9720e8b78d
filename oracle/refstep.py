"""The reference's time step on the host cores (test infrastructure / CPU baseline).

Drives oracle/_ref/libpicref.so -- the reference's own RawKernel sources
compiled for the CPU -- through ref_step (oracle/ref_driver.cpp), i.e.
SimulationManager._step (src/simulation.py:640-660) on the reference's AoS
FP64 arrays with OpenMP over kernel blocks.  The multigrid uses the
reference's parameters (5 levels, omega 1.9, 5 smoothing and 20 coarsest
sweeps, 50 cycles: src/Solvers.py:260, src/multigrid.py:445) with the mask and
scaling fixes it needs to run.  MCC runs the part of
MCC.null_collision_method before its early return (elastic table).
Only bench.py's CPU-baseline leg and the tests use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import oracle as O

QE, ME, AMU, EPS0 = 1.6e-19, 9.10938356e-31, 1.66e-27, 8.85418782e-12


class RefState(C.Structure):
    _fields_ = [
        ("m", C.c_int), ("n", C.c_int), ("last_alive", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double), ("np2c", C.c_double), ("eps0", C.c_double),
        ("R", C.c_void_p), ("R_old", C.c_void_p), ("V", C.c_void_p), ("part_type", C.c_void_p),
        ("q_type", C.c_void_p), ("m_type", C.c_void_p), ("m_type_inv", C.c_void_p),
        ("rho", C.c_void_p), ("b", C.c_void_p), ("phi", C.c_void_p), ("E", C.c_void_p),
        ("bc_idx", C.c_void_p), ("bc_val", C.c_void_p), ("n_bc", C.c_int),
        ("mg", C.c_void_p), ("tol", C.c_double),
        ("smooth_iter", C.c_int), ("solve_iter", C.c_int), ("max_cycles", C.c_int),
        ("do_mcc", C.c_int), ("gas_density", C.c_double), ("xs_energy", C.c_void_p), ("xs_sigma", C.c_void_p),
        ("xs_len", C.c_int), ("mcc_species", C.c_int),
        ("speeds", C.c_void_p), ("energies", C.c_void_p), ("sigma", C.c_void_p), ("rand_buf", C.c_void_p),
        ("mcc_mask", C.c_void_p), ("rng", C.c_ulonglong),
        ("last_cycles", C.c_int), ("last_rel", C.c_double), ("collided", C.c_longlong),
    ]


class ReferenceCPU:
    """One reference simulation: electrons (type 1) and ions (type 2) in metres, FP64.

    e, i: (x, y, vx, vy, vz) arrays, positions in grid units (converted to metres).
    """

    def __init__(self, nodes, dx, dt, e, i, np2c, ion_mass, left_V=0.0, tol=1e-8, mcc_table=None, gas_density=0.0,
                 threads=0, levels=5, omega=1.9, smooth_iter=5, solve_iter=20, max_cycles=50):
        L = O.ref()
        L.ref_set_parallel(1, int(threads))
        self.threads = L.ref_max_threads()
        m = n = int(nodes)
        ne, ni = len(e[0]), len(i[0])
        N = ne + ni
        self.N = N
        self.R = np.empty((N, 2))
        self.R[:ne, 0], self.R[:ne, 1] = e[0].astype(np.float64) * dx, e[1].astype(np.float64) * dx
        self.R[ne:, 0], self.R[ne:, 1] = i[0].astype(np.float64) * dx, i[1].astype(np.float64) * dx
        self.V = np.empty((N, 3))
        for k in range(3):
            self.V[:ne, k] = e[2 + k]
            self.V[ne:, k] = i[2 + k]
        self.R_old = np.zeros_like(self.R)
        self.part_type = np.concatenate([np.full(ne, 1, np.int32), np.full(ni, 2, np.int32)])
        self.q_type = np.array([0.0, -QE, QE])
        self.m_type = np.array([0.0, ME, ion_mass])
        self.m_type_inv = np.array([0.0, 1 / ME, 1 / ion_mass])
        G = m * n
        self.rho, self.b, self.phi, self.E = np.zeros(G), np.zeros(G), np.zeros(G), np.zeros(2 * G)
        idx = np.arange(G).reshape(n, m)
        edges = np.unique(np.concatenate([idx[0, :], idx[-1, :], idx[:, 0], idx[:, -1]]))
        vals = np.where(np.isin(edges, idx[1:-1, 0]), left_V, 0.0)
        self.bc_idx = edges.astype(np.int32)
        self.bc_val = vals.astype(np.float64)
        self.phi[self.bc_idx] = self.bc_val
        bc_lookup = np.zeros(G, np.int32)
        bc_lookup[self.bc_idx] = 1
        self.mg = L.ref_mg_create(bc_lookup, m, dx, levels, omega)
        self.speeds, self.energies, self.sigma = np.zeros(N), np.zeros(N), np.zeros(N)
        self.mcc_mask = np.zeros(N, np.uint8)
        s = RefState()
        s.m, s.n, s.last_alive = m, n, N
        s.dx, s.dy, s.dt, s.np2c, s.eps0 = dx, dx, dt, np2c, EPS0
        for name in ("R", "R_old", "V", "part_type", "q_type", "m_type", "m_type_inv", "rho", "b", "phi", "E",
                     "bc_idx", "bc_val", "speeds", "energies", "sigma", "mcc_mask"):
            setattr(s, name, getattr(self, name).ctypes.data)
        s.n_bc = len(self.bc_idx)
        s.mg = self.mg
        s.tol, s.smooth_iter, s.solve_iter, s.max_cycles = tol, smooth_iter, solve_iter, max_cycles
        if mcc_table is not None:
            self.xs_e = np.ascontiguousarray(mcc_table[0], np.float64)
            self.xs_s = np.ascontiguousarray(mcc_table[1], np.float64)
            s.do_mcc, s.gas_density = 1, gas_density
            s.xs_energy, s.xs_sigma, s.xs_len = self.xs_e.ctypes.data, self.xs_s.ctypes.data, len(self.xs_e)
            s.mcc_species = 1
        s.rng = 12345
        self.state = s

    def step(self):
        O.ref().ref_step(C.byref(self.state))
        return self.state.last_cycles, self.state.last_rel

    def close(self):
        if self.mg:
            O.ref().ref_mg_destroy(self.mg)
            self.mg = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def time_steps(ref: ReferenceCPU, steps: int, warmup: int = 1):
    for _ in range(warmup):
        ref.step()
    t0 = time.perf_counter()
    cycles = []
    for _ in range(steps):
        c, _ = ref.step()
        cycles.append(c)
    dt = time.perf_counter() - t0
    return dt, cycles


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_cores() -> int:
    return os.cpu_count() or 1
