"""Ensembles of independent collisionless simulations stepped as one graph.

The reference runs one simulation per process (src/simulation.py:562-567).
An ensemble here is a list of PICSimulation members with their own grids,
particle counts, tiles, sort intervals and multigrid options, stepped
together by pic_ens_step: one CUDA graph launch runs n steps of every member,
each step one persistent particle pass over all members' work items between
the members' own preparations and field solves (pic_b200/csrc/step.cu).

The ensemble workload: grid sides drawn from {129, 257, 513} nodes, particle
counts per species uniform in [1e5, 2e6], Te uniform in [1, 5] eV, left-wall
voltage uniform in [0, 200] V, seeds base + i, collisionless.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import Consts, _lib, workloads
from .simulation import PICSimulation

SIDES = (129, 257, 513)


def ensemble_workloads(count=64, seed=2026, n_range=(100_000, 2_000_000), sides=SIDES):
    """Member workloads of the ensemble (seeded)."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(count):
        side = int(rng.choice(sides))
        n_e, n_i = (int(v) for v in rng.integers(n_range[0], n_range[1] + 1, 2))
        out.append(workloads.Workload(f"member{i}", side, n_e, n_i, Te=float(rng.uniform(1.0, 5.0)),
                                      left_V=float(rng.uniform(0.0, 200.0)), steps=500, seed=seed + i))
    return out


def member_simulation(w: workloads.Workload, tile=16, sort_interval=20, coarsest_max=9, omega=1.15,
                      mg_launch="graph", use_graph=True, seed=None, push_kernel="ring") -> PICSimulation:
    """A collisionless simulation of workload w (graph-captured steps)."""
    mask, phi_bc = workloads.dirichlet(w)
    species = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=w.n_e + 64),
               dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=w.n_i + 64)]
    return PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, species, mask, phi_bc, tol=w.tol, max_cycles=50,
                         sort_interval=sort_interval, tile=tile, mcc=None, seed=w.seed if seed is None else seed,
                         use_graph=use_graph, mg_launch=mg_launch, coarsest_max=coarsest_max, omega=omega,
                         push_kernel=push_kernel)


def member_arrays(w: workloads.Workload):
    """Seeded initial particles of a member: [(x, y, vx, vy, vz) electrons, ions]."""
    rng = np.random.Generator(np.random.Philox(w.seed))
    return [workloads.species_arrays(w, "e", rng), workloads.species_arrays(w, "i", rng)]


class Ensemble:
    """Steps every member together (pic_ens_*).  Members stay owned by the
    caller, must be loaded and initialised, and must outlive the ensemble."""

    def __init__(self, members):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        self._h = C.c_void_p()
        _lib.call("pic_ens_create", arr, len(self.members), C.byref(self._h))

    def step(self, n=1):
        _lib.call("pic_ens_step", self._h, int(n), _lib.stream_ptr())

    @property
    def fused_pass(self) -> bool:
        """True when the members' particle passes run as one persistent launch
        over all members' work items (pic_ens_fused_pass)."""
        f = C.c_int()
        _lib.call("pic_ens_fused_pass", self._h, C.byref(f))
        return bool(f.value)

    @fused_pass.setter
    def fused_pass(self, on: bool):
        _lib.call("pic_ens_set_fused_pass", self._h, int(bool(on)))

    def particle_count(self):
        return sum(sum(m.counters()["count"]) for m in self.members)

    def close(self):
        if self._h is not None and self._h.value:
            _lib.load().pic_ens_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
