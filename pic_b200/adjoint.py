"""Differentiable collisionless step: gradients of a final-density loss with
respect to electrode potentials and an initial-velocity perturbation, from
the hand-written adjoint in pic_b200/csrc/adjoint.cu (pic_adj_*), behind a
torch.autograd.Function.

The reference has no differentiable path; the forward model is its step
order (src/simulation.py:622-660) in FP64.  The differentiable workload:
  257x257 nodes (dx = 1e-4 m), 1e6 electrons + 1e6 ions, collisionless, 200
  steps of 1e-11 s; four electrode segments V1..V4 = left, bottom, right and
  top walls (corners belong to the left and right walls), V uniform in
  [0, 50] V; loss = mean over nodes of (n_e - n_target)^2 with n_target a
  seeded smooth Gaussian profile; perturbation vx += A sin(2 pi x / L) on the
  electrons; checkpoints every 20 steps.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import Consts, _lib, workloads


def wall_segments(nx, ny):
    """Dirichlet mask (all edges) and segment index per node: 0 left, 1 bottom,
    2 right, 3 top; the corners belong to the left and right walls."""
    mask = np.zeros((ny, nx), np.uint8)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    seg = np.full((ny, nx), -1, np.int32)
    seg[0, :] = 1
    seg[-1, :] = 3
    seg[:, 0] = 0
    seg[:, -1] = 2
    return mask.reshape(-1), seg.reshape(-1)


def target_density(nx, ny, n0, seed):
    """n0 (1 + a exp(-r^2 / 2 s^2)) with centre, width and amplitude drawn from the seed."""
    rng = np.random.Generator(np.random.Philox(seed))
    cx, cy = rng.uniform(0.3, 0.7, 2) * np.array([nx - 1, ny - 1])
    s = rng.uniform(0.1, 0.25) * (nx - 1)
    a = rng.uniform(0.3, 0.8)
    j, i = np.mgrid[0:ny, 0:nx]
    return (n0 * (1.0 + a * np.exp(-((i - cx) ** 2 + (j - cy) ** 2) / (2 * s * s)))).reshape(-1)


@dataclass
class AdjWorkload:
    nodes: int = 257
    n: int = 1_000_000  # per species
    steps: int = 200
    checkpoint_every: int = 20
    dx: float = 1e-4
    dt: float = 1e-11
    Te: float = 2.0
    Ti: float = 0.03
    n0: float = 1e14
    tol: float = 1e-11  # relative residual of every Poisson solve (near the FP64 floor at 257^2); 0: fixed cycles
    max_cycles: int = 60
    seed: int = 4

    def base(self) -> workloads.Workload:
        return workloads.Workload("adjoint", self.nodes, self.n, self.n, dx=self.dx, Te=self.Te, Ti=self.Ti,
                                  n0=self.n0, dt=self.dt, seed=self.seed)


class AdjointProblem:
    """One differentiable run: set the particles and target, then forward(V, A)
    gives the loss and backward() the gradients at those parameters."""

    def __init__(self, nx, ny, dx, dy, dt, species, mask, segment, nseg, steps, checkpoint_every, loss_species=0,
                 phi_fixed=None, tol=1e-12, max_cycles=60, eps0=Consts.eps0):
        d = _lib.AdjDesc()
        d.nx, d.ny, d.dx, d.dy, d.dt, d.eps0 = int(nx), int(ny), float(dx), float(dy), float(dt), float(eps0)
        d.nspecies = len(species)
        for k, s in enumerate(species):
            d.species[k] = _lib.AdjSpecies(int(s["n"]), float(s["charge"]), float(s["mass"]), float(s["np2c"]))
        self._mask = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        self._seg = np.ascontiguousarray(segment, dtype=np.int32).reshape(-1)
        self._fixed = None if phi_fixed is None else np.ascontiguousarray(phi_fixed, dtype=np.float64).reshape(-1)
        d.h_dirichlet = self._mask.ctypes.data
        d.h_segment = self._seg.ctypes.data
        d.h_phi_fixed = None if self._fixed is None else self._fixed.ctypes.data
        d.nseg = int(nseg)
        d.steps = int(steps)
        d.checkpoint_every = int(checkpoint_every)
        d.loss_species = int(loss_species)
        d.tol = float(tol)
        d.max_cycles = int(max_cycles)
        self.nseg = int(nseg)
        self.nx, self.ny = int(nx), int(ny)
        self._desc = d
        self._keep = []
        self._h = C.c_void_p()
        _lib.call("pic_adj_create", C.byref(d), C.byref(self._h))

    @staticmethod
    def _dev(a):
        return None if a is None else torch.as_tensor(a, dtype=torch.float64, device="cuda").contiguous()

    def set_particles(self, s, x, y, vx, vy, dvx=None, dvy=None):
        """Initial state of species s: positions in grid units, velocities and
        the perturbation direction in m/s."""
        arrs = [self._dev(a) for a in (x, y, vx, vy, dvx, dvy)]
        _lib.call("pic_adj_set_particles", self._h, int(s), *[_lib.ptr(a) for a in arrs], _lib.stream_ptr())
        torch.cuda.current_stream().synchronize()

    def set_target(self, target):
        t = self._dev(target)
        _lib.call("pic_adj_set_target", self._h, _lib.ptr(t), _lib.stream_ptr())
        torch.cuda.current_stream().synchronize()

    def forward(self, V, A) -> float:
        v = np.ascontiguousarray(np.asarray(V, dtype=np.float64).reshape(-1))
        assert v.size == self.nseg
        loss = C.c_double()
        _lib.call("pic_adj_forward", self._h, v.ctypes.data, float(A), C.byref(loss), _lib.stream_ptr())
        return loss.value

    def backward(self):
        dV = np.zeros(max(1, self.nseg))
        dA = C.c_double()
        _lib.call("pic_adj_backward", self._h, dV.ctypes.data, C.byref(dA), _lib.stream_ptr())
        return dV[: self.nseg].copy(), dA.value

    def freeze_absorption(self, on=True):
        """Reuse the last forward pass's absorption steps in later forward passes
        (the fixed mask the adjoint differentiates with)."""
        _lib.call("pic_adj_freeze_absorption", self._h, int(bool(on)))

    def state(self):
        """Device views after the last forward pass: x, y, ux, uy (FP64), death (int32), phi."""
        from .simulation import device_view

        p = [C.c_void_p() for _ in range(6)]
        _lib.call("pic_adj_state", self._h, *[C.byref(q) for q in p])
        n = sum(s.n for s in self._desc.species[: self._desc.nspecies])
        G = self.nx * self.ny
        f8, i4 = torch.float64, torch.int32
        return (device_view(p[0].value, n, f8), device_view(p[1].value, n, f8), device_view(p[2].value, n, f8),
                device_view(p[3].value, n, f8), device_view(p[4].value, n, i4), device_view(p[5].value, G, f8))

    def close(self):
        if self._h is not None and self._h.value:
            torch.cuda.synchronize()
            _lib.load().pic_adj_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ElectrodeLoss(torch.autograd.Function):
    """loss = ElectrodeLoss.apply(V, A, problem): V (nseg,) and A () FP64 tensors."""

    @staticmethod
    def forward(ctx, V, A, problem):
        ctx.problem = problem
        loss = problem.forward(V.detach().cpu().numpy(), float(A))
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        dV, dA = ctx.problem.backward()
        g = float(g)
        return torch.tensor(dV * g, dtype=torch.float64), torch.tensor(dA * g, dtype=torch.float64), None


def build(w: AdjWorkload):
    """The differentiable workload: (problem, V0, A0, inputs), with the
    electrons' perturbation direction sin(2 pi x / L) in vx."""
    b = w.base()
    rng = np.random.Generator(np.random.Philox(w.seed))
    e = workloads.species_arrays(b, "e", rng)
    i = workloads.species_arrays(b, "i", rng)
    V0 = rng.uniform(0.0, 50.0, 4)
    A0 = 1e4
    mask, seg = wall_segments(w.nodes, w.nodes)
    species = [dict(n=w.n, charge=-Consts.qe, mass=Consts.me, np2c=b.np2c(w.n)),
               dict(n=w.n, charge=Consts.qe, mass=workloads.ION_MASS, np2c=b.np2c(w.n))]
    prob = AdjointProblem(w.nodes, w.nodes, w.dx, w.dx, w.dt, species, mask, seg, 4, w.steps, w.checkpoint_every,
                          tol=w.tol, max_cycles=w.max_cycles)
    ex, ey, evx, evy = (np.asarray(a, np.float64) for a in e[:4])
    ix, iy, ivx, ivy = (np.asarray(a, np.float64) for a in i[:4])
    dvx = np.sin(2 * np.pi * ex / (w.nodes - 1))
    prob.set_particles(0, ex, ey, evx, evy, dvx, np.zeros_like(dvx))
    prob.set_particles(1, ix, iy, ivx, ivy)
    target = target_density(w.nodes, w.nodes, w.n0, w.seed + 1)
    prob.set_target(target)
    inputs = dict(e=(ex, ey, evx, evy, dvx), i=(ix, iy, ivx, ivy), target=target, mask=mask, seg=seg, species=species)
    return prob, V0, A0, inputs
