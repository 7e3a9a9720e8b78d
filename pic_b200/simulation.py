"""Time-step drivers.

``reference_step`` / ``reference_init_step`` replay SimulationManager._step /
_init_step (src/simulation.py:622-660) on the drop-in objects, one operator
call per reference call.  ``PICSimulation`` is the fast path: the whole step
in one particle pass plus the field solve (pic_sim_*, pic_b200/csrc/step.cu).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import Consts, _lib
from .MCC import MccTables


def reference_init_step(particles, grid, solver, dt, boundaries=None):
    """_init_step (src/simulation.py:622-637)."""
    grid.update_density(particles)
    solver.solve(grid)
    grid.update_E()
    particles.update_V(grid, -dt / 2)


def reference_step(particles, grid, dt, solver, mcc=None):
    """_step (src/simulation.py:640-660) with wall absorption in place of the
    axis reflection; `mcc` is an optional callable run after the kick."""
    particles.update_R(dt)
    particles.update_axis(dt)
    grid.update_density(particles)
    solver.solve(grid)
    grid.update_E()
    particles.update_V(grid, dt)
    if mcc is not None:
        mcc(particles)


class _DevArray:
    """__cuda_array_interface__ wrapper of a library-owned device buffer."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_view(ptr, n, dtype=torch.float32):
    typestr = {torch.float32: "<f4", torch.float64: "<f8", torch.int32: "<i4"}[dtype]
    return torch.as_tensor(_DevArray(ptr, n, typestr), device="cuda")


class PICSimulation:
    """The fused electrostatic PIC step on one GPU.

    species: list of dicts with keys name, charge (C), mass (kg), np2c, capacity.
    dirichlet / phi_bc: node mask (1 = Dirichlet) and potentials, nx*ny.
    min_cycles: V-cycles every step's field solve runs before it first tests
    the residual against tol (then one at a time until converged); a solve from
    the extrapolated potential of the last two steps needs at least two at the
    tolerances of a PIC step, and cycles that are not tested cost no WHILE-node
    iteration in the captured step.
    coarse_fp32: keep the mixed-precision V-cycle's direct solve of its first
    level of at most 33^2 nodes in FP32 (default: FP64).
    push_kernel: how the particle pass streams the particles, all with
    bit-identical results: "ring" (the block streams chunks through one
    shared ring of bulk copies; the fastest measured), "warp" (every warp
    streams its own groups through its own stage buffers, E tiles by bulk
    tensor copies) or "warp_agg" ("warp" with warp-aggregated deposit atomics).
    geometry: "cartesian", or "rz" for the axisymmetric r-z step (the
    reference's Grid.Cylindrical = 1): x axial, y radial (row 0 the axis, a
    free row), vx axial, vy radial, vz azimuthal; np2c counts real particles;
    rho is the charge density of the node volumes; the drift turns (vy, vz)
    into the particle's new local frame.
    """

    def __init__(self, nx, ny, dx, dy, dt, species, dirichlet, phi_bc=None, tol=1e-8, max_cycles=50,
                 precision="mixed", pre_sweeps=2, post_sweeps=2, omega=1.15, sort_interval=20, tile=16,
                 mcc: MccTables | None = None, seed=0, use_graph=False, eps0=Consts.eps0, mg_launch="graph",
                 coarsest_max=9, geometry="cartesian", min_cycles=2, push_kernel="ring", coarse_fp32=False):
        self.nx, self.ny, self.dx, self.dy, self.dt = int(nx), int(ny), float(dx), float(dy), float(dt)
        self.species = list(species)
        self.geometry = geometry
        d = _lib.SimDesc()
        d.nx, d.ny, d.dx, d.dy, d.dt, d.eps0 = self.nx, self.ny, self.dx, self.dy, self.dt, eps0
        d.nspecies = len(self.species)
        for k, s in enumerate(self.species):
            d.species[k] = _lib.SpeciesDesc(int(s["capacity"]), float(s["charge"]), float(s["mass"]),
                                            float(s["np2c"]))
        self._mask = np.ascontiguousarray(np.asarray(dirichlet).reshape(-1) != 0, dtype=np.uint8)
        self._phi_bc = np.ascontiguousarray(np.zeros(self.nx * self.ny) if phi_bc is None else phi_bc,
                                            dtype=np.float64).reshape(-1)
        d.h_dirichlet = self._mask.ctypes.data
        d.h_phi_bc = self._phi_bc.ctypes.data
        d.tol = float(tol)
        d.max_cycles = int(max_cycles)
        d.mg = _lib.MgOptions(_lib.PIC_MG_MIXED if precision == "mixed" else _lib.PIC_MG_FP64, pre_sweeps,
                              post_sweeps, omega, int(coarsest_max), _lib.MG_LAUNCH_MODES[mg_launch],
                              _lib.GEOMETRIES[geometry], int(bool(coarse_fp32)))
        d.sort_interval = int(sort_interval)
        d.tile = int(tile)
        self._mcc_desc = mcc.desc() if mcc is not None else None
        d.mcc = C.cast(C.pointer(self._mcc_desc), C.c_void_p) if mcc is not None else None
        d.seed = int(seed)
        d.use_graph = int(use_graph)
        d.min_cycles = int(min_cycles)
        d.push_kernel = _lib.PUSH_KERNELS[push_kernel]
        self._desc = d
        self._h = C.c_void_p()
        _lib.call("pic_sim_create", C.byref(d), _lib.stream_ptr(), C.byref(self._h))

    def close(self):
        if self._h is not None and self._h.value:
            torch.cuda.synchronize()
            _lib.load().pic_sim_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state ----
    def load(self, s, x, y, vx, vy, vz=None):
        """Load species s: positions in grid units, velocities in m/s (numpy arrays,
        host torch tensors or device tensors)."""
        arrs = [x, y, vx, vy, vz]
        if all(a is None or isinstance(a, np.ndarray) for a in arrs):
            host = [None if a is None else np.ascontiguousarray(a, dtype=np.float32) for a in arrs]
            n = len(host[0])
            _lib.call("pic_sim_load_species", self._h, s, *[None if a is None else a.ctypes.data for a in host], n, 1,
                      _lib.stream_ptr())
        elif all(a is None or (isinstance(a, torch.Tensor) and a.device.type == "cpu") for a in arrs):
            # host tensors (pinned ones copy by DMA without staging)
            host = [None if a is None else a.to(torch.float32).contiguous() for a in arrs]
            n = host[0].numel()
            _lib.call("pic_sim_load_species", self._h, s, *[None if a is None else a.data_ptr() for a in host], n, 1,
                      _lib.stream_ptr())
        else:
            dev = [None if a is None else torch.as_tensor(a, dtype=torch.float32, device="cuda").contiguous()
                   for a in arrs]
            n = dev[0].numel()
            _lib.call("pic_sim_load_species", self._h, s, *[_lib.ptr(a) for a in dev], n, 0, _lib.stream_ptr())

    def init(self):
        rc = _lib.load().pic_sim_init(self._h, _lib.stream_ptr())
        if rc not in (_lib.PIC_OK, _lib.PIC_ERR_NOT_CONVERGED):
            _lib.check(rc, "pic_sim_init")
        return rc

    def step(self, n=1):
        rc = _lib.load().pic_sim_step(self._h, int(n), _lib.stream_ptr())
        if rc not in (_lib.PIC_OK, _lib.PIC_ERR_NOT_CONVERGED):
            _lib.check(rc, "pic_sim_step")
        return rc

    def sync(self):
        _lib.call("pic_sim_sync", self._h, _lib.stream_ptr())

    def counters(self) -> dict:
        c = _lib.SimCounters()
        _lib.call("pic_sim_read_counters", self._h, C.byref(c), _lib.stream_ptr())
        ns = len(self.species)
        return {
            "absorbed": [c.absorbed[s] for s in range(ns)],
            "collisions": [[c.collisions[s][k] for k in range(_lib.PIC_MAX_PROCESSES)] for s in range(ns)],
            "null_candidates": [c.null_candidates[s] for s in range(ns)],
            "born": [c.born[s] for s in range(ns)],
            "dropped_births": c.dropped_births,
            "nu_overflow": c.nu_overflow,
            "count": [c.count[s] for s in range(ns)],
            "last_cycles": c.last_cycles,
            "last_rel_res": c.last_rel_res,
            "steps": c.steps,
            "electrode_absorbed": [c.electrode_absorbed[s] for s in range(ns)],
            "candidate_overflow": c.candidate_overflow,
        }

    def particle_buffer(self, x_range=None, y_range=None, out=None):
        """The renderer's particle vertex buffer (src/Render.py:544-571) as a
        device tensor (n, 3) float32: positions normalised to [-1, 1] over the
        ranges in metres (default: the grid), and the species type (index + 1),
        live particles in species order.  `out` (capacity, 3) is reused when given."""
        xr = x_range or (0.0, self.dx * (self.nx - 1))
        yr = y_range or (0.0, self.dy * (self.ny - 1))
        if out is None:
            cap = sum(int(s["capacity"]) for s in self.species)
            out = torch.empty((cap, 3), dtype=torch.float32, device="cuda")
        n = C.c_int()
        _lib.call("pic_sim_particle_buffer", self._h, out.data_ptr(), out.shape[0], float(xr[0]), float(xr[1]),
                  float(yr[0]), float(yr[1]), C.byref(n), _lib.stream_ptr())
        return out[: n.value]

    def mg_effective_launch(self) -> str:
        """The launch mode of the field solves ("dst" where the sine-transform solve applies)."""
        m = C.c_int()
        _lib.call("pic_sim_solver_mode", self._h, C.byref(m))
        return {v: k for k, v in _lib.MG_LAUNCH_MODES.items()}[m.value]

    def diagnostics(self) -> dict:
        """Kinetic energy and momentum per species, field energy and Gauss's law
        terms of the current state (pic_sim_diagnostics)."""
        d = _lib.SimDiag()
        _lib.call("pic_sim_diagnostics", self._h, C.byref(d), _lib.stream_ptr())
        ns = len(self.species)
        return {"live": [d.live[s] for s in range(ns)], "kinetic": [d.kinetic[s] for s in range(ns)],
                "momentum": [[d.momentum[s][c] for c in range(3)] for s in range(ns)],
                "field_energy": d.field_energy, "gauss_flux": d.gauss_flux, "gauss_charge": d.gauss_charge,
                "div_error_l2": d.div_error_l2}

    def species_arrays(self, s):
        """Zero-copy torch views (x, y, vx, vy, vz) of the first `count` slots of species s."""
        ptrs = [C.c_void_p() for _ in range(5)]
        _lib.call("pic_sim_species_arrays", self._h, s, *[C.byref(p) for p in ptrs])
        n = self.counters()["count"][s]
        return tuple(device_view(p.value, n) for p in ptrs)

    def read_particles(self, s, out):
        """Copies the slots in use of species s to the host tensor `out`
        (float32, page-locked for an asynchronous copy, at least 5 * count
        values) as rows x, y, vx, vy, vz, one copy per array on the current
        stream; returns the (5, count) view of `out`."""
        n = C.c_int()
        _lib.call("pic_sim_read_particles", self._h, s, out.data_ptr(), out.numel(), C.byref(n), _lib.stream_ptr())
        return out[: 5 * n.value].view(5, n.value)

    def sort(self):
        """The cell sort of every species now (what a step runs every sort_interval steps)."""
        _lib.call("pic_sim_sort", self._h, _lib.stream_ptr())

    def fields(self):
        """Zero-copy views: phi (FP64), rho of the last deposit, Ex, Ey (float32), all nx*ny."""
        p = [C.c_void_p() for _ in range(4)]
        _lib.call("pic_sim_fields", self._h, *[C.byref(q) for q in p])
        G = self.nx * self.ny
        return (device_view(p[0].value, G, torch.float64), device_view(p[1].value, G), device_view(p[2].value, G),
                device_view(p[3].value, G))

    def kernel_launches(self) -> int:
        """Kernel launches issued since creation."""
        return int(_lib.load().pic_sim_kernel_launches(self._h))

    def set_wait_limit(self, polls=-1):
        """Polls a bounded device wait (the particle pass's bulk copies, the
        persistent solve's grid barriers) makes before it gives up; the next
        counters() raises PicError(PIC_ERR_TIMEOUT).  -1 restores the default."""
        _lib.call("pic_sim_set_wait_limit", self._h, int(polls))

    def set_profiling(self, on: bool):
        _lib.call("pic_sim_set_profiling", self._h, int(bool(on)))

    def read_profile(self) -> dict:
        p = _lib.SimProfile()
        _lib.call("pic_sim_read_profile", self._h, C.byref(p))
        out = {name: {"ms": p.ms[k], "count": p.count[k]} for k, name in enumerate(_lib.PHASES)}
        out["mg_cycles"] = p.mg_cycles
        return out
