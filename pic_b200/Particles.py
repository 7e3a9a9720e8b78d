"""Particles2D: drop-in for src/Particles.py:283-690, Cartesian or r-z.

Storage is one SoA group per species (x, y, vx, vy, vz float32 on the GPU),
positions in grid units (x/dx, y/dy) and velocities in m/s, instead of the
reference's AoS FP64 R (N,2) / V (N,3) with a part_type column.  The
reference's attributes are provided as computed views: ``R`` and ``V`` (FP64,
metres and m/s, live particles of all species in species order) and
``part_type``.  Slots of absorbed particles hold NaN until ``compact()``.

cylindrical=True (r-z): x is the axial and y the radial position, vx, vy,
vz the axial, radial and azimuthal velocities.  update_V is the reference's
cylindrical kick (src/Particles.py:183-248, the same gather as Cartesian);
update_R drifts in 3D and turns (vy, vz) into the new local frame
(pic_update_R_rz), where the reference drifts in the plane and reflects at
the axis (src/Particles.py:267-280).  The loaders then draw radii uniform in
volume (density proportional to r).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

DEVICE = "cuda"


class Species:
    """One species' SoA arrays (capacity slots; the first n are in use)."""

    def __init__(self, name, mass, charge, collision_model, capacity):
        self.name = name
        self.mass = float(mass)
        self.charge = float(charge)
        self.collision_model = int(collision_model)
        self.capacity = int(capacity)
        self.n = 0
        self.np2c = None
        z = lambda: torch.zeros(self.capacity, dtype=torch.float32, device=DEVICE)  # noqa: E731
        self.x, self.y, self.vx, self.vy, self.vz = z(), z(), z(), z(), z()

    def arrays(self):
        return self.x, self.y, self.vx, self.vy, self.vz


class Particles2D:
    """Particles2D(N) -- N slots per species (src/Particles.py:284)."""

    def __init__(self, N, cylindrical=False):
        self.cylindrical = bool(cylindrical)
        self.N = int(N)
        self.species: list[Species] = []
        self.part_name = ["reserved"]
        self.np2c = 1
        self.grid = None  # the Grid2D whose dx, dy define the grid units
        self.absorbed = torch.zeros(1, dtype=torch.int64, device=DEVICE)
        self.mcc_mask = None
        self.mcc_count = 0
        self._gen = torch.Generator(device="cpu")
        self._gen.manual_seed(0)

    # ---- species tables (src/Particles.py:318-352) ----
    def add_species(self, species_name: str, species_mass: float, species_charge: float, collision_model: int = 0):
        if len(self.species) >= _lib.PIC_MAX_SPECIES:
            raise ValueError(f"at most {_lib.PIC_MAX_SPECIES} species")
        self.part_name.append(species_name)
        self.species.append(Species(species_name, species_mass, species_charge, collision_model, self.N))

    @property
    def species_count(self):
        return len(self.species)

    @property
    def m_type(self):
        return torch.tensor([0.0] + [s.mass for s in self.species], dtype=torch.float64)

    @property
    def m_type_inv(self):
        return torch.tensor([0.0] + [1.0 / s.mass for s in self.species], dtype=torch.float64)

    @property
    def q_type(self):
        return torch.tensor([0.0] + [s.charge for s in self.species], dtype=torch.float64)

    @property
    def collision_model(self):
        return torch.tensor([128] + [s.collision_model for s in self.species], dtype=torch.int32)

    def species_np2c(self, s: Species) -> float:
        return float(self.np2c if s.np2c is None else s.np2c)

    def get_species(self, species) -> Species:
        if isinstance(species, Species):
            return species
        if isinstance(species, int):
            return self.species[species - 1]
        return self.species[self.part_name.index(species) - 1]

    def set_mcc_mask(self):
        """Species with collision model 0 take part in MCC (src/Particles.py:354-357)."""
        self.mcc_mask = [s.collision_model == 0 for s in self.species]
        self.mcc_count = sum(s.n for s, m in zip(self.species, self.mcc_mask) if m)

    def __len__(self):
        return self.last_alive

    @property
    def last_alive(self):
        return sum(s.n for s in self.species)

    def __str__(self):
        return f"Particles2D, {self.last_alive} particles, {self.species_count} species"

    # ---- loading ----
    def _require_grid(self, grid=None):
        g = grid if grid is not None else self.grid
        if g is None:
            raise ValueError("attach a Grid2D first (particles.grid = grid) to convert metres to grid units")
        self.grid = g
        return g

    def load_species_arrays(self, species, x, y, vx, vy, vz=None, grid=None):
        """Append particles given in metres and m/s (host or device arrays)."""
        g = self._require_grid(grid)
        s = self.get_species(species)
        x = torch.as_tensor(x, dtype=torch.float64)
        n = int(x.numel())
        if s.n + n > s.capacity:
            raise _lib.PicError(_lib.PIC_ERR_OUT_OF_CAPACITY, f"species {s.name}: {s.n + n} > {s.capacity}")
        cols = [
            (x / g.dx).float(),
            (torch.as_tensor(y, dtype=torch.float64) / g.dy).float(),
            torch.as_tensor(vx, dtype=torch.float32),
            torch.as_tensor(vy, dtype=torch.float32),
            torch.zeros(n, dtype=torch.float32) if vz is None else torch.as_tensor(vz, dtype=torch.float32),
        ]
        for dst, src in zip(s.arrays(), cols):
            dst[s.n:s.n + n].copy_(src.reshape(-1))
        s.n += n

    def uniform_species_load(self, x1, y1, x2, y2, n, species, grid=None):
        """Uniform positions in [x1,x2]x[y1,y2]; vx one U(-0.1,0.1) value, vy = 0,
        as src/Particles.py:683-690 (seeded here)."""
        n = int(n)
        u = torch.rand((2, n), generator=self._gen, dtype=torch.float64)
        vx0 = float(torch.rand(1, generator=self._gen, dtype=torch.float64) * 0.2 - 0.1)
        self.load_species_arrays(species, x1 + (x2 - x1) * u[0], self._radial(y1, y2, u[1]), torch.full((n,), vx0),
                                 torch.zeros(n), None, grid)

    def _radial(self, y1, y2, u):
        """y1 + (y2 - y1) u; in r-z, radii with density proportional to r (uniform in volume)."""
        if not self.cylindrical:
            return y1 + (y2 - y1) * u
        return (y1 * y1 + (y2 * y2 - y1 * y1) * u) ** 0.5

    def maxwellian_species_load(self, x1, y1, x2, y2, n, species, T_eV, seed=0, grid=None):
        """Uniform positions and Maxwellian velocities N(0, sqrt(kT/m)) per component."""
        from .Consts import qe

        s = self.get_species(species)
        rng = np.random.Generator(np.random.Philox(seed))
        vth = np.sqrt(T_eV * qe / s.mass)
        x = rng.uniform(x1, x2, n)
        y = self._radial(y1, y2, rng.uniform(0.0, 1.0, n)) if self.cylindrical else rng.uniform(y1, y2, n)
        self.load_species_arrays(species, x, y, rng.normal(0, vth, n), rng.normal(0, vth, n), rng.normal(0, vth, n),
                                 grid)

    # ---- reference views ----
    @property
    def R(self):
        g = self._require_grid()
        xs = [torch.stack([s.x[:s.n].double() * g.dx, s.y[:s.n].double() * g.dy], 1) for s in self.species]
        return torch.cat(xs) if xs else torch.zeros((0, 2), dtype=torch.float64, device=DEVICE)

    @property
    def V(self):
        vs = [torch.stack([s.vx[:s.n], s.vy[:s.n], s.vz[:s.n]], 1).double() for s in self.species]
        return torch.cat(vs) if vs else torch.zeros((0, 3), dtype=torch.float64, device=DEVICE)

    @property
    def part_type(self):
        ts = [torch.full((s.n,), k + 1, dtype=torch.int32, device=DEVICE) for k, s in enumerate(self.species)]
        return torch.cat(ts) if ts else torch.zeros(0, dtype=torch.int32, device=DEVICE)

    # ---- push (src/Particles.py:359-410) ----
    def update_R(self, dt):
        """x += v dt (src/Particles.py:359-367); r-z: the drift of pic_update_R_rz."""
        g = self._require_grid()
        for s in self.species:
            if not s.n:
                continue
            if self.cylindrical:
                _lib.call("pic_update_R_rz", _lib.ptr(s.x), _lib.ptr(s.y), _lib.ptr(s.vx), _lib.ptr(s.vy),
                          _lib.ptr(s.vz), s.n, float(dt / g.dx), float(dt / g.dy), _lib.stream_ptr())
            else:
                _lib.call("pic_update_R", _lib.ptr(s.x), _lib.ptr(s.y), _lib.ptr(s.vx), _lib.ptr(s.vy), s.n,
                          float(dt / g.dx), float(dt / g.dy), None, None, _lib.stream_ptr())

    def update_axis(self, dt=None):
        """Wall absorption on all four walls.  The reference reflects at y < 0
        here (src/Particles.py:267-280, 369-376); this build absorbs instead."""
        g = self._require_grid()
        for s in self.species:
            if s.n:
                _lib.call("pic_absorb", _lib.ptr(s.x), _lib.ptr(s.y), s.n, g.m, g.n, _lib.ptr(self.absorbed),
                          _lib.stream_ptr())

    absorb = update_axis

    def update_V(self, grid, dt):
        """Gather E at each particle and kick v += q/m E dt (src/Particles.py:378-410)."""
        self.grid = grid
        for s in self.species:
            if s.n:
                _lib.call("pic_update_V", _lib.ptr(s.x), _lib.ptr(s.y), _lib.ptr(s.vx), _lib.ptr(s.vy), s.n,
                          _lib.ptr(grid.E[0]), _lib.ptr(grid.E[1]), grid.m, grid.n, float(s.charge / s.mass * dt),
                          _lib.stream_ptr())

    # ---- removal and sorting ----
    def compact(self):
        """Drop dead slots, keeping the order of the live ones (stable)."""
        for s in self.species:
            if s.n == 0:
                continue
            live = ~torch.isnan(s.x[:s.n])
            k = int(live.sum())
            for a in s.arrays():
                a[:k] = a[:s.n][live].clone()
            s.n = k

    def remove(self, indices, species=1):
        """Mark the given slots of a species dead and compact (src/Particles.py:634-652,
        which swaps with the tail; this keeps the survivors' order).  Returns the count."""
        s = self.get_species(species)
        idx = torch.as_tensor(indices, device=DEVICE, dtype=torch.int64)
        if idx.numel() == 0:
            return 0
        s.x[idx] = float("nan")
        s.y[idx] = float("nan")
        before = s.n
        self.compact()
        return before - s.n

    def sort(self, tile=16):
        """Deterministic stable sort of every species by tile-major cell key
        (replaces src/Particles.py:550-632).  Returns the permutations."""
        g = self._require_grid()
        perms = []
        for s in self.species:
            if s.n == 0:
                perms.append(torch.zeros(0, dtype=torch.int32, device=DEVICE))
                continue
            sorter = _lib.C.c_void_p()
            _lib.call("pic_sorter_create", s.capacity, g.m, g.n, tile, _lib.C.byref(sorter))
            try:
                outs = [torch.empty_like(a) for a in s.arrays()]
                perm = torch.empty(s.capacity, dtype=torch.int32, device=DEVICE)
                cnt = torch.zeros(1, dtype=torch.int32, device=DEVICE)
                _lib.call("pic_sort", sorter, *[_lib.ptr(a) for a in s.arrays()], s.n, *[_lib.ptr(o) for o in outs],
                          _lib.ptr(perm), _lib.ptr(cnt), None, _lib.stream_ptr())
                k = int(cnt.item())
                s.x, s.y, s.vx, s.vy, s.vz = outs
                s.n = k
                perms.append(perm[:k].clone())
            finally:
                torch.cuda.synchronize()
                _lib.load().pic_sorter_destroy(sorter)
        return perms
