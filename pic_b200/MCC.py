"""MCC: drop-in for src/MCC.py (null-collision Monte-Carlo collisions).

``null_collision_method`` keeps the reference's signature
(src/MCC.py:308-315) but performs a complete null-collision step on the GPU
(pic_mcc_apply): candidate selection with P_null = 1 - exp(-nu' dt), process
choice by the cumulative n_g sigma_k(E) v, and scattering -- where the
reference returns before applying any collision (src/MCC.py:394).  Energies
are in eV (the reference compares joules with eV tables).  Random numbers
come from Philox4x32-10 keyed by ``seed`` and a step counter.

``MccTables`` describes the processes of every species for the fused step
(pic_b200.simulation.PICSimulation) and for ``MccOperator``.
"""
from __future__ import annotations

import ctypes as C
import hashlib

import numpy as np
import torch

from . import Consts, _lib

ELASTIC, EXCITATION, IONIZATION, CHARGE_EXCHANGE = (_lib.PIC_ELASTIC, _lib.PIC_EXCITATION, _lib.PIC_IONIZATION,
                                                    _lib.PIC_CHARGE_EXCHANGE)


def read_cross_section(filename):
    """Two whitespace-separated columns (eV, m^2) -> (energies, sigma) (src/MCC.py:126-145).
    Returns (None, None) and prints on error, like the reference."""
    try:
        rows = []
        with open(filename) as f:
            for line in f:
                p = line.split()
                if len(p) == 2:
                    rows.append((float(p[0]), float(p[1])))
        a = np.asarray(rows, dtype=np.float64)
        return a[:, 0], a[:, 1]
    except Exception as e:  # noqa: BLE001 - reference behaviour
        print(f"Error reading cross-section file {filename}: {e}")
        return None, None


def log_grid(e0=0.01, e1=1000.0, n=1000):
    return np.geomspace(e0, e1, n)


def resample(energy, sigma, grid):
    """Linear interpolation in E (src/MCC.py:62-79), clamped at the ends (:54-60)."""
    return np.interp(grid, np.asarray(energy, np.float64), np.asarray(sigma, np.float64))


class MccTables:
    """Per-species process lists on a shared log-spaced energy grid."""

    def __init__(self, energy, gas_density, gas_temperature, gas_mass):
        self.energy = np.ascontiguousarray(energy, dtype=np.float64)
        self.gas_density = float(gas_density)
        self.gas_temperature = float(gas_temperature)
        self.gas_mass = float(gas_mass)
        self.species = {}  # index -> list of (type, threshold, sigma)
        self.products = {}  # index -> (born electron species, born ion species)

    def add(self, species_index, ptype, sigma, threshold=0.0):
        sig = np.ascontiguousarray(sigma, dtype=np.float64)
        if sig.shape != self.energy.shape:
            raise ValueError("sigma must be tabulated on the shared energy grid")
        self.species.setdefault(species_index, []).append((int(ptype), float(threshold), sig))
        return self

    def set_products(self, species_index, electron_species, ion_species):
        self.products[species_index] = (int(electron_species), int(ion_species))
        return self

    def desc(self):
        """A pic_mcc_desc; keep the returned object alive while it is used."""
        d = _lib.MccDesc()
        d.ne = len(self.energy)
        d.h_energy = self.energy.ctypes.data
        d.gas_density = self.gas_density
        d.gas_temperature = self.gas_temperature
        d.gas_mass = self.gas_mass
        keep = [self.energy]
        for s, procs in self.species.items():
            sd = d.species[s]
            sd.nproc = len(procs)
            for k, (t, thr, sig) in enumerate(procs):
                sd.type[k] = t
                sd.threshold[k] = thr
                sd.h_sigma[k] = sig.ctypes.data
                keep.append(sig)
            sd.born_electron_species, sd.born_ion_species = self.products.get(s, (-1, -1))
        d._keep = keep
        return d


class MccOperator:
    """A pic_mcc handle plus a birth buffer, for the per-operator API."""

    def __init__(self, tables: MccTables, masses, dt, birth_capacity=1 << 16, seed=0):
        self.tables = tables
        self._desc = tables.desc()
        masses = (C.c_double * len(masses))(*masses)
        self._h = C.c_void_p()
        _lib.call("pic_mcc_create", C.byref(self._desc), len(masses), masses, float(dt), C.byref(self._h))
        self.seed = int(seed)
        self.step = 0
        dev = "cuda"
        z = lambda: torch.zeros(birth_capacity, dtype=torch.float32, device=dev)  # noqa: E731
        self.bx, self.by, self.bvx, self.bvy, self.bvz = z(), z(), z(), z(), z()
        self.bspecies = torch.zeros(birth_capacity, dtype=torch.int32, device=dev)
        self.bcount = torch.zeros(1, dtype=torch.int32, device=dev)
        self.counters = torch.zeros(30, dtype=torch.int64, device=dev)
        self._bb = _lib.BirthBuffer(self.bx.data_ptr(), self.by.data_ptr(), self.bvx.data_ptr(), self.bvy.data_ptr(),
                                    self.bvz.data_ptr(), self.bspecies.data_ptr(), self.bcount.data_ptr(),
                                    birth_capacity)

    def query(self, s):
        nu, p, inv = C.c_double(), C.c_double(), C.c_double()
        _lib.call("pic_mcc_query", self._h, s, C.byref(nu), C.byref(p), C.byref(inv))
        return nu.value, p.value, inv.value

    def apply(self, s, x, y, vx, vy, vz, n, step=None):
        st = self.step if step is None else step
        _lib.call("pic_mcc_apply", self._h, s, _lib.ptr(x), _lib.ptr(y), _lib.ptr(vx), _lib.ptr(vy), _lib.ptr(vz),
                  int(n), self.seed, int(st), C.byref(self._bb), _lib.ptr(self.counters), _lib.stream_ptr())
        if step is None:
            self.step += 1

    def take_births(self):
        k = min(int(self.bcount.item()), self.bx.numel())
        out = (self.bspecies[:k].clone(), self.bx[:k].clone(), self.by[:k].clone(), self.bvx[:k].clone(),
               self.bvy[:k].clone(), self.bvz[:k].clone())
        self.bcount.zero_()
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize()
                _lib.load().pic_mcc_destroy(h)
            except Exception:
                pass
            self._h = None


# Operators of null_collision_method, keyed by what determines them: the
# cross-section tables' contents (a digest, so that a new table object with
# the same values reuses the operator and one with other values never does),
# the gas, dt, the seed and the species' masses.  At most _MAX_OPERATORS are
# kept, the least recently used dropped first.
_operators: dict = {}
_MAX_OPERATORS = 8


def _operator_key(particles, density, cross_sections, dt, ionization, seed, gas_temperature, gas_mass, threshold):
    h = hashlib.sha1()
    for table in cross_sections:
        for col in table:
            h.update(b"none" if col is None else np.ascontiguousarray(col, dtype=np.float64).tobytes())
            h.update(b"|")
        h.update(b"||")
    masses = tuple((s.mass, s.charge, s.collision_model) for s in particles.species)
    return (h.hexdigest(), float(density), float(dt), bool(ionization), int(seed), float(gas_temperature),
            float(gas_mass), float(threshold), masses)


def null_collision_method(particles, density, cross_sections, dt, max_particles, IONIZATION=True, seed=0,
                          gas_temperature=300.0, gas_mass=40 * Consts.AMU, ionization_threshold=15.6):
    """MCC for the species with collision model 0 (src/MCC.py:308-415).

    cross_sections = ((E_el, sigma_el), (E_ion, sigma_ion)) in (eV, m^2);
    elastic always, ionisation when IONIZATION.  New electrons join the MCC
    species; new ions join the first positively charged species (the
    reference creates no ions, src/MCC.py:283-305)."""
    particles.set_mcc_mask()
    targets = [k for k, on in enumerate(particles.mcc_mask) if on]
    if not targets:
        return
    s_e = targets[0]
    ions = [k for k, s in enumerate(particles.species) if s.charge > 0]
    s_i = ions[0] if ions else s_e
    grid = log_grid()
    key = _operator_key(particles, density, cross_sections, dt, IONIZATION, seed, gas_temperature, gas_mass,
                        ionization_threshold)
    op = _operators.pop(key, None)
    if op is None:
        t = MccTables(grid, density, gas_temperature, gas_mass)
        t.add(s_e, ELASTIC, resample(*cross_sections[0], grid))
        if IONIZATION and len(cross_sections) > 1 and cross_sections[1][0] is not None:
            e_ion, s_ion = cross_sections[1]
            thr = float(e_ion[np.argmax(np.asarray(s_ion) > 0)]) if np.any(np.asarray(s_ion) > 0) else \
                ionization_threshold
            t.add(s_e, IONIZATION, resample(e_ion, s_ion, grid), threshold=thr)
            t.set_products(s_e, s_e, s_i)
        op = MccOperator(t, [s.mass for s in particles.species], dt, seed=seed)
    _operators[key] = op  # most recently used last
    while len(_operators) > _MAX_OPERATORS:
        _operators.pop(next(iter(_operators)))
    sp = particles.species[s_e]
    op.apply(s_e, sp.x, sp.y, sp.vx, sp.vy, sp.vz, sp.n)
    species, bx, by, bvx, bvy, bvz = op.take_births()
    g = particles.grid
    for k in range(len(particles.species)):
        sel = species == k
        if int(sel.sum()) == 0:
            continue
        particles.load_species_arrays(k + 1, bx[sel].double() * g.dx, by[sel].double() * g.dy, bvx[sel], bvy[sel],
                                      bvz[sel])
