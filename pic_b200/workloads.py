"""Seeded synthetic inputs for the benchmark and parity workloads.

The reference publishes no dataset; each workload is described by its grid,
particle counts, temperatures, density, boundary voltages and (for the MCC
workload) analytic cross-section formulas, and generated from a Philox seed.
  small      129x129 nodes, dx = 1e-4 m, 1e5 electrons + 1e5 ions (40 amu),
             Te = 2 eV, Ti = 0.03 eV, n0 = 1e14 m^-3, grounded walls,
             dt = 1e-11 s, multigrid to 1e-8, collisionless
  mcc        513x513 nodes, 4M + 4M particles, left wall 100 V, argon-like
             gas 1e21 m^-3 at 300 K with elastic / excitation / ionisation
             (electrons) and charge exchange (ions) on 1000 log-spaced
             energies 0.01-1000 eV
  large      2049x2049 nodes, 64M + 64M particles, electrons half in a
             Gaussian blob (sigma = 0.2 L), multigrid to 1e-10
Positions are uniform in the domain (grid units), velocity components
Maxwellian N(0, sqrt(kT/m)); np2c = n0 L^2 / N per species.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import Consts
from .MCC import CHARGE_EXCHANGE, ELASTIC, EXCITATION, IONIZATION, MccTables, log_grid

ION_MASS = 40 * Consts.AMU


@dataclass
class Workload:
    name: str
    nodes: int
    n_e: int
    n_i: int
    dx: float = 1e-4
    Te: float = 2.0
    Ti: float = 0.03
    n0: float = 1e14
    dt: float = 1e-11
    tol: float = 1e-8
    left_V: float = 0.0
    mcc: bool = False
    steps: int = 100
    seed: int = 0
    blob: bool = False
    gas_density: float = 1e21
    gas_temperature: float = 300.0
    extra: dict = field(default_factory=dict)

    @property
    def L(self):
        return self.dx * (self.nodes - 1)

    def np2c(self, n):
        return self.n0 * self.L * self.L / n


SMALL = Workload("small", 129, 100_000, 100_000, tol=1e-8, steps=100)
MCC = Workload("mcc", 513, 4_000_000, 4_000_000, left_V=100.0, mcc=True, steps=1000)
LARGE = Workload("large", 2049, 64_000_000, 64_000_000, tol=1e-10, steps=200, blob=True)
WORKLOADS = {w.name: w for w in (SMALL, MCC, LARGE)}


def scaled(w: Workload, nodes=None, n=None, **kw) -> Workload:
    """A copy with a different grid and particle count (parity-test sizes)."""
    d = dict(w.__dict__)
    if nodes is not None:
        d["nodes"] = nodes
    if n is not None:
        d["n_e"] = d["n_i"] = n
    d.update(kw)
    return Workload(**d)


def species_arrays(w: Workload, which: str, rng: np.random.Generator):
    """(x, y, vx, vy, vz) as float32 numpy arrays: positions in grid units."""
    n = w.n_e if which == "e" else w.n_i
    mass = Consts.me if which == "e" else ION_MASS
    T = w.Te if which == "e" else w.Ti
    top = np.float32(w.nodes - 1)
    if which == "e" and w.blob:
        h = n // 2
        c = 0.5 * (w.nodes - 1)
        sig = 0.2 * (w.nodes - 1)
        bx, by = rng.normal(c, sig, h), rng.normal(c, sig, h)
        bad = (bx < 0) | (bx >= top) | (by < 0) | (by >= top)
        while bad.any():
            k = int(bad.sum())
            bx[bad], by[bad] = rng.normal(c, sig, k), rng.normal(c, sig, k)
            bad = (bx < 0) | (bx >= top) | (by < 0) | (by >= top)
        x = np.concatenate([bx, rng.uniform(0, w.nodes - 1, n - h)])
        y = np.concatenate([by, rng.uniform(0, w.nodes - 1, n - h)])
    else:
        x = rng.uniform(0, w.nodes - 1, n)
        y = rng.uniform(0, w.nodes - 1, n)
    vth = np.sqrt(T * Consts.qe / mass)
    v = rng.normal(0.0, vth, (3, n))
    x = np.minimum(x.astype(np.float32), np.nextafter(top, np.float32(0)))
    y = np.minimum(y.astype(np.float32), np.nextafter(top, np.float32(0)))
    return x, y, v[0].astype(np.float32), v[1].astype(np.float32), v[2].astype(np.float32)


def dirichlet(w: Workload):
    """All edge nodes Dirichlet; left column at left_V, corners grounded."""
    n = w.nodes
    mask = np.zeros((n, n), np.uint8)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    phi = np.zeros((n, n))
    phi[1:-1, 0] = w.left_V
    return mask.reshape(-1), phi.reshape(-1)


def cross_sections(energy=None):
    """The MCC workload's analytic tables on 1000 log-spaced energies (eV, m^2)."""
    E = log_grid() if energy is None else energy
    el = 1e-19 * (1.0 + E / 10.0) ** -0.5
    with np.errstate(divide="ignore", invalid="ignore"):
        exc = np.where(E > 11.5, 2e-21 * np.log(E / 11.5) / (E / 11.5), 0.0)
        ion = np.where(E > 15.8, 3e-20 * np.log(E / 15.8) / (E / 15.8), 0.0)
    cx = np.full_like(E, 5e-19)
    return E, el, exc, ion, cx


def mcc_tables(w: Workload, electrons=0, ions=1) -> MccTables:
    E, el, exc, ion, cx = cross_sections()
    t = MccTables(E, w.gas_density, w.gas_temperature, ION_MASS)
    t.add(electrons, ELASTIC, el).add(electrons, EXCITATION, exc, 11.5).add(electrons, IONIZATION, ion, 15.8)
    t.set_products(electrons, electrons, ions)
    t.add(ions, CHARGE_EXCHANGE, cx)
    return t
