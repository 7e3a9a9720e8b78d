"""Grid2D: drop-in for src/Grid.py:198-376, Cartesian or r-z.

Node arrays live on the GPU as torch tensors (torch is used only for device
memory).  ``rho`` is float32 charge density (C/m^3), ``phi`` FP64 potential,
``E`` float32 (2, m*n) field, ``b`` FP64 Poisson right-hand side.  Index
layout as the reference: idx = j*m + i with m nodes in x (src/Grid.py:140).

cylindrical=True is the axisymmetric r-z grid (src/Grid.py:5-93): x (m
nodes) is the axis z, y (n nodes, rows) the radius, row 0 on the axis.  The
deposit is divided by the node volumes of the linear weighting (so a uniform
load gives a uniform density), and E_r vanishes on the axis.  The reference
divides by ring volumes indexed along the wrong axis and does not zero E_r
there (src/Grid.py:66-93).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

DEVICE = "cuda"


class Grid2D:
    """Grid2D(m, n, X, Y) -- m, n are NODE counts; dx = X/(m-1) (src/Grid.py:199-228)."""

    def __init__(self, m, n, X, Y, cylindrical=False):
        self.cylindrical = bool(cylindrical)
        self.m = int(m)
        self.n = int(n)
        self.X = float(X)
        self.Y = float(Y)
        self.dx = self.X / (self.m - 1)
        self.dy = self.Y / (self.n - 1)
        self.gridshape = (self.m, self.n)
        self.node_count = self.m * self.n
        self.cell_size = (self.dx, self.dy)
        self.cell_count = (self.m - 1) * (self.n - 1)
        self.domain = (self.X, self.Y)
        G = self.node_count
        self.rho = torch.zeros(G, dtype=torch.float32, device=DEVICE)
        self.b = torch.zeros(G, dtype=torch.float64, device=DEVICE)
        self.phi = torch.zeros(G, dtype=torch.float64, device=DEVICE)
        self.E = torch.zeros((2, G), dtype=torch.float32, device=DEVICE)

    def update_E(self):
        """E = -grad(phi) (src/Grid.py:232-243); r-z: E_r = 0 on the axis."""
        _lib.call("pic_update_E_rz" if self.cylindrical else "pic_update_E", _lib.ptr(self.phi), _lib.ptr(self.E[0]),
                  _lib.ptr(self.E[1]), self.m, self.n, self.dx, self.dy, _lib.stream_ptr())

    def update_density(self, particles):
        """CIC charge deposit of every species, rho in C/m^3 (src/Grid.py:246-294);
        r-z: divided by the node volumes (pic_rz_density)."""
        self.rho.zero_()
        for s in particles.species:
            if s.n == 0:
                continue
            scale = s.charge * particles.species_np2c(s) / (self.dx * self.dy)
            _lib.call("pic_deposit", _lib.ptr(s.x), _lib.ptr(s.y), s.n, scale, _lib.ptr(self.rho), self.m, self.n,
                      _lib.stream_ptr())
        if self.cylindrical:
            _lib.call("pic_rz_density", _lib.ptr(self.rho), self.m, self.n, self.dy, _lib.stream_ptr())

    def update_J(self, particles):
        pass

    def minmax_phi(self):
        return torch.min(self.phi), torch.max(self.phi)

    def minmax_rho(self):
        return torch.min(self.rho), torch.max(self.rho)

    def save_to_txt(self, filename, fields=None, header=None):
        """Columns x, y, fields... in '%.2e' (the format of src/Grid.py:306-375)."""
        if fields is None:
            fields = {"rho": self.rho, "phi": self.phi, "E_x": self.E[0], "E_y": self.E[1]}
        j, i = np.divmod(np.arange(self.node_count), self.m)
        cols = [i * self.dx, j * self.dy]
        names = []
        for name, f in fields.items():
            names.append(name)
            cols.append(f.detach().cpu().numpy() if isinstance(f, torch.Tensor) else np.asarray(f))
        if header is None:
            header = "x y " + " ".join(names)
        np.savetxt(filename, np.column_stack(cols), header=header, comments="# ", fmt="%.2e")
