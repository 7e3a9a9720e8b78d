"""Boundaries: drop-in for src/Boundaries.py:4-58.

Rasterises Equipotential segments ``((j1, k1, j2, k2), V)`` into Dirichlet
node indices and values (``conditions``) and the node mask ``bc_lookup``
(1 = Dirichlet).  The segment walk steps both coordinates by the sign of
their difference until the end point, as the reference does
(src/Boundaries.py:36-52).  Later segments overwrite earlier values on
shared nodes.  The cell wall map (src/Boundaries.py:61-99) feeds only the
reference's unused collision tracer and is not built.
"""
from __future__ import annotations

import numpy as np
import torch

DEVICE = "cuda"


def boundary_array(bounds, gridshape):
    m = gridshape[0]
    idx, val = [], []
    for (m1, n1, m2, n2), V in bounds:
        m1, n1, m2, n2 = int(m1), int(n1), int(m2), int(n2)
        dm, dn = int(np.sign(m2 - m1)), int(np.sign(n2 - n1))
        x, y = m1, n1
        while True:
            idx.append(y * m + x)
            val.append(float(V))
            if x == m2 and y == n2:
                break
            x += dm
            y += dn
    return np.asarray(idx, dtype=np.int32), np.asarray(val, dtype=np.float64)


class Boundaries:
    def __init__(self, bounds, grid):
        idx, val = boundary_array(bounds, grid.gridshape)
        self.conditions_host = (idx, val)
        self.conditions = (torch.as_tensor(idx, device=DEVICE), torch.as_tensor(val, device=DEVICE))
        lookup = np.zeros(grid.m * grid.n, dtype=np.int32)
        lookup[idx] = 1
        self.bc_lookup_host = lookup
        self.bc_lookup = torch.as_tensor(lookup, device=DEVICE)
        # last write wins on shared nodes, as cupy fancy assignment does
        phi_bc = np.zeros(grid.m * grid.n)
        phi_bc[idx] = val
        self.phi_bc_host = phi_bc
        self.walls = None
        self.wall_lookup = None
        self.bound_tuple = [tuple(int(v) for v in seg[0]) for seg in bounds]


def walls_box(grid, left=0.0, bottom=0.0, right=0.0, top=0.0):
    """Four wall segments of a rectangular domain.  Corners belong to the
    bottom and top walls (written last), so grounded horizontal walls win
    over a biased left/right wall at the corners."""
    m, n = grid.m, grid.n
    return [((0, 0, 0, n - 1), left), ((m - 1, 0, m - 1, n - 1), right), ((0, 0, m - 1, 0), bottom),
            ((0, n - 1, m - 1, n - 1), top)]
