"""ConfigParser: reader of the reference's .inp input files (src/ConfigParser.py)
and a builder of the fused simulation from them.

The file is a sequence of named blocks, `Name { key = value ... }` (the name
on the line of the brace or the line before it), with `//` comments.  The
reader returns the reference's dictionary (src/ConfigParser.py:206-230):
system, variables, boundaries [((j1, k1, j2, k2), C)], species, grid,
control, loads, plus `mcc` (the MCC blocks).  Values are evaluated as
arithmetic over numbers and the Variables block's names, in file order;
values that are not such an expression (names like `electrons`, `gmres`)
stay strings.  Unlike the reference, which substitutes variable names as
substrings and calls eval (so that a variable `X` would also rewrite `Jmax`),
expressions are parsed and only numbers, names, + - * / // % **, unary
signs and abs/int/float/pow/min/max/sqrt calls are evaluated.

`build_simulation` turns a configuration into a PICSimulation: Grid J x K
nodes over [x1s, x1f] x [x2s, x2f], the Equipotential segments as Dirichlet
nodes (src/Boundaries.py:36-52; the grid edges are always Dirichlet, except
the axis row x2 = x2s of a cylindrical grid), the Species, uniform Load boxes
with Maxwellian velocities, and Control.dt.  Grid.Cylindrical = 1 builds the
axisymmetric r-z simulation (x1 axial, x2 radial), with Load radii uniform
in volume.
"""
from __future__ import annotations

import ast
import math
import operator

import numpy as np

from . import Consts
from .Boundaries import boundary_array

_BINARY = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
           ast.FloorDiv: operator.floordiv, ast.Mod: operator.mod, ast.Pow: operator.pow}
_CALLS = {"abs": abs, "int": int, "float": float, "pow": pow, "min": min, "max": max, "sqrt": math.sqrt}


def evaluate(expr, names):
    """The value of an arithmetic expression over numbers and `names`, as a
    float; the stripped text itself when it is not one."""
    text = str(expr).strip()

    def ev(n):
        if isinstance(n, ast.Expression):
            return ev(n.body)
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)) and not isinstance(n.value, bool):
            return n.value
        if isinstance(n, ast.Name):
            v = names.get(n.id)
            if isinstance(v, (int, float)) and not isinstance(v, bool):
                return v
            raise KeyError(n.id)
        if isinstance(n, ast.BinOp) and type(n.op) in _BINARY:
            return _BINARY[type(n.op)](ev(n.left), ev(n.right))
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, (ast.UAdd, ast.USub)):
            v = ev(n.operand)
            return v if isinstance(n.op, ast.UAdd) else -v
        if (isinstance(n, ast.Call) and isinstance(n.func, ast.Name) and n.func.id in _CALLS and not n.keywords):
            return _CALLS[n.func.id](*[ev(a) for a in n.args])
        raise ValueError(ast.dump(n))

    try:
        return float(ev(ast.parse(text, mode="eval")))
    except (SyntaxError, KeyError, ValueError, TypeError, ZeroDivisionError, OverflowError):
        return text


def _system_value(text):
    t = text.strip()
    if t.lower() in ("true", "false"):
        return t.lower() == "true"
    for conv in (int, float):
        try:
            return conv(t)
        except ValueError:
            pass
    return t


class ConfigParser:
    """parse_file(path) -> the configuration dictionary (see the module docstring)."""

    def __init__(self):
        self.variables = {}
        self.system = {}
        self.grid = {}
        self.control = {}
        self.equipotentials = []
        self.species = []
        self.loads = []
        self.mcc = []

    # ---- blocks ----
    @staticmethod
    def _pairs(lines):
        for line in lines:
            if "=" in line:
                key, value = line.split("=", 1)
                yield key.strip(), value.strip()

    def _eval_block(self, lines):
        return {k: evaluate(v, self.variables) for k, v in self._pairs(lines)}

    def _block(self, name, lines):
        if name == "Variables":
            for k, v in self._pairs(lines):
                self.variables[k] = evaluate(v, self.variables)
        elif name == "System":
            self.system.update({k: _system_value(v) for k, v in self._pairs(lines)})
        elif name == "Grid":
            self.grid.update(self._eval_block(lines))
        elif name == "Control":
            for k, v in self._pairs(lines):
                self.control[k] = v.strip("'\"") if v[:1] in "'\"" else evaluate(v, self.variables)
        elif name == "Equipotential":
            b = self._eval_block(lines)
            if all(k in b for k in ("j1", "k1", "j2", "k2", "C")):
                self.equipotentials.append(((b["j1"], b["k1"], b["j2"], b["k2"]), b["C"]))
        elif name == "Species":
            s = self._eval_block(lines)
            if not all(k in s for k in ("name", "m", "q", "collisionModel")):
                raise ValueError(f"incomplete Species block: {sorted(s)}")
            self.species.append(s)
        elif name == "Load":
            self.loads.append(self._eval_block(lines))
        elif name == "MCC":
            self.mcc.append(self._eval_block(lines))

    def parse_text(self, text):
        name, body, previous = None, [], ""
        for raw in text.split("\n"):
            line = raw.split("//", 1)[0].strip()
            if not line:
                continue
            if line.endswith("{"):
                head = line[:-1].strip()
                name, body = (head if head else previous), []
            elif line == "}":
                if name is not None:
                    self._block(name, body)
                name, body = None, []
            elif name is not None:
                body.append(line)
            else:
                previous = line
        return self.config()

    def parse_file(self, path):
        with open(path) as f:
            return self.parse_text(f.read())

    def config(self):
        return {"system": dict(self.system), "variables": dict(self.variables), "boundaries": list(self.equipotentials),
                "species": [dict(s) for s in self.species], "grid": dict(self.grid), "control": dict(self.control),
                "loads": [dict(l) for l in self.loads], "mcc": [dict(m) for m in self.mcc]}


def multigrid_compatible(nodes, coarsest=33):
    """Node counts the multigrid hierarchy accepts: (nodes - 1) halves down to at most `coarsest` nodes."""
    n = int(nodes)
    while n > coarsest:
        if (n - 1) % 2:
            return False
        n = (n - 1) // 2 + 1
    return n >= 3


def build_simulation(cfg, seed=0, temperature_eV=None, np2c=None, tol=1e-8, sort_interval=20, use_graph=True,
                     cartesian=False, **kw):
    """A PICSimulation of the configuration with its Load blocks loaded.

    Grid.Cylindrical = 1 gives the r-z simulation unless cartesian=True.
    Load velocities are Maxwellian at Load.temperature (eV), else at
    `temperature_eV`, else zero; np2c per Load block (Load.np2c), else
    `np2c`, else the reference's 1 (src/Particles.py:326)."""
    from .simulation import PICSimulation

    grid = cfg["grid"]
    rz = bool(int(grid.get("Cylindrical", 0))) and not cartesian
    m, n = int(grid["J"]), int(grid["K"])
    for name, v in (("J", m), ("K", n)):
        if not multigrid_compatible(v):
            raise ValueError(f"Grid.{name} = {v} nodes: the multigrid needs 2^k * c + 1 nodes (c <= 32), "
                             f"e.g. 129 or 257")
    X = float(grid.get("x1f", 1.0)) - float(grid.get("x1s", 0.0))
    Y = float(grid.get("x2f", 1.0)) - float(grid.get("x2s", 0.0))
    dx, dy = X / (m - 1), Y / (n - 1)
    x0, y0 = float(grid.get("x1s", 0.0)), float(grid.get("x2s", 0.0))
    dt = float(cfg["control"]["dt"])
    idx, val = boundary_array(cfg["boundaries"], (m, n)) if cfg["boundaries"] else (np.zeros(0, int), np.zeros(0))
    mask = np.zeros(m * n, np.uint8)
    phi_bc = np.zeros(m * n)
    mask[idx] = 1
    phi_bc[idx] = val
    edge = np.zeros((n, m), bool)
    edge[-1, :] = edge[:, 0] = edge[:, -1] = True
    if not rz:
        edge[0, :] = True
    mask[edge.reshape(-1)] = 1

    names = [str(s["name"]) for s in cfg["species"]]
    counts = {nm: 0 for nm in names}
    for load in cfg["loads"]:
        counts[str(load["speciesName"])] += int(load["n"])
    max_total = int(cfg["system"].get("MAX_PARTICLES", 0))
    species = []
    for s in cfg["species"]:
        nm = str(s["name"])
        cap = max(counts[nm] + counts[nm] // 4 + 64, max_total // max(1, len(names)))
        p2c = next((float(l["np2c"]) for l in cfg["loads"] if str(l["speciesName"]) == nm and "np2c" in l),
                   1.0 if np2c is None else float(np2c))
        species.append(dict(name=nm, charge=float(s["q"]), mass=float(s["m"]), np2c=p2c, capacity=cap))
    sim = PICSimulation(m, n, dx, dy, dt, species, mask, phi_bc, tol=tol, sort_interval=sort_interval, seed=seed,
                        use_graph=use_graph, geometry="rz" if rz else "cartesian", **kw)
    rng = np.random.Generator(np.random.Philox(seed))
    per = {nm: [] for nm in names}
    for load in cfg["loads"]:
        nm = str(load["speciesName"])
        s = species[names.index(nm)]
        k = int(load["n"])
        x = (rng.uniform(float(load["x1MinMKS"]), float(load["x1MaxMKS"]), k) - x0) / dx
        if rz:
            # radii uniform in volume: r^2 uniform between the bounds (measured from the axis x2s)
            r1, r2 = float(load["x2MinMKS"]) - y0, float(load["x2MaxMKS"]) - y0
            y = np.sqrt(rng.uniform(r1 * r1, r2 * r2, k)) / dy
        else:
            y = (rng.uniform(float(load["x2MinMKS"]), float(load["x2MaxMKS"]), k) - y0) / dy
        T = load.get("temperature", temperature_eV)
        vth = math.sqrt(float(T) * Consts.qe / s["mass"]) if T is not None else 0.0
        v = rng.normal(0.0, vth, (3, k)) if vth > 0 else np.zeros((3, k))
        per[nm].append(np.vstack([x, y, v]).astype(np.float32))
    for s_i, nm in enumerate(names):
        if per[nm]:
            a = np.hstack(per[nm])
            top_x, top_y = np.float32(m - 1), np.float32(n - 1)
            a[0] = np.minimum(a[0], np.nextafter(top_x, np.float32(0)))
            a[1] = np.minimum(a[1], np.nextafter(top_y, np.float32(0)))
            sim.load(s_i, a[0], a[1], a[2], a[3], a[4])
    return sim


def save_fields(sim, filename, header=None):
    """Grid fields of a PICSimulation in the reference's text format
    (src/Grid.py:306-375): columns x, y, rho, phi, E_x, E_y, '%.2e'."""
    phi, rho, ex, ey = (f.detach().cpu().numpy() for f in sim.fields())
    j, i = np.divmod(np.arange(sim.nx * sim.ny), sim.nx)
    cols = [i * sim.dx, j * sim.dy, rho, phi, ex, ey]
    np.savetxt(filename, np.column_stack(cols), header=header or "x y rho phi E_x E_y", comments="# ", fmt="%.2e")
