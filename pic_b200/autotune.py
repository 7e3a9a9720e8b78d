"""Autotuner for the fused step: tile size, sort interval and multigrid depth.

The reference has no tuner (its launch shapes are fixed in the RawKernel
calls).  The choices here trade against each other on the GPU:
  tile           cells per side of a push work tile: larger tiles stage more
                 E field per unit and flush more charge per unit
  sort_interval  steps between cell sorts: a sort costs about two particle
                 passes, while the particles drift out of their tiles between
                 sorts (untiled particles gather and deposit in global memory)
  coarsest_max   largest side of the coarsest multigrid level (V-cycle depth)
  omega          over-relaxation of the red-black smoother (cycles per solve)
  mg_launch      multigrid launch mode: the graph loop of tiled kernels, or
                 one thread-block cluster per solve (faster on small grids)

Candidates are timed on the GPU (CUDA events over graph-launched steps) by a
coordinate descent from a default, one parameter at a time; results are kept
per workload shape (grid side, particle count rounded to a power of two) and
may be cached in a JSON file.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import asdict, dataclass
from typing import Callable

SPACE = {"tile": (8, 16, 32), "sort_interval": (10, 20, 40, 80), "coarsest_max": (5, 9, 17),
         "omega": (1.0, 1.15, 1.3), "mg_launch": ("graph", "cluster")}
DEFAULT = {"tile": 16, "sort_interval": 20, "coarsest_max": 9, "omega": 1.15, "mg_launch": "graph"}
ORDER = ("tile", "sort_interval", "coarsest_max", "omega", "mg_launch")


@dataclass
class Choice:
    tile: int
    sort_interval: int
    coarsest_max: int
    ns_per_particle_step: float  # measured cost of the chosen configuration
    omega: float = DEFAULT["omega"]
    mg_launch: str = DEFAULT["mg_launch"]

    def config(self) -> dict:
        return {"tile": self.tile, "sort_interval": self.sort_interval, "coarsest_max": self.coarsest_max,
                "omega": self.omega, "mg_launch": self.mg_launch}


def shape_key(nodes: int, particles: int) -> str:
    """Grid side and the particle count rounded to the nearest power of two."""
    return f"{int(nodes)}:{2 ** int(round(math.log2(max(1, particles))))}"


def coordinate_descent(measure: Callable[[dict], float], space=SPACE, start=DEFAULT, order=ORDER):
    """Minimise measure(config) one parameter at a time (each parameter once,
    in `order`, the others held at their best values so far), starting from
    `start` (or a parameter's first candidate where `start` is not one).  Returns
    (best config, its cost, every measured (config, cost))."""
    order = [k for k in order if k in space]
    best = {k: (start[k] if start[k] in space[k] else space[k][0]) for k in order}
    seen = {}

    def cost(cfg):
        k = tuple(sorted(cfg.items()))
        if k not in seen:
            seen[k] = float(measure(dict(cfg)))
        return seen[k]

    best_cost = cost(best)
    for p in order:
        for v in space[p]:
            cand = dict(best, **{p: v})
            c = cost(cand)
            if c < best_cost:
                best, best_cost = cand, c
    return best, best_cost, [(dict(k), v) for k, v in seen.items()]


class Autotuner:
    """Tunes and remembers the configuration of each workload shape."""

    def __init__(self, cache_path: str | None = None, space=SPACE, steps=80, warmup=4):
        self.cache_path = cache_path
        self.space = space
        self.steps = int(steps)
        self.warmup = int(warmup)
        self.cache: dict[str, Choice] = {}
        self.measurements = 0
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = {k: Choice(**v) for k, v in json.load(f).items()}

    def save(self):
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump({k: asdict(v) for k, v in self.cache.items()}, f, indent=1, sort_keys=True)

    def measure(self, make_sim: Callable[[dict], object], cfg: dict) -> float:
        """ns per particle-step of a simulation built by make_sim(cfg) (loaded and
        initialised), over `steps` graph-launched steps after `warmup` steps."""
        import torch

        sim = make_sim(cfg)
        try:
            sim.step(self.warmup)
            torch.cuda.synchronize()
            n0 = sum(sim.counters()["count"])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            sim.step(self.steps)
            e1.record()
            torch.cuda.synchronize()
            n1 = sum(sim.counters()["count"])
            self.measurements += 1
            return e0.elapsed_time(e1) * 1e6 / (0.5 * (n0 + n1) * self.steps)
        finally:
            sim.close()

    def tune(self, key: str, make_sim: Callable[[dict], object]) -> Choice:
        if key in self.cache:
            return self.cache[key]
        best, cost, _ = coordinate_descent(lambda cfg: self.measure(make_sim, cfg), self.space)
        ch = Choice(best["tile"], best["sort_interval"], best["coarsest_max"], cost,
                    best.get("omega", DEFAULT["omega"]), best.get("mg_launch", DEFAULT["mg_launch"]))
        self.cache[key] = ch
        self.save()
        return ch

    def tune_workload(self, w) -> Choice:
        """Tunes a collisionless ensemble member's shape (pic_b200.ensemble)."""
        from . import ensemble

        def make(cfg):
            sim = ensemble.member_simulation(w, **cfg)
            for s, a in enumerate(ensemble.member_arrays(w)):
                sim.load(s, *a)
            sim.init()
            return sim

        return self.tune(shape_key(w.nodes, w.n_e + w.n_i), make)

    def tune_ensemble(self, workloads) -> list[Choice]:
        """One choice per member; each distinct shape is measured once, on the
        first member of that shape."""
        return [self.tune_workload(w) for w in workloads]
