"""Build recipe for oracle/_ref/libpicref.so (test infrastructure only).

The reference (dimad285/PIC) is Python + CuPy: its GPU kernels are CUDA-C
source strings passed to ``cupy.RawKernel``.  This recipe reads those strings
straight out of the reference's own files with ``ast`` (nothing is copied into
this repository), puts ``cuda_shim.h`` in front of them and ``ref_driver.cpp``
behind them, and pipes the result into g++.  The only output is the shared
library in ``oracle/_ref/``; no source file is written.

Kernels taken, by the name given to RawKernel:
    src/Grid.py        update_density_direct_cartesian (:96-154), update_E (:157-196)
    src/Particles.py   update_particle_velocity_direct (:117-180), update_r_kernel (:251-264),
                       update_particle_axis (:267-280), sort_particles_sparse (:595-617)
    src/multigrid.py   gauss_seidel_red_black (:13-49), residual_kernel (:52-81),
                       restriction_kernel (:84-134), prolong_kernel (:138-196),
                       coarsen_bc_mask (:235-274)
    src/MCC.py         compute_speeds_and_energies (:7-30), interpolate_cross_sections (:32-83)
``#include`` lines inside the strings are dropped (the shim provides what they
would).  Usage:  python oracle/ref_build.py [--reference DIR] [--out DIR]  (or set PIC_REFERENCE_DIR)
"""
from __future__ import annotations

import argparse
import ast
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference tree: --reference DIR, else $PIC_REFERENCE_DIR, else the
# container's read-only checkout
DEFAULT_REFERENCE = os.environ.get("PIC_REFERENCE_DIR", "/root/reference")

WANTED = {
    "src/Grid.py": ["update_density_direct_cartesian", "update_E"],
    "src/Particles.py": [
        "update_particle_velocity_direct",
        "update_r_kernel",
        "update_particle_axis",
        "sort_particles_sparse",
    ],
    "src/multigrid.py": [
        "gauss_seidel_red_black",
        "residual_kernel",
        "restriction_kernel",
        "prolong_kernel",
        "coarsen_bc_mask",
    ],
    "src/MCC.py": ["compute_speeds_and_energies", "interpolate_cross_sections"],
}


def _raw_kernels(path: str) -> dict[str, str]:
    """Map kernel name -> CUDA-C source for every cp.RawKernel(src, name) call in a file."""
    tree = ast.parse(open(path, encoding="utf-8").read(), filename=path)
    found: dict[str, str] = {}
    for node in ast.walk(tree):
        if not isinstance(node, ast.Call):
            continue
        fn = node.func
        if not (isinstance(fn, ast.Attribute) and fn.attr == "RawKernel"):
            continue
        if len(node.args) < 2:
            continue
        src, name = node.args[0], node.args[1]
        if isinstance(src, ast.Constant) and isinstance(name, ast.Constant):
            found[str(name.value)] = str(src.value)
    return found


def kernel_sources(reference: str) -> str:
    parts = []
    for rel, names in WANTED.items():
        kernels = _raw_kernels(os.path.join(reference, rel))
        for name in names:
            if name not in kernels:
                raise RuntimeError(f"kernel {name!r} not found in {rel}")
            body = "\n".join(
                line for line in kernels[name].splitlines() if not line.lstrip().startswith("#include")
            )
            parts.append(f"// ---- {rel}: {name}\n{body}\n")
    return "\n".join(parts)


def build(reference: str = DEFAULT_REFERENCE, out_dir: str | None = None, quiet: bool = False) -> str:
    out_dir = out_dir or os.path.join(HERE, "_ref")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libpicref.so")
    unit = '#include "cuda_shim.h"\n' + kernel_sources(reference) + '\n#include "ref_driver.cpp"\n'
    cmd = [
        "g++", "-std=c++20", "-O3", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
        "-w", "-I", HERE, "-x", "c++", "-", "-o", out,
    ]
    subprocess.run(cmd, input=unit.encode(), check=True)
    if not quiet:
        print(f"built {out}")
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if not os.path.isdir(a.reference):
        print(f"reference tree not found at {a.reference}; nothing to build", file=sys.stderr)
        return 1
    build(a.reference, a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
