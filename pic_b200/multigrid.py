"""MultigridSolver: drop-in for src/multigrid.py:277-455.

The solve runs on the GPU through pic_mg_* (pic_b200/csrc/multigrid.cu):
FP32 (or FP64) V-cycles with red-black Gauss-Seidel smoothing inside an FP64
iterative-refinement loop.  Deviations from the reference, each needed for
the solver to converge (the reference's own wiring cannot run):
  * the mask means 1 = Dirichlet on every level (the reference mixes
    1 = Dirichlet and 1 = interior between its kernels, src/multigrid.py:33,143);
  * `rho` is the right-hand side f of lap(phi) = f with no extra h^2 factor;
  * `levels` is advisory: the grid is coarsened down to <= 9 nodes and solved
    exactly there;
  * `omega` is the smoother's over-relaxation; the reference's 1.9 is
    accepted, but a red-black smoother inside a V-cycle converges fastest
    near 1.15 (measured on 513^2: 5 V(2,2) cycles to 1e-8 instead of 6 at 1.0).

geometry="rz" solves the axisymmetric Poisson equation (the reference's
cylindrical Laplacian, src/Solvers.py:100-166, which its multigrid never
used): x is the axis, y the radius with row 0 on the axis; the axis row is
free (symmetry) rather than a boundary.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib


class MultigridSolver:
    def __init__(self, bc_mask, nx, ny, h, levels=4, omega=1.15, precision="mixed", pre_sweeps=2, post_sweeps=2,
                 hy=None, launch="graph", geometry="cartesian", coarse_fp32=False):
        self.nx, self.ny = int(nx), int(ny)
        self.h = float(h)
        self.hy = float(h if hy is None else hy)
        self.levels = levels
        self.omega = float(omega)
        mask = np.ascontiguousarray(torch.as_tensor(bc_mask).cpu().numpy().reshape(-1) != 0, dtype=np.uint8)
        if mask.size != self.nx * self.ny:
            raise ValueError("bc_mask must have nx*ny entries")
        self.precision = precision
        self.geometry = geometry
        opts = _lib.MgOptions(_lib.PIC_MG_MIXED if precision == "mixed" else _lib.PIC_MG_FP64, pre_sweeps,
                              post_sweeps, self.omega, 9, _lib.MG_LAUNCH_MODES[launch], _lib.GEOMETRIES[geometry],
                              int(bool(coarse_fp32)))
        self._h = C.c_void_p()
        _lib.call("pic_mg_create", self.nx, self.ny, self.h, self.hy, mask.ctypes.data, C.byref(opts),
                  C.byref(self._h))
        self.last_info = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize()
                _lib.load().pic_mg_destroy(h)
            except Exception:
                pass
            self._h = None

    def effective_launch(self) -> str:
        """The launch mode solves use ("cluster" falls back to "graph" where it does not apply)."""
        m = C.c_int()
        _lib.call("pic_mg_effective_launch_mode", self._h, C.byref(m))
        return {v: k for k, v in _lib.MG_LAUNCH_MODES.items()}[m.value]

    def set_wait_limit(self, polls=-1):
        """Polls a grid barrier of the persistent solve makes before the solve
        gives up with PIC_ERR_TIMEOUT (raised as PicError); -1 restores the default."""
        _lib.call("pic_mg_set_wait_limit", self._h, int(polls))

    def solve(self, phi, rho, tol=1e-5, smooth_iter=5, solve_iter=20, max_cycles=50, raise_on_fail=False):
        """Solve lap(phi) = rho in place; returns (phi, (cycles, rel_res)) like src/multigrid.py:445-455.
        smooth_iter/solve_iter are accepted for signature compatibility."""
        assert phi.dtype == torch.float64 and rho.dtype == torch.float64 and phi.is_cuda and rho.is_cuda
        info = _lib.MgInfo()
        rc = _lib.load().pic_mg_solve(self._h, _lib.ptr(phi), _lib.ptr(rho), float(tol), int(max_cycles),
                                      C.byref(info), _lib.stream_ptr())
        if rc not in (_lib.PIC_OK, _lib.PIC_ERR_NOT_CONVERGED) or (raise_on_fail and rc != _lib.PIC_OK):
            _lib.check(rc, "pic_mg_solve")
        self.last_info = info
        return phi, (info.cycles, info.rel_res)


class ConjugateGradientSolver:
    """The 'cg' / 'gmres' branches of the reference's Solver (src/Solvers.py:245-258,
    cupyx cg and gmres): flexible preconditioned conjugate gradients on the GPU
    (pic_cg_*), FP64, each iteration preconditioned by one V-cycle of
    `precond` (a MultigridSolver of the same grid and mask) when given.  The
    Cartesian 5-point system is symmetric, so this is also the solution GMRES
    converges to."""

    def __init__(self, bc_mask, nx, ny, h, hy=None, precond: MultigridSolver | None = None):
        self.nx, self.ny = int(nx), int(ny)
        mask = np.ascontiguousarray(torch.as_tensor(bc_mask).cpu().numpy().reshape(-1) != 0, dtype=np.uint8)
        self.precond = precond
        self._h = C.c_void_p()
        _lib.call("pic_cg_create", self.nx, self.ny, float(h), float(h if hy is None else hy), mask.ctypes.data,
                  precond._h if precond is not None else None, C.byref(self._h))
        self.last_info = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().pic_cg_destroy(h)
            except Exception:
                pass
            self._h = None

    def solve(self, phi, rho, tol=1e-5, max_iter=200, raise_on_fail=False):
        """Solve lap(phi) = rho in place; returns (phi, (iterations, rel_res))."""
        assert phi.dtype == torch.float64 and rho.dtype == torch.float64 and phi.is_cuda and rho.is_cuda
        info = _lib.MgInfo()
        rc = _lib.load().pic_cg_solve(self._h, _lib.ptr(phi), _lib.ptr(rho), float(tol), int(max_iter),
                                      C.byref(info), _lib.stream_ptr())
        if rc not in (_lib.PIC_OK, _lib.PIC_ERR_NOT_CONVERGED) or (raise_on_fail and rc != _lib.PIC_OK):
            _lib.check(rc, "pic_cg_solve")
        self.last_info = info
        return phi, (info.cycles, info.rel_res)
