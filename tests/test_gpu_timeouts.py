"""Failure detection: the bounded device waits give up, report PIC_ERR_TIMEOUT
and leave the context and the objects usable.

No GPU is made to fault or hang: the wait limits are lowered so that a wait
that would have succeeded gives up instead, the kernels return normally, and
the host reads the error flag.
  * The persistent multigrid solve (one cooperative launch, grid barriers
    between its phases): with a barrier limit of one poll the blocks that
    arrive before the last one give up; every later barrier then gives up too,
    so every block returns.  The same solver then converges with the default
    limit.
  * The fused particle pass (chunks, or E tiles, streamed into shared memory
    by bulk copies completed on mbarriers): with a limit of zero polls every
    block gives up at its first wait, after waiting (with the default limit)
    for the copies in flight.  The simulation then steps normally once
    reloaded.
"""
import numpy as np
import pytest
import torch

from pic_b200 import Consts, _lib, workloads
from pic_b200.multigrid import MultigridSolver
from pic_b200.simulation import PICSimulation

pytestmark = pytest.mark.gpu


def test_persistent_solve_barrier_timeout_is_reported():
    n = 257
    w = workloads.scaled(workloads.SMALL, nodes=n)
    mask, _ = workloads.dirichlet(w)
    rng = np.random.default_rng(3)
    f = torch.as_tensor(rng.normal(size=n * n) * 1e9, device="cuda")
    f[torch.as_tensor(mask, device="cuda") == 1] = 0
    mg = MultigridSolver(mask, n, n, w.dx, launch="persistent")
    mg.set_wait_limit(1)
    phi = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.PicError) as e:
        mg.solve(phi, f, tol=1e-10, max_cycles=30)
    assert e.value.code == _lib.PIC_ERR_TIMEOUT
    assert "grid barrier" in str(e.value)
    torch.cuda.synchronize()  # the context is intact
    mg.set_wait_limit(-1)
    phi.zero_()
    _, (cycles, rel) = mg.solve(phi, f, tol=1e-10, max_cycles=30, raise_on_fail=True)
    assert rel < 1e-10 and cycles > 0


@pytest.mark.parametrize("push_kernel", ["ring", "warp", "pipe"])
def test_particle_pass_wait_timeout_is_reported(push_kernel):
    w = workloads.scaled(workloads.SMALL, n=50_000)
    mask, phi_bc = workloads.dirichlet(w)
    sp = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=w.n_e),
          dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=w.n_i)]
    sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp, mask, phi_bc, tol=w.tol, sort_interval=10,
                        use_graph=True, push_kernel=push_kernel)
    rng = np.random.Generator(np.random.Philox(4))
    arrays = [workloads.species_arrays(w, "e", rng), workloads.species_arrays(w, "i", rng)]
    for s, a in enumerate(arrays):
        sim.load(s, *a)
    sim.init()
    sim.step(3)  # the captured step exists; the new limit makes it re-captured
    sim.set_wait_limit(0)
    sim.step(2)
    with pytest.raises(_lib.PicError) as e:
        sim.counters()
    assert e.value.code == _lib.PIC_ERR_TIMEOUT
    torch.cuda.synchronize()
    sim.counters()  # the flag was cleared with the report
    sim.set_wait_limit(-1)
    for s, a in enumerate(arrays):
        sim.load(s, *a)
    sim.init()
    c0 = sim.counters()
    sim.step(3)
    c1 = sim.counters()
    live = sum(int(torch.isfinite(sim.species_arrays(s)[0]).sum()) for s in range(2))
    assert live == w.n_e + w.n_i - (sum(c1["absorbed"]) - sum(c0["absorbed"]))
    assert c1["last_rel_res"] < w.tol
    sim.close()
