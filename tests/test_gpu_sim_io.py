"""Reading the particles back (pic_sim_read_particles) and the cell sort on
demand (pic_sim_sort) of the fused simulation."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from pic_b200 import Consts, _lib, workloads
from pic_b200.simulation import PICSimulation

pytestmark = pytest.mark.gpu

TILE = 16


def make(w, sort_interval=5, mcc=None):
    mask, phi_bc = workloads.dirichlet(w)
    sp = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
          dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
    sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp, mask, phi_bc, tol=w.tol, max_cycles=60,
                        sort_interval=sort_interval, mcc=mcc, seed=3, use_graph=True, tile=TILE)
    rng = np.random.Generator(np.random.Philox(w.seed))
    for s, which in enumerate(("e", "i")):
        sim.load(s, *workloads.species_arrays(w, which, rng))
    sim.init()
    return sim


def host_arrays(sim, s):
    return np.stack([t.cpu().numpy() for t in sim.species_arrays(s)])


def test_read_particles_matches_the_device_arrays():
    """The rows x, y, vx, vy, vz of the slots in use, dead ones (NaN) included,
    bit for bit; twice in a row into the same buffer; too small a buffer is
    refused with PIC_ERR_OUT_OF_CAPACITY."""
    w = workloads.scaled(workloads.MCC, nodes=129, n=80_000, gas_density=3e22)
    sim = make(w, mcc=workloads.mcc_tables(w))
    sim.step(7)
    sim.sync()
    for s in range(2):
        want = host_arrays(sim, s)
        out = torch.empty(5 * 2 * w.n_e, dtype=torch.float32).pin_memory()
        for _ in range(2):
            got = sim.read_particles(s, out)
            torch.cuda.current_stream().synchronize()
            assert got.shape == want.shape
            np.testing.assert_array_equal(got.numpy().view(np.uint32), want.view(np.uint32))
        small = torch.empty(5 * want.shape[1] - 1, dtype=torch.float32).pin_memory()
        with pytest.raises(_lib.PicError) as e:
            sim.read_particles(s, small)
        assert e.value.code == _lib.PIC_ERR_OUT_OF_CAPACITY
    sim.close()


def test_sort_on_demand_orders_by_tile_and_keeps_every_particle():
    """pic_sim_sort between steps: the live particles, and only they, in
    stable tile-major cell order (the dead slots dropped); then the steps go on
    with the particles conserved."""
    w = workloads.scaled(workloads.SMALL, n=60_000, Te=20.0)
    sim = make(w, sort_interval=1000)
    sim.step(6)
    sim.sync()
    before = [host_arrays(sim, s) for s in range(2)]
    sim.sort()
    torch.cuda.synchronize()
    c = sim.counters()
    m = w.nodes
    for s in range(2):
        a = before[s]
        live = np.isfinite(a[0])
        keys = O.sort_keys(a[0], a[1], m, m, TILE)
        order = np.argsort(keys, kind="stable")[: int(live.sum())]
        got = host_arrays(sim, s)
        assert c["count"][s] == int(live.sum()) == got.shape[1]
        np.testing.assert_array_equal(got.view(np.uint32), a[:, order].view(np.uint32))
    absorbed0 = c["absorbed"]
    sim.step(4)
    sim.sync()
    c = sim.counters()
    for s in range(2):
        live = int(np.isfinite(host_arrays(sim, s)[0]).sum())
        assert live == before[s].shape[1] - (c["absorbed"][s] - absorbed0[s]) - int((~np.isfinite(before[s][0])).sum())
    sim.close()


def test_read_particles_of_an_empty_species():
    """A species with no particles loaded reads back as zero columns, and the
    simulation steps with it."""
    w = workloads.scaled(workloads.SMALL, n=20_000)
    mask, phi_bc = workloads.dirichlet(w)
    sp = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
          dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
    sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp, mask, phi_bc, tol=w.tol, max_cycles=60,
                        sort_interval=5, seed=3, use_graph=True)
    rng = np.random.Generator(np.random.Philox(w.seed))
    sim.load(0, *workloads.species_arrays(w, "e", rng))
    empty = np.zeros(0, np.float32)
    sim.load(1, empty, empty, empty, empty, empty)
    sim.init()
    sim.step(6)
    sim.sync()
    out = torch.empty(5 * 16, dtype=torch.float32).pin_memory()
    got = sim.read_particles(1, out)
    assert tuple(got.shape) == (5, 0)
    assert sim.counters()["count"][1] == 0
    sim.close()
