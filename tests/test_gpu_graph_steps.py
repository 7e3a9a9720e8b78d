"""The captured step against the same steps launched kernel by kernel.

With use_graph the step runs as CUDA graphs (one per step; its side branch
prepares the next step, with that step's cell sort when one is due).  Both
paths must keep the same sort schedule, random streams (MCC
candidates and outcomes keyed by step and slot), step counter and solver
cycle counts, so the particle arrays line up slot by slot.  Equality is to
FP32 round-off: collisions and particles outside their staged tile deposit
through global float atomics, whose order differs between runs.  The gas
has no ionisation here: ionisation products take their slots in the order
the collisions finish, which differs between any two runs.
"""
import numpy as np
import pytest
import torch

from pic_b200 import Consts, workloads
from pic_b200.MCC import CHARGE_EXCHANGE, ELASTIC, EXCITATION, MccTables
from pic_b200.simulation import PICSimulation

pytestmark = pytest.mark.gpu


def tables(w):
    E, el, exc, _, cx = workloads.cross_sections()
    t = MccTables(E, w.gas_density, w.gas_temperature, workloads.ION_MASS)
    return t.add(0, ELASTIC, el).add(0, EXCITATION, exc, 11.5).add(1, CHARGE_EXCHANGE, cx)


def build(w, use_graph, sort_interval):
    mask, phi_bc = workloads.dirichlet(w)
    sp_ = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
           dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
    sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp_, mask, phi_bc, tol=w.tol, max_cycles=60,
                        sort_interval=sort_interval, mcc=tables(w), seed=11, use_graph=use_graph)
    rng = np.random.Generator(np.random.Philox(w.seed))
    for s, which in enumerate("ei"):
        sim.load(s, *workloads.species_arrays(w, which, rng))
    sim.init()
    return sim


@pytest.mark.parametrize("chunks", [[27], [3, 9, 1, 14]])
def test_graph_steps_match_eager_steps(chunks):
    # sort every 10 steps; 27 steps in all, so that the last captured step
    # has not sorted ahead for the next one (the order would differ then)
    w = workloads.scaled(workloads.MCC, nodes=129, n=60_000, gas_density=3e22, left_V=40.0)
    eager, graph = build(w, False, 10), build(w, True, 10)
    for n in chunks:
        eager.step(n)
        graph.step(n)
    for sim in (eager, graph):
        sim.sync()
    ce, cg = eager.counters(), graph.counters()
    assert cg["steps"] == ce["steps"] == sum(chunks)
    for key in ("absorbed", "collisions", "count", "null_candidates"):
        assert cg[key] == ce[key], key
    assert ce["collisions"][0][0] > 0 and ce["collisions"][0][1] > 0 and ce["collisions"][1][0] > 0
    assert cg["last_cycles"] == ce["last_cycles"]
    for s in range(2):
        a = [t.cpu().numpy() for t in eager.species_arrays(s)]
        b = [t.cpu().numpy() for t in graph.species_arrays(s)]
        np.testing.assert_array_equal(np.isnan(a[0]), np.isnan(b[0]))
        live = ~np.isnan(a[0])
        for k in range(5):
            # positions to 1e-4 cells, velocities to 1e-5 of the largest
            atol = 1e-4 if k < 2 else 1e-5 * np.abs(a[k][live]).max()
            np.testing.assert_allclose(b[k][live], a[k][live], rtol=0, atol=atol, err_msg=f"species {s} {k}")
    phi_e, phi_g = eager.fields()[0].cpu().numpy(), graph.fields()[0].cpu().numpy()
    np.testing.assert_allclose(phi_g, phi_e, rtol=0, atol=1e-6 * np.abs(phi_e).max())
    for sim in (eager, graph):
        sim.close()


@pytest.mark.parametrize("use_graph", [False, True])
def test_min_cycles_run_before_the_first_test(use_graph):
    # tol 1e-4 from the extrapolated potential: one V-cycle suffices (the
    # first cuts the residual of a PIC step about 500-fold); min_cycles=3
    # runs three whatever the residual, and ends closer to the solution
    w = workloads.scaled(workloads.SMALL, n=20_000)
    mask, phi_bc = workloads.dirichlet(w)
    got = {}
    for mc in (0, 3):
        sp_ = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
               dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
        sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp_, mask, phi_bc, tol=1e-4, max_cycles=60,
                            sort_interval=0, use_graph=use_graph, min_cycles=mc)
        rng = np.random.Generator(np.random.Philox(w.seed))
        for s, which in enumerate("ei"):
            sim.load(s, *workloads.species_arrays(w, which, rng))
        sim.init()
        sim.step(4)
        sim.sync()
        c = sim.counters()
        got[mc] = (c["last_cycles"], c["last_rel_res"])
        sim.close()
    assert got[0][0] < 3 and got[0][1] < 1e-4, got
    assert got[3][0] == 3 and got[3][1] < got[0][1], got
