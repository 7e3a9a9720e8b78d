"""Ensembles: members stepped together in one graph (pic_ens_step) against
twins stepped alone (pic_sim_step) from the same inputs.

The members differ in grid side, particle counts, tile, sort interval and
multigrid depth.  The deposit's global flush uses float atomics, so the two
runs differ in the last bits of rho; the comparison allows for that:
particle counts equal, phi within 1e-4 of its largest value (both solves
stop at a 1e-8 relative residual, possibly after different cycle counts),
and slot-by-slot positions
within 1e-3 cells on at least 99 % of the slots (this also requires every
member's cell sorts to have run at the same steps in both runs, since a sort
reorders the slots)."""
import numpy as np
import pytest
import torch

from pic_b200 import ensemble, workloads

pytestmark = pytest.mark.gpu

MEMBERS = [  # (side, n_e, n_i, tile, sort_interval, coarsest_max)
    (129, 30_000, 20_000, 16, 5, 9),
    (257, 60_000, 45_000, 8, 7, 17),
    (129, 12_000, 16_000, 8, 3, 9),
    (257, 25_000, 35_000, 16, 10, 9),
    (513, 50_000, 50_000, 16, 4, 33),
]


def _workloads():
    out = []
    rng = np.random.Generator(np.random.Philox(99))
    for i, (side, ne, ni, *_ ) in enumerate(MEMBERS):
        out.append(workloads.Workload(f"m{i}", side, ne, ni, Te=float(rng.uniform(1, 5)),
                                      left_V=float(rng.uniform(0, 200)), seed=500 + i))
    return out


def _make(w, cfg, push_kernel="ring"):
    _, _, _, tile, K, cmax = cfg
    sim = ensemble.member_simulation(w, tile=tile, sort_interval=K, coarsest_max=cmax, push_kernel=push_kernel)
    for s, a in enumerate(ensemble.member_arrays(w)):
        sim.load(s, *a)
    sim.init()
    return sim


def _state(sim):
    sim.sync()
    torch.cuda.synchronize()
    c = sim.counters()
    xs = [sim.species_arrays(s)[0][: c["count"][s]].cpu().numpy().copy() for s in range(2)]
    phi = sim.fields()[0].cpu().numpy().copy()
    return c, xs, phi


@pytest.mark.parametrize("structure", ["branches", "one_pass", "mixed_kernels"])
def test_ensemble_matches_members_stepped_alone(structure, steps=23):
    """branches (the default): every member's particle pass is its own launch in
    its branch; one_pass: every member on the ring pass and one particle pass
    spans all members; mixed_kernels: one member takes the per-warp pass, so
    the one pass does not apply and the branches run."""
    ws = _workloads()
    kinds = ["warp"] + ["ring"] * (len(MEMBERS) - 1) if structure == "mixed_kernels" else ["ring"] * len(MEMBERS)
    together = [_make(w, cfg, k) for w, cfg, k in zip(ws, MEMBERS, kinds)]
    alone = [_make(w, cfg, k) for w, cfg, k in zip(ws, MEMBERS, kinds)]
    ens = ensemble.Ensemble(together)
    assert not ens.fused_pass
    ens.fused_pass = structure != "branches"
    assert ens.fused_pass == (structure == "one_pass")
    ens.step(steps - 3)
    ens.step(3)  # a second launch of the same graph
    for sim in alone:
        sim.step(steps)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(together, alone)):
        ca, xa, pa = _state(a)
        cb, xb, pb = _state(b)
        assert ca["steps"] == cb["steps"] == steps, i
        assert ca["count"] == cb["count"], (i, ca["count"], cb["count"])
        scale = max(1.0, float(np.abs(pb).max()))
        assert np.abs(pa - pb).max() <= 1e-4 * scale, i
        for s in range(2):
            close = np.abs(xa[s] - xb[s]) <= 1e-3
            assert close.mean() >= 0.99, (i, s, close.mean())
    ens.close()
    for sim in together + alone:
        sim.close()


def test_ensemble_rejects_eager_members_and_duplicates():
    w = _workloads()[0]
    sim = ensemble.member_simulation(w, use_graph=False)
    from pic_b200 import _lib

    with pytest.raises(_lib.PicError):
        ensemble.Ensemble([sim])
    g = ensemble.member_simulation(w)
    with pytest.raises(_lib.PicError):
        ensemble.Ensemble([g, g])
    sim.close()
    g.close()


@pytest.mark.parametrize("one_pass", [True, False])
def test_ensemble_with_collisions_matches_members_stepped_alone(one_pass):
    """Members with null-collision MCC (the MCC workload's tables, a denser gas
    so that collisions and ionisation products occur every step), in the one
    particle pass over all members or in a pass per member, against the same
    members stepped alone.
    After two steps (one of them with collisions) the two agree to FP32
    rounding, with the same candidates and collisions.  Then
    the runs drift apart in the last bits (rho's global float atomics: the
    candidates' and products' deposits), and a particle that ends a step in
    another cell shifts the slots after the next sort, and with them the
    Philox streams of the candidates: after twelve steps collision, product and
    particle counts agree to within a few standard deviations, phi to 1e-3 of
    its largest value and the positions' quantiles to half a cell."""
    from pic_b200 import Consts
    from pic_b200.simulation import PICSimulation

    def make(i):
        w = workloads.scaled(workloads.MCC, nodes=129 if i == 0 else 257, n=40_000 + 10_000 * i, gas_density=3e22,
                             Te=8.0, seed=700 + i)
        mask, phi_bc = workloads.dirichlet(w)
        sp = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
              dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
        sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp, mask, phi_bc, tol=w.tol, max_cycles=50,
                            sort_interval=5, mcc=workloads.mcc_tables(w), seed=w.seed, use_graph=True)
        for s, a in enumerate(ensemble.member_arrays(w)):
            sim.load(s, *a)
        sim.init()
        return sim

    together = [make(i) for i in range(2)]
    alone = [make(i) for i in range(2)]
    ens = ensemble.Ensemble(together)
    ens.fused_pass = one_pass
    assert ens.fused_pass == one_pass
    # two steps (the second kicks and collides, no sort between them): the
    # same candidates and collisions, the particles that were there before
    # equal to FP32 rounding (the products' slots follow atomic order; the
    # charge tiles' flush adds floats in atomic order, so E, and the kick, may
    # differ in a last bit between any two runs)
    ens.step(2)
    for sim in alone:
        sim.step(2)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(together, alone)):
        ca, cb = a.counters(), b.counters()
        assert ca["collisions"] == cb["collisions"] and ca["born"] == cb["born"], i
        assert ca["count"] == cb["count"] and ca["absorbed"] == cb["absorbed"], i
        for s in range(2):
            n = ca["count"][s] - ca["born"][s]
            for k in range(5):
                ga = a.species_arrays(s)[k][:n].cpu().numpy()
                gb = b.species_arrays(s)[k][:n].cpu().numpy()
                scale = float(np.nanmax(np.abs(gb))) if np.isfinite(gb).any() else 0.0
                np.testing.assert_allclose(ga, gb, rtol=1e-6, atol=1e-6 * scale, equal_nan=True)
    ens.step(10)
    for sim in alone:
        sim.step(10)
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(together, alone)):
        ca, xa, pa = _state(a)
        cb, xb, pb = _state(b)
        assert sum(ca["collisions"][0]) > 0 and ca["born"][0] > 0, i
        for s in range(2):
            for k in range(4):
                a_, b_ = ca["collisions"][s][k], cb["collisions"][s][k]
                assert abs(a_ - b_) <= 3 * np.sqrt(b_) + 5, (i, s, k, a_, b_)
            assert abs(ca["born"][s] - cb["born"][s]) <= 3 * np.sqrt(cb["born"][s]) + 5, i
            assert abs(ca["count"][s] - cb["count"][s]) <= 3 * np.sqrt(cb["born"][s] + 1) + 5, i
        # collided particles that differ between the runs change phi by a few
        # particles' fields
        scale = max(1.0, float(np.abs(pb).max()))
        assert np.abs(pa - pb).max() <= 1e-3 * scale, i
        for s in range(2):
            # as distributions (a slot shift after a sort moves particles, not their
            # positions; a few dozen particles that differ move a quantile by a few
            # tenths of a cell at most)
            q = np.linspace(0.01, 0.99, 99)
            ga, gb = xa[s][np.isfinite(xa[s])], xb[s][np.isfinite(xb[s])]
            assert np.abs(np.quantile(ga, q) - np.quantile(gb, q)).max() <= 0.5, (i, s)
    ens.close()
    for sim in together + alone:
        sim.close()
