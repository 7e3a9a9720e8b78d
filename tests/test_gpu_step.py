"""The fused time step (PICSimulation) against the oracle and the drop-in operators.

Bit-exact: every particle pass given the same E (kick, drift, absorption),
the absorbed counts, E from phi, and the sort order.  Tolerances: phi
through the FP64 residual; the deposit per node within
2e-6 * sum|contrib| + k * 2^-20 * |scale| (k contributions; the fused pass
accumulates tile charge as fixed point with 2^-19 resolution per weight);
the FP32 trajectories against the FP64 reference arithmetic after 20 steps
(max |dx| <= 2e-3 cells, the FP32 grid-unit resolution times the step count).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle.fp64_step import fp64_reference_run
from pic_b200 import Consts, workloads
from pic_b200.simulation import PICSimulation

pytestmark = pytest.mark.gpu


def make_sim(w, sort_interval, mcc=None, cap_factor=2, seed=0, push_kernel="ring"):
    mask, phi_bc = workloads.dirichlet(w)
    sp_ = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=cap_factor * w.n_e),
           dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=cap_factor * w.n_i)]
    sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp_, mask, phi_bc, tol=w.tol, max_cycles=60,
                        sort_interval=sort_interval, mcc=mcc, seed=seed, push_kernel=push_kernel)
    rng = np.random.Generator(np.random.Philox(w.seed))
    arrays = [workloads.species_arrays(w, "e", rng), workloads.species_arrays(w, "i", rng)]
    for s, a in enumerate(arrays):
        sim.load(s, *a)
    return sim, arrays, mask, phi_bc


def host(sim, s):
    return [a.cpu().numpy().copy() for a in sim.species_arrays(s)]


def oracle_sort(arrs, w, tile=16):
    keys = O.sort_keys(arrs[0], arrs[1], w.nodes, w.nodes, tile)
    live = ~np.isnan(arrs[0])
    order = np.argsort(keys, kind="stable")[: int(live.sum())]
    return [a[order] for a in arrs]


def consts(w):
    kq_e = np.float32(-Consts.qe / Consts.me * w.dt)
    kq_i = np.float32(Consts.qe / workloads.ION_MASS * w.dt)
    return [kq_e, kq_i], np.float32(w.dt / w.dx)


def assert_bits(a, b):
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_array_equal(a[~np.isnan(a)].view(np.uint32), b[~np.isnan(b)].view(np.uint32))


@pytest.mark.parametrize("push_kernel", ["ring", "warp", "warp_agg", "pipe"])
@pytest.mark.parametrize("sort_interval", [0, 1])
def test_particle_passes_bit_exact(sort_interval, push_kernel):
    w = workloads.scaled(workloads.SMALL, n=30_000)
    sim, arrays, mask, _ = make_sim(w, sort_interval, push_kernel=push_kernel)
    kqs, dtdx = consts(w)
    m = w.nodes
    ref = [list(a) for a in arrays]
    if sort_interval:
        ref = [oracle_sort(a, w) for a in ref]
    # init: deposit, solve, E, half kick back
    rc = sim.init()
    phi, rho, Ex, Ey = (f.cpu().numpy().copy() for f in sim.fields())
    ex, ey = O.update_E_f32(phi, m, m, w.dx, w.dx)
    np.testing.assert_array_equal(Ex, ex)
    np.testing.assert_array_equal(Ey, ey)
    f = -rho.astype(np.float64) / Consts.eps0
    f[mask == 1] = 0
    assert np.sqrt(O.residual_f64(phi, f, mask, m, m, w.dx, w.dx) / np.sum(f * f)) < w.tol
    exact = np.zeros(m * m)
    absum = np.zeros(m * m)
    fixed = np.zeros(m * m)
    for s, a in enumerate(ref):
        scale = np.float32(sim.species[s]["charge"] * sim.species[s]["np2c"] / (w.dx * w.dx))
        O.deposit_f32(a[0], a[1], scale, m, m, exact, absum)
        fixed += O.deposit_counts(a[0], a[1], m, m) * 2.0**-20 * abs(float(scale))
    assert np.all(np.abs(rho - exact) <= 2e-6 * absum + fixed + 1e-30)
    for s, a in enumerate(ref):
        O.kick_f32(a[0], a[1], a[2], a[3], ex, ey, np.float32(np.float64(kqs[s]) * -0.5), m, m)
        got = host(sim, s)
        for k in range(4):
            assert_bits(got[k], a[k])
    # step 1: drift + absorb + deposit (the kick of init is already applied)
    sim.step(1)
    absorbed = [0, 0]
    for s in range(2):
        if sort_interval:
            ref[s] = oracle_sort(ref[s], w)
        absorbed[s] = O.drift_absorb_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], dtdx, dtdx, m, m)
        got = host(sim, s)
        assert_bits(got[0], ref[s][0])
        assert_bits(got[1], ref[s][1])
    assert sim.counters()["absorbed"] == absorbed
    _, _, Ex1, Ey1 = (f.cpu().numpy().copy() for f in sim.fields())
    # step 2: kick with E of step 1, drift, absorb
    sim.step(1)
    for s in range(2):
        if sort_interval:
            ref[s] = oracle_sort(ref[s], w)
        O.kick_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], Ex1, Ey1, kqs[s], m, m)
        O.drift_absorb_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], dtdx, dtdx, m, m)
        got = host(sim, s)
        for k in range(4):
            assert_bits(got[k], ref[s][k])
    assert rc in (0, 3)


def test_trajectories_against_fp64_reference():
    w = workloads.scaled(workloads.SMALL, n=20_000, left_V=20.0)
    steps = 20
    sim, arrays, _, _ = make_sim(w, 0)
    sim.init()
    sim.step(steps)
    sim.sync()
    ref = fp64_reference_run(w, arrays, steps, [-Consts.qe, Consts.qe], [Consts.me, workloads.ION_MASS]).P
    worst = 0.0
    for s in range(2):
        got = host(sim, s)
        # a particle within the FP32 error of a wall may be absorbed in one run only
        differ = np.isnan(got[0]) != np.isnan(ref[s][0])
        assert differ.sum() <= max(2, 1e-3 * len(differ))
        live = ~np.isnan(ref[s][0]) & ~np.isnan(got[0])
        worst = max(worst, float(np.max(np.abs(got[0][live] - ref[s][0][live] / w.dx))))
        worst = max(worst, float(np.max(np.abs(got[1][live] - ref[s][1][live] / w.dx))))
        vscale = np.abs(ref[s][2][live]).max()
        assert np.max(np.abs(got[2][live] - ref[s][2][live])) <= 1e-4 * vscale
    print(f"max |dx| after {steps} steps: {worst:.3e} cells")
    assert worst <= 2e-3


def test_fused_step_with_mcc_bookkeeping():
    w = workloads.scaled(workloads.MCC, nodes=129, n=200_000, gas_density=3e22)
    tables = workloads.mcc_tables(w)
    sim, _, _, _ = make_sim(w, 4, mcc=tables, seed=77)
    sim.init()
    sim.step(12)
    sim.sync()
    c = sim.counters()
    assert sum(c["collisions"][0]) > 0 and c["collisions"][1][0] > 0
    assert c["dropped_births"] == 0 and c["candidate_overflow"] == 0
    for s in range(2):
        live = int((~torch.isnan(sim.species_arrays(s)[0])).sum())
        assert live == w.n_e - c["absorbed"][s] + c["born"][s]
    assert 0 < c["born"][0] <= c["collisions"][0][2] and c["born"][1] <= c["collisions"][0][2]


@pytest.mark.parametrize("push_kernel", ["ring", "pipe"])
def test_fused_step_with_mcc_and_electrodes_bookkeeping(push_kernel):
    """Null-collision MCC in a dense gas with internal electrode lines: the
    collision candidates (finished after the pass) and their ionisation
    products drift through the same electrode test as every other particle.
    Every particle is accounted for: live = loaded - wall-absorbed -
    electrode-collected + born, per species, with collections among the
    candidates' drifts too."""
    w = workloads.scaled(workloads.MCC, nodes=129, n=150_000, gas_density=3e22, Te=20.0)
    m = w.nodes
    mask2 = np.zeros((m, m), np.uint8)
    mask2[0, :] = mask2[-1, :] = mask2[:, 0] = mask2[:, -1] = 1
    phi2 = np.zeros((m, m))
    xa, xb, top = (m - 1) // 4, 3 * (m - 1) // 4, (m - 1) // 2
    mask2[0:top + 1, xa] = 1
    mask2[0:top + 1, xb] = 1
    phi2[1:top + 1, xa] = -5.0
    phi2[1:top + 1, xb] = 5.0
    sp_ = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
           dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
    sim = PICSimulation(m, m, w.dx, w.dx, 1e-10, sp_, mask2.reshape(-1), phi2.reshape(-1), tol=w.tol,
                        max_cycles=60, sort_interval=4, mcc=workloads.mcc_tables(w), seed=91, use_graph=True,
                        push_kernel=push_kernel)
    rng = np.random.Generator(np.random.Philox(w.seed))
    for s, which in enumerate(("e", "i")):
        sim.load(s, *workloads.species_arrays(w, which, rng))
    sim.init()
    sim.step(10)
    sim.sync()
    c = sim.counters()
    assert sum(c["collisions"][0]) > 0 and c["born"][0] > 0
    assert c["electrode_absorbed"][0] > 0
    assert c["dropped_births"] == 0 and c["candidate_overflow"] == 0
    for s, n0 in enumerate((w.n_e, w.n_i)):
        live = int((~torch.isnan(sim.species_arrays(s)[0])).sum())
        assert live == n0 - c["absorbed"][s] - c["electrode_absorbed"][s] + c["born"][s]
    sim.close()


@pytest.mark.parametrize("push_kernel", ["ring", "warp", "warp_agg", "pipe"])
def test_internal_electrodes_collect_bit_exact(push_kernel):
    """Cathode and anode lines inside the domain (the equipotentials of the
    reference's test.inp, at x = L/4 and 3L/4 from the bottom wall to half
    height): drifts that cross them are collected, bit-exact against the
    oracle's FP32 crossing test, and counted apart from the wall absorption."""
    w = workloads.scaled(workloads.SMALL, n=60_000, Te=20.0)
    m = w.nodes
    mask2 = np.zeros((m, m), np.uint8)
    mask2[0, :] = mask2[-1, :] = mask2[:, 0] = mask2[:, -1] = 1
    phi2 = np.zeros((m, m))
    xa, xb, top = (m - 1) // 4, 3 * (m - 1) // 4, (m - 1) // 2
    mask2[0:top + 1, xa] = 1
    mask2[0:top + 1, xb] = 1
    phi2[1:top + 1, xa] = -5.0
    phi2[1:top + 1, xb] = 5.0
    mask, phi_bc = mask2.reshape(-1), phi2.reshape(-1)
    sp_ = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=2 * w.n_e),
           dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i), capacity=2 * w.n_i)]
    # dt 1e-10 s: 20 eV electrons move ~0.3 cells a step, many cross the lines
    dt = 1e-10
    sim = PICSimulation(m, m, w.dx, w.dx, dt, sp_, mask, phi_bc, tol=w.tol, max_cycles=60, sort_interval=0,
                        push_kernel=push_kernel)
    rng = np.random.Generator(np.random.Philox(w.seed))
    ref = [list(workloads.species_arrays(w, "e", rng)), list(workloads.species_arrays(w, "i", rng))]
    for s, a in enumerate(ref):
        sim.load(s, *a)
    vb, hb = O.electrode_bits(mask, m, m)
    kqs = [np.float32(-Consts.qe / Consts.me * dt), np.float32(Consts.qe / workloads.ION_MASS * dt)]
    dtdx = np.float32(dt / w.dx)
    sim.init()
    _, _, ex, ey = (f.cpu().numpy().copy() for f in sim.fields())
    for s, a in enumerate(ref):
        O.kick_f32(a[0], a[1], a[2], a[3], ex, ey, np.float32(np.float64(kqs[s]) * -0.5), m, m)
    walls, collected = [0, 0], [0, 0]
    for step in range(2):
        sim.step(1)
        for s in range(2):
            if step:
                O.kick_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], ex, ey, kqs[s], m, m)
            a, c = O.drift_absorb_electrodes_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], dtdx, dtdx, m, m, vb,
                                                  hb)
            walls[s] += a
            collected[s] += c
            got = host(sim, s)
            for k in range(4):
                assert_bits(got[k], ref[s][k])
        _, _, ex, ey = (f.cpu().numpy().copy() for f in sim.fields())
    cnt = sim.counters()
    assert cnt["absorbed"] == walls
    assert cnt["electrode_absorbed"] == collected
    assert collected[0] > 100  # the electrons do reach the electrodes


def test_diagnostics_match_numpy():
    """pic_sim_diagnostics against numpy FP64 sums over the same arrays and fields."""
    w = workloads.scaled(workloads.SMALL, n=40_000)
    sim, arrays, mask, _ = make_sim(w, 20)
    sim.init()
    sim.step(5)
    sim.sync()
    d = sim.diagnostics()
    m = w.nodes
    for s in range(2):
        x, y, vx, vy, vz = (a.astype(np.float64) for a in host(sim, s))
        live = ~np.isnan(x)
        sp = sim.species[s]
        assert d["live"][s] == int(live.sum())
        v2 = vx[live] ** 2 + vy[live] ** 2 + vz[live] ** 2
        assert d["kinetic"][s] == pytest.approx(0.5 * sp["mass"] * sp["np2c"] * v2.sum(), rel=1e-12)
        mom = [sp["mass"] * sp["np2c"] * c[live].sum() for c in (vx, vy, vz)]
        np.testing.assert_allclose(d["momentum"][s], mom, rtol=1e-9, atol=1e-40)
    phi, rho, ex, ey = (f.cpu().numpy().astype(np.float64) for f in sim.fields())
    dx = dy = w.dx
    assert d["field_energy"] == pytest.approx(0.5 * np.sum(rho * phi) * dx * dy, rel=1e-12)
    E = [ex.reshape(m, m), ey.reshape(m, m)]
    flux = (E[0][:, -1].sum() - E[0][:, 0].sum()) * dy + (E[1][-1, :].sum() - E[1][0, :].sum()) * dx
    assert d["gauss_flux"] == pytest.approx(flux, rel=1e-10, abs=1e-12 * np.abs(E[0]).max() * m * dx)
    assert d["gauss_charge"] == pytest.approx(rho.sum() * dx * dy / Consts.eps0, rel=1e-12)
    dex = np.empty((m, m))
    dey = np.empty((m, m))
    dex[:, 1:-1] = (E[0][:, 2:] - E[0][:, :-2]) / (2 * dx)
    dex[:, 0] = (E[0][:, 1] - E[0][:, 0]) / dx
    dex[:, -1] = (E[0][:, -1] - E[0][:, -2]) / dx
    dey[1:-1, :] = (E[1][2:, :] - E[1][:-2, :]) / (2 * dy)
    dey[0, :] = (E[1][1, :] - E[1][0, :]) / dy
    dey[-1, :] = (E[1][-1, :] - E[1][-2, :]) / dy
    err = np.sqrt(np.sum((dex + dey - rho.reshape(m, m) / Consts.eps0) ** 2))
    assert d["div_error_l2"] == pytest.approx(err, rel=1e-9)


def test_particle_buffer_matches_numpy():
    """The headless particle vertex buffer (the renderer's VBO, src/Render.py:544-571):
    live particles in species order, normalised positions and species types,
    bit-exact against numpy with the same FP64 arithmetic, after absorption has
    left dead slots; a buffer that is too small raises."""
    w = workloads.scaled(workloads.SMALL, n=50_000, left_V=80.0)
    sim, _, _, _ = make_sim(w, 0)
    sim.init()
    sim.step(30)
    sim.sync()
    assert sum(sim.counters()["absorbed"]) > 0
    xr, yr = (0.001, 0.011), (-0.002, 0.0128)
    got = sim.particle_buffer(xr, yr).cpu().numpy()
    want = []
    for s in range(2):
        x, y = (t.cpu().numpy().astype(np.float64) for t in sim.species_arrays(s)[:2])
        live = np.isfinite(x)
        xm, ym = x[live] * w.dx, y[live] * w.dx
        want.append(np.stack([2.0 * (xm - xr[0]) / (xr[1] - xr[0]) - 1.0, 2.0 * (ym - yr[0]) / (yr[1] - yr[0]) - 1.0,
                              np.full(xm.size, s + 1.0)], 1).astype(np.float32))
    want = np.concatenate(want)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    small = torch.empty((10, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(Exception):
        sim.particle_buffer(xr, yr, out=small)
    sim.close()
