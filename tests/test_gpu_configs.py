"""Parity at the stated workloads, at their full sizes and step counts.

small (129^2 nodes, 1e5 + 1e5 particles, Te 2 eV, Ti 0.03 eV, grounded
walls, multigrid to 1e-8, 100 steps, collisionless) through PICSimulation's
captured step, two ways:
  * every one of the 100 particle passes bit-exact against the FP32 oracle
    driven by the build's own E (kick, drift, absorption, sort order), the
    absorbed counts per pass exact, E from phi bit-exact, phi through its
    FP64 residual and rho within the deposit tolerance, every step;
  * against the reference's step in FP64 (oracle/fp64_step.py): rho, phi and E
    at the start (same positions) and after 100 steps, and the trajectories
    after 100 steps, within the FP32 tolerances below.

mcc (513^2 nodes, 4M + 4M particles, left wall 100 V, argon-like gas with
elastic, excitation, ionisation and charge exchange) at full size: the first
two steps of the captured step (the second one kicks and collides) against
the oracle's FP32 restatement and its replay of the same Philox counters for
the null-collision candidates (k_mcc_bits) and the collisions (k_collide):
candidate and per-process collision counts and absorbed counts exact, the
particles that did not collide bit-exact, the collided ones and the
ionisation products within 2e-6 of the speed (cosf, sinf and logf may differ
from the C library in the last bit), rho, phi and E as above.

Reference step restated: src/simulation.py:622-660.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle.fp64_step import fp64_reference_run
from pic_b200 import Consts, workloads
from pic_b200.MCC import MccOperator
from pic_b200.simulation import PICSimulation

pytestmark = pytest.mark.gpu

CHARGES = [-Consts.qe, Consts.qe]
MASSES = [Consts.me, workloads.ION_MASS]
TILE = 16


def build(w, sort_interval, mcc=None, seed=0, cap_factor=2):
    mask, phi_bc = workloads.dirichlet(w)
    sp_ = [dict(name="e", charge=CHARGES[0], mass=MASSES[0], np2c=w.np2c(w.n_e), capacity=cap_factor * w.n_e),
           dict(name="i", charge=CHARGES[1], mass=MASSES[1], np2c=w.np2c(w.n_i), capacity=cap_factor * w.n_i)]
    sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, sp_, mask, phi_bc, tol=w.tol, max_cycles=60,
                        sort_interval=sort_interval, mcc=mcc, seed=seed, use_graph=True, tile=TILE)
    rng = np.random.Generator(np.random.Philox(w.seed))
    arrays = [workloads.species_arrays(w, "e", rng), workloads.species_arrays(w, "i", rng)]
    for s, a in enumerate(arrays):
        sim.load(s, *a)
    return sim, arrays, mask, phi_bc


def host(sim, s):
    return [a.cpu().numpy().copy() for a in sim.species_arrays(s)]


def fields(sim):
    return [f.cpu().numpy().copy() for f in sim.fields()]


def oracle_sort(arrs, m):
    keys = O.sort_keys(arrs[0], arrs[1], m, m, TILE)
    live = ~np.isnan(arrs[0])
    order = np.argsort(keys, kind="stable")[: int(live.sum())]
    return [a[order] for a in arrs]


def assert_bits(got, want, what):
    assert got.shape == want.shape, what
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want), err_msg=what)
    live = ~np.isnan(want)
    np.testing.assert_array_equal(got[live].view(np.uint32), want[live].view(np.uint32), err_msg=what)


def scales(sim, w):
    return [np.float32(sim.species[s]["charge"] * sim.species[s]["np2c"] / (w.dx * w.dx)) for s in range(2)]


def check_fields(sim, w, mask, ref, what):
    """E bit-exact from phi; phi's recomputed FP64 residual below tol; rho
    within 2e-6 * sum|contrib| + count * 2^-20 * |scale| of the exact sum of the
    FP32 contributions of the oracle's particles (the fused pass accumulates
    tile charge as 2^-19 fixed point)."""
    m = w.nodes
    phi, rho, Ex, Ey = fields(sim)
    ex, ey = O.update_E_f32(phi, m, m, w.dx, w.dx)
    np.testing.assert_array_equal(Ex, ex, err_msg=f"{what}: Ex")
    np.testing.assert_array_equal(Ey, ey, err_msg=f"{what}: Ey")
    f = -rho.astype(np.float64) / Consts.eps0
    f[mask == 1] = 0
    rel = np.sqrt(O.residual_f64(phi, f, mask, m, m, w.dx, w.dx) / np.sum(f * f))
    assert rel < w.tol, f"{what}: residual {rel}"
    exact, absum, fixed = np.zeros(m * m), np.zeros(m * m), np.zeros(m * m)
    for s, a in enumerate(ref):
        sc = scales(sim, w)[s]
        live = ~np.isnan(a[0])
        O.deposit_f32(a[0][live], a[1][live], sc, m, m, exact, absum)
        fixed += O.deposit_counts(a[0], a[1], m, m) * 2.0**-20 * abs(float(sc))
    bad = np.abs(rho - exact) > 2e-6 * absum + fixed + 1e-30
    assert not bad.any(), f"{what}: rho off at {np.flatnonzero(bad)[:5]}"
    return phi, rho, Ex, Ey



def field_error(fp, phi, rho, Ex, Ey):
    """Max-norm errors of the build's rho, phi and E against the FP64 run, each
    relative to the FP64 field's largest magnitude."""
    ex, ey = fp.E
    return {"rho": float(np.abs(rho - fp.rho).max() / np.abs(fp.rho).max()),
            "phi": float(np.abs(phi - fp.phi).max() / max(np.abs(fp.phi).max(), 1e-300)),
            "E": float(max(np.abs(Ex - ex).max(), np.abs(Ey - ey).max()) / max(np.abs(ex).max(), np.abs(ey).max()))}


def test_small_workload_100_steps_against_oracle_and_fp64():
    w = workloads.SMALL
    assert (w.nodes, w.n_e, w.n_i, w.tol, w.steps, w.left_V) == (129, 100_000, 100_000, 1e-8, 100, 0.0)
    interval = 20
    m = w.nodes
    sim, arrays, mask, _ = build(w, interval)
    # vz takes no part in a collisionless Cartesian step: it carries each
    # particle's loaded slot, so the sort permutation is checked bit for bit and
    # the build's slots map back to the FP64 run's
    tagged = [list(a) for a in arrays]
    for s in range(2):
        tagged[s][4] = np.arange(tagged[s][0].size, dtype=np.float32)
        sim.load(s, *tagged[s])
    kq = [np.float32(CHARGES[s] / MASSES[s] * w.dt) for s in range(2)]
    dtdx = np.float32(w.dt / w.dx)
    ref = [oracle_sort([a.copy() for a in sp], m) for sp in tagged]  # init sorts
    assert sim.init() == 0
    phi0, rho0, Ex0, Ey0 = check_fields(sim, w, mask, ref, "init")
    for s in range(2):
        O.kick_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], Ex0, Ey0, np.float32(np.float64(kq[s]) * -0.5), m, m)
    fp = fp64_reference_run(w, arrays, 0, CHARGES, MASSES)  # the FP64 step on the same particles
    errors = {"init": field_error(fp, phi0, rho0, Ex0, Ey0)}
    E_prev = (Ex0, Ey0)
    absorbed = [0, 0]
    presorted = False
    for i in range(w.steps):
        if i % interval == 0 and not presorted:
            ref = [oracle_sort(a, m) for a in ref]
        presorted = False
        assert sim.step(1) == 0
        for s in range(2):
            if i > 0:
                O.kick_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], E_prev[0], E_prev[1], kq[s], m, m)
            absorbed[s] += O.drift_absorb_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], dtdx, dtdx, m, m)
        if i > 0 and (i + 1) % interval == 0:
            # a captured step sorts the particles for the next step beside its field solve
            ref = [oracle_sort(a, m) for a in ref]
            presorted = True
        assert sim.counters()["absorbed"] == absorbed, f"step {i + 1}"
        for s in range(2):
            got = host(sim, s)
            for k in range(5):
                assert_bits(got[k], ref[s][k], f"step {i + 1} species {s} array {k}")
        _, _, Ex, Ey = check_fields(sim, w, mask, ref, f"step {i + 1}")
        E_prev = (Ex, Ey)
    assert sum(absorbed) > 0
    # against the FP64 step after 100 steps (sync applies the build's pending kick)
    sim.sync()
    for _ in range(w.steps):
        fp.step()
    phi, rho, Ex, Ey = fields(sim)
    errors["final"] = field_error(fp, phi, rho, Ex, Ey)
    worst, vworst = 0.0, 0.0
    for s in range(2):
        got = host(sim, s)
        slot = got[4].astype(np.int64)
        P = [a[slot] for a in fp.P[s]]
        live = ~np.isnan(got[0]) & ~np.isnan(P[0])
        worst = max(worst, float(np.max(np.abs(got[0][live] - P[0][live] / w.dx))),
                    float(np.max(np.abs(got[1][live] - P[1][live] / w.dx))))
        vs = max(np.abs(P[2][live]).max(), np.abs(P[3][live]).max())
        vworst = max(vworst, float(max(np.abs(got[2][live] - P[2][live]).max(),
                                       np.abs(got[3][live] - P[3][live]).max())) / vs)
    differ = sum(abs(a - b) for a, b in zip(fp.absorbed, absorbed))
    print(f"small workload, 100 steps: max |dx| {worst:.3e} cells, max |dv| / max |v| {vworst:.3e}, "
          f"absorbed {absorbed} (FP64 {fp.absorbed}), field errors {errors}")
    # a particle within the FP32 rounding of a wall may be absorbed in one run only
    # measured on a B200: max |dx| 3.8e-4 cells, |dv| / max |v| 9.3e-7, absorbed
    # counts equal; rho, phi, E 1.8e-6, 3.6e-7, 2.1e-6 at the start and 3.5e-4,
    # 1.4e-5, 4.6e-5 after 100 steps (the trajectories' FP32 drift, seen
    # through the deposit)
    assert differ <= 4
    assert worst <= 2e-3
    assert vworst <= 1e-5
    e0, e1 = errors["init"], errors["final"]
    assert e0["rho"] <= 1e-5 and e0["phi"] <= 2e-6 and e0["E"] <= 1e-5
    assert e1["rho"] <= 2e-3 and e1["phi"] <= 1e-4 and e1["E"] <= 3e-4
    sim.close()


def oracle_mcc_species(tables, dt, s):
    """The oracle's view of species s's collision tables, with the sim's nu'."""
    op = MccOperator(tables, MASSES, dt)
    nu, _, inv = op.query(s)
    procs = tables.species[s]
    return O.mcc_species(tables.energy, [p[2] for p in procs], [p[0] for p in procs], [p[1] for p in procs],
                         tables.gas_density, MASSES[s], tables.gas_mass, tables.gas_temperature, nu, inv, s)


def test_mcc_workload_full_size_step_against_oracle():
    w = workloads.MCC
    assert (w.nodes, w.n_e, w.n_i, w.left_V, w.gas_density) == (513, 4_000_000, 4_000_000, 100.0, 1e21)
    m = w.nodes
    seed = 0x5EED_0001
    tables = workloads.mcc_tables(w)
    interval = 80
    sim, arrays, mask, _ = build(w, interval, mcc=tables, seed=seed, cap_factor=1.25)
    kq = [np.float32(CHARGES[s] / MASSES[s] * w.dt) for s in range(2)]
    dtdx = np.float32(w.dt / w.dx)
    ref = [oracle_sort([a.copy() for a in sp], m) for sp in arrays]  # init and step 1 sort (idempotent)
    assert sim.init() == 0
    _, _, Ex0, Ey0 = check_fields(sim, w, mask, ref, "init")
    for s in range(2):
        O.kick_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], Ex0, Ey0, np.float32(np.float64(kq[s]) * -0.5), m, m)
    # step 1: drift, absorb, deposit (no kick or collisions: the half kick is init's)
    assert sim.step(1) == 0
    absorbed = [O.drift_absorb_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], dtdx, dtdx, m, m) for s in range(2)]
    assert sim.counters()["absorbed"] == absorbed
    for s in range(2):
        got = host(sim, s)
        for k in range(5):
            assert_bits(got[k], ref[s][k], f"step 1 species {s} array {k}")
    _, _, Ex1, Ey1 = check_fields(sim, w, mask, ref, "step 1")
    n_before = [ref[s][0].size for s in range(2)]
    # step 2 (pass counter 2): kick, null-collision candidates, collisions, drift, absorb, deposit
    assert sim.step(1) == 0
    step = 2
    counts = np.zeros((2, 4), np.int64)
    cands = [0, 0]
    collided = [np.zeros(n_before[s], bool) for s in range(2)]
    births = [[], []]  # per species: (x, y, vx, vy, vz) rows before their drift
    for s in range(2):
        a = ref[s]
        O.kick_f32(a[0], a[1], a[2], a[3], Ex1, Ey1, kq[s], m, m)
        S, keep = oracle_mcc_species(tables, w.dt, s)
        mark = O.mcc_candidates(S, n_before[s], step, seed)
        mark[np.isnan(a[0])] = 0
        cands[s] = int(mark.sum())
        born_e, born_i = tables.products.get(s, (-1, -1))
        for i in np.flatnonzero(mark):
            v = [a[2][i], a[3][i], a[4][i]]
            proc, be, bi = O.mcc_collide(S, int(i), step, seed, v)
            if proc < 0:
                continue
            counts[s, proc] += 1
            collided[s][i] = True
            a[2][i], a[3][i], a[4][i] = v
            if tables.species[s][proc][0] == workloads.IONIZATION:
                births[born_e].append((a[0][i], a[1][i], *be))
                births[born_i].append((a[0][i], a[1][i], *bi))
        absorbed[s] += O.drift_absorb_f32(a[0], a[1], a[2], a[3], dtdx, dtdx, m, m)
        del keep
    c = sim.counters()
    assert c["null_candidates"] == cands
    np.testing.assert_array_equal(np.asarray(c["collisions"])[:, :4], counts)
    # measured: about 3200 elastic electron collisions and a dozen ion charge
    # exchanges in the step; excitation and ionisation (thresholds 11.5 and
    # 15.8 eV) are rare at 2 eV
    assert counts[0, 0] > 1000 and counts[1, 0] > 0
    # births: drifted with their own velocity; those that leave the domain are never stored
    born = []
    for s in range(2):
        b = np.asarray(births[s], np.float32).reshape(-1, 5).T.copy()
        b = [b[k].copy() for k in range(5)]
        O.drift_absorb_f32(b[0], b[1], b[2], b[3], dtdx, dtdx, m, m)
        keep_b = ~np.isnan(b[0])
        born.append([arr[keep_b] for arr in b])
    assert c["born"] == [born[0][0].size, born[1][0].size]
    assert c["absorbed"] == absorbed
    for s in range(2):
        got = host(sim, s)
        a = ref[s]
        n = n_before[s]
        assert got[0].size == n + born[s][0].size
        for k in range(5):
            g = got[k][:n]
            assert_bits(g[~collided[s]], a[k][~collided[s]], f"step 2 species {s} array {k} (not collided)")
        speed = np.sqrt(sum(a[k][collided[s]].astype(np.float64) ** 2 for k in (2, 3, 4)))
        for k in (2, 3, 4):
            assert np.all(np.abs(got[k][:n][collided[s]] - a[k][collided[s]]) <= 2e-6 * speed + 1e-3)
        for k in (0, 1):
            # a collided particle may also leave the domain (NaN in both)
            g, r = got[k][:n][collided[s]], a[k][collided[s]]
            np.testing.assert_array_equal(np.isnan(g), np.isnan(r))
            ok = ~np.isnan(r)
            assert np.all(np.abs(g[ok] - r[ok]) <= 2e-6 * speed[ok] * dtdx + 1e-4)
        # the products, as multisets per component (their slots follow atomic order)
        for k in range(5):
            g, r = np.sort(got[k][n:]), np.sort(born[s][k])
            tol = 1e-4 if k < 2 else 2e-6 * (np.abs(r).max() if r.size else 0.0) + 1e-3
            assert np.all(np.abs(g - r) <= tol), f"species {s} products array {k}"
    full = [[np.concatenate([ref[s][k], born[s][k]]) for k in range(5)] for s in range(2)]
    check_fields_loose_collided(sim, w, mask, full, collided, n_before)
    sim.close()


def check_fields_loose_collided(sim, w, mask, full, collided, n_before):
    """check_fields after a step with collisions: the deposit of the collided
    particles and of the products (whose positions agree to FP32 rounding, not
    bit for bit) is compared with the build's own positions for them."""
    fixed = []
    for s in range(2):
        got = host(sim, s)
        a = [arr.copy() for arr in full[s]]
        n = n_before[s]
        idx = np.flatnonzero(collided[s])
        for k in (0, 1):
            a[k][idx] = got[k][idx]
            a[k][n:] = got[k][n:]
        fixed.append(a)
    check_fields(sim, w, mask, fixed, "step 2")


def test_large_workload_grid_steps_against_oracle():
    """The large workload's grid and tolerance (2049^2 nodes, the electrons half
    in a Gaussian blob of sigma 0.2 L, multigrid to a 1e-10 relative residual),
    as a fused PIC step with 4M + 4M particles (the particle passes do not
    depend on the count; the bench times the full 64M + 64M): init and two
    steps bit-exact against the oracle, phi's FP64 residual below 1e-10 every
    time, rho within the deposit tolerance."""
    w = workloads.scaled(workloads.LARGE, n=4_000_000)
    assert (w.nodes, w.tol, w.blob) == (2049, 1e-10, True)
    m = w.nodes
    sim, arrays, mask, _ = build(w, 80, cap_factor=1.25)
    kq = [np.float32(CHARGES[s] / MASSES[s] * w.dt) for s in range(2)]
    dtdx = np.float32(w.dt / w.dx)
    ref = [oracle_sort([a.copy() for a in sp], m) for sp in arrays]
    assert sim.init() == 0
    _, _, Ex0, Ey0 = check_fields(sim, w, mask, ref, "init")
    for s in range(2):
        O.kick_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], Ex0, Ey0, np.float32(np.float64(kq[s]) * -0.5), m, m)
    E_prev = None
    absorbed = [0, 0]
    for i in range(2):
        assert sim.step(1) == 0
        for s in range(2):
            if i > 0:
                O.kick_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], E_prev[0], E_prev[1], kq[s], m, m)
            absorbed[s] += O.drift_absorb_f32(ref[s][0], ref[s][1], ref[s][2], ref[s][3], dtdx, dtdx, m, m)
        assert sim.counters()["absorbed"] == absorbed
        for s in range(2):
            got = host(sim, s)
            for k in range(5):
                assert_bits(got[k], ref[s][k], f"step {i + 1} species {s} array {k}")
        _, _, Ex, Ey = check_fields(sim, w, mask, ref, f"step {i + 1}")
        E_prev = (Ex, Ey)
    sim.close()
