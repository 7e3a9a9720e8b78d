"""Pin the CPU oracle against the reference's own kernels.

tests/golden/*.npz were produced by running the reference's RawKernel sources
(compiled for the CPU by oracle/ref_build.py) on seeded inputs; see
tests/golden/make_golden.py.  The oracle's FP64 restatement must reproduce
them bit for bit.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10
    assert [int(v) for v in O.philox4x32_10([0, 0, 0, 0], [0, 0])] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C,
                                                                          0x9B00DBD8]
    assert [int(v) for v in O.philox4x32_10([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == [0x408F276D, 0x41C83B0E,
                                                                                     0xA20BC7C6, 0x6D5451FD]
    assert [int(v) for v in O.philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                            [0xA4093822, 0x299F31D0])] == [0xD16CFE09, 0x94FDCCEB, 0x5001E420,
                                                                           0x24126EA1]


def test_deposit_matches_reference_bitwise():
    g = load("particles_17x13.npz")
    m, n, dx, dy = int(g["m"]), int(g["n"]), float(g["dx"]), float(g["dy"])
    R, pt, q = g["R"], g["part_type"], g["q_type"]
    rho = np.zeros(m * n)
    for p in range(len(pt)):  # the reference's particle order
        O.deposit_f64(R[p:p + 1, 0], R[p:p + 1, 1], q[pt[p]] * float(g["np2c"]), dx, dy, m, n, rho=rho)
    rho = rho / (dx * dy)
    np.testing.assert_array_equal(rho, g["rho"])


def test_update_E_matches_reference_bitwise():
    g = load("particles_17x13.npz")
    m, n = int(g["m"]), int(g["n"])
    ex, ey = O.update_E_f64(g["phi"], m, n, float(g["dx"]), float(g["dy"]))
    np.testing.assert_array_equal(ex, g["E"][:m * n])
    np.testing.assert_array_equal(ey, g["E"][m * n:])


def test_update_V_matches_reference_bitwise():
    g = load("particles_17x13.npz")
    m, n, dx, dy, dt = int(g["m"]), int(g["n"]), float(g["dx"]), float(g["dy"]), float(g["dt"])
    R, V, pt = g["R"], g["V"].copy(), g["part_type"]
    ex, ey = g["E"][:m * n].copy(), g["E"][m * n:].copy()
    for p in range(len(pt)):
        k = dt * g["q_type"][pt[p]] * g["m_type_inv"][pt[p]]
        vx, vy = V[p:p + 1, 0].copy(), V[p:p + 1, 1].copy()
        O.lib().or_update_V_f64(R[p:p + 1, 0].copy(), R[p:p + 1, 1].copy(), vx, vy, 1, ex, ey, k, dx, dy, m, n, 1)
        V[p, 0], V[p, 1] = vx[0], vy[0]
    np.testing.assert_array_equal(V, g["V_kicked"])


def test_update_R_matches_reference_bitwise():
    g = load("particles_17x13.npz")
    R, V = g["R"], g["V_drift_in"]
    x, y = R[:, 0].copy(), R[:, 1].copy()
    O.lib().or_update_R_f64(x, y, V[:, 0].copy(), V[:, 1].copy(), len(x), 1e-10)
    np.testing.assert_array_equal(np.stack([x, y], 1), g["R_drift"])
    np.testing.assert_array_equal(g["R_old"], R)


def test_axis_kernel_reflects_and_build_absorbs():
    """The reference reflects particles with y < 0 (src/Particles.py:267-280);
    this build absorbs them on all four walls.  Document both."""
    g = load("particles_17x13.npz")
    R, V = g["R_drift"], g["V_drift_in"]
    below = R[:, 1] < 0
    assert below.any()
    np.testing.assert_array_equal(g["R_axis"][below, 1], -R[below, 1])
    np.testing.assert_array_equal(g["V_axis"][below, 1], -V[below, 1])
    x, y = R[:, 0].copy(), R[:, 1].copy()
    X = float(g["dx"]) * (int(g["m"]) - 1)
    Y = float(g["dy"]) * (int(g["n"]) - 1)
    absorbed = O.lib().or_absorb_f64(x, y, len(x), X, Y)
    out = (R[:, 0] < 0) | (R[:, 0] > X) | (R[:, 1] < 0) | (R[:, 1] > Y)
    assert absorbed == int(out.sum())
    assert np.isnan(x[out]).all() and not np.isnan(x[~out]).any()


def test_multigrid_kernels_match_reference_bitwise():
    g = load("multigrid_17.npz")
    n, h, bc, om = int(g["n"]), float(g["h"]), g["bc"], float(g["omega"])
    red = O.rb_sor_color(g["phi"].copy(), g["rhs"], bc, h * h, om, n, n, 1)
    np.testing.assert_array_equal(red, g["gs_red"])
    black = O.rb_sor_color(red.copy(), g["rhs"], bc, h * h, om, n, n, 0)
    np.testing.assert_array_equal(black, g["gs_black"])
    np.testing.assert_array_equal(O.residual_ref(g["phi"], g["rhs"], bc, 1.0 / (h * h), n, n), g["residual"])
    np.testing.assert_array_equal(O.restrict_ref(g["rhs"], n, n), g["restricted"])
    nc = (n + 1) // 2
    free = (1 - bc).astype(np.int32)
    np.testing.assert_array_equal(O.prolong_ref(g["phi"].copy(), g["coarse_in"], free, nc, nc), g["prolonged"])
    np.testing.assert_array_equal(O.coarsen_mask_ref(free, n, n, nc, nc), g["coarse_free"])


def test_oracle_residual_operator_agrees_with_reference_residual():
    g = load("multigrid_17.npz")
    n, h, bc = int(g["n"]), float(g["h"]), g["bc"]
    _, r = O.residual_f64(g["phi"], g["rhs"], bc.astype(np.uint8), n, n, h, h, want_r=True)
    ref = g["residual"]
    np.testing.assert_allclose(r, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_mcc_kernels_match_reference_bitwise():
    g = load("mcc.npz")
    speed, energy = O.speeds_energies_ref(g["V"], g["part_type"], g["m_type"])
    np.testing.assert_array_equal(speed, g["speeds"])
    np.testing.assert_array_equal(energy, g["energies"])
    np.testing.assert_array_equal(O.interp_ref(g["e_ev"], g["xs_e"], g["xs_s"], g["mcc_mask"]), g["sigma"])


def test_sort_matches_reference_serial_order():
    g = load("sort.npz")
    perm = O.counting_sort(g["cells"].astype(np.uint32), int(g["ncells"]))
    np.testing.assert_array_equal(perm.astype(np.int32), g["sorted_indices"])
    np.testing.assert_array_equal(perm, np.argsort(g["cells"], kind="stable"))


@pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built here")
def test_golden_regenerates_identically(tmp_path):
    """When the reference tree is present, its kernels still give the committed vectors."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("mg", os.path.join(GOLD, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.HERE = str(tmp_path)
    rng = np.random.Generator(np.random.Philox(20261203))
    mod.gen_particle_fixtures(rng)
    a, b = np.load(tmp_path / "particles_17x13.npz"), load("particles_17x13.npz")
    for k in b.files:
        np.testing.assert_array_equal(a[k], b[k])
