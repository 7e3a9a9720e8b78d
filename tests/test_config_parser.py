"""The .inp reader (pic_b200/ConfigParser.py): blocks, comments, variables,
safe arithmetic, and the simulation builder on the GPU."""
import numpy as np
import pytest

from pic_b200 import ConfigParser as CP

TEXT = """
Description
{
A small two-electrode gap, all walls grounded.
}
System
{
  MAX_PARTICLES = 400000   // room for both species
  SAVE_FIELDS = true
}
Variables
{
  V0 = 40
  Jmax = 129
  Kmax = Jmax
  X = 0.0128
  dtBase = 2.0e-11
  half = V0 / 2
}
Grid
{
  Cylindrical = 0
  J = Jmax
  K = Kmax
  x1s = 0
  x1f = X
  x2s = 0
  x2f = X
}
Control
{
  dt = dtBase
  solver = 'multigrid'
}
Species
{
  name = electrons
  m = 9.11E-31
  q = -1.60E-19
  collisionModel = 0
}
Species
{
  name = ions
  m = 40 * 1.66e-27
  q = 1.6e-19
  collisionModel = 1
}
Equipotential
{
  C = -half
  name = cathode
  j1 = (Jmax - 1) / 4
  j2 = (Jmax - 1) / 4
  k1 = 0
  k2 = (Kmax - 1) / 2
}
Equipotential
{
  C = half
  name = anode
  j1 = 3 * (Jmax - 1) / 4
  j2 = 3 * (Jmax - 1) / 4
  k1 = 0
  k2 = (Kmax - 1) / 2
}
Load
{
  speciesName = electrons
  n = 50000
  x1MinMKS = 0.001
  x1MaxMKS = 0.0118
  x2MinMKS = 0.001
  x2MaxMKS = 0.0118
  temperature = 2
  np2c = 1e5
}
Load
{
  speciesName = ions
  n = 50000
  x1MinMKS = 0.001
  x1MaxMKS = 0.0118
  x2MinMKS = 0.001
  x2MaxMKS = 0.0118
  np2c = 1e5
}
MCC
{
  gas = Ar
  temperature = 300
}
"""


def test_blocks_and_values():
    cfg = CP.ConfigParser().parse_text(TEXT)
    assert cfg["system"] == {"MAX_PARTICLES": 400000, "SAVE_FIELDS": True}
    v = cfg["variables"]
    assert v["Kmax"] == 129.0 and v["half"] == 20.0
    assert cfg["grid"]["J"] == 129.0 and cfg["grid"]["x1f"] == 0.0128
    assert cfg["control"] == {"dt": 2e-11, "solver": "multigrid"}
    assert [s["name"] for s in cfg["species"]] == ["electrons", "ions"]
    assert cfg["species"][1]["m"] == pytest.approx(40 * 1.66e-27)
    assert cfg["boundaries"] == [((32.0, 0.0, 32.0, 64.0), -20.0), ((96.0, 0.0, 96.0, 64.0), 20.0)]
    assert len(cfg["loads"]) == 2 and cfg["loads"][0]["temperature"] == 2.0
    assert cfg["mcc"] == [{"gas": "Ar", "temperature": 300.0}]


def test_names_are_not_substituted_as_substrings():
    # X and Jmax are both variables; "Jmax" must not be read as "J" + "max" or rewritten through X
    names = {"X": 2.0, "Jmax": 128.0}
    assert CP.evaluate("Jmax / 4", names) == 32.0
    assert CP.evaluate("X * Jmax", names) == 256.0
    assert CP.evaluate("Xmax", names) == "Xmax"


def test_only_arithmetic_is_evaluated():
    assert CP.evaluate("__import__('os').getcwd()", {}) == "__import__('os').getcwd()"
    assert CP.evaluate("(1).__class__", {}) == "(1).__class__"
    assert CP.evaluate("pow(2, 10) + sqrt(16)", {}) == 1028.0
    assert CP.evaluate("electrons", {}) == "electrons"


def test_grid_node_counts():
    assert CP.multigrid_compatible(129) and CP.multigrid_compatible(513) and CP.multigrid_compatible(97)
    assert not CP.multigrid_compatible(128) and not CP.multigrid_compatible(1000)


def test_node_counts_must_coarsen():
    for text in (TEXT, TEXT.replace("Cylindrical = 0", "Cylindrical = 1")):
        cfg = CP.ConfigParser().parse_text(text.replace("Jmax = 129", "Jmax = 128"))
        with pytest.raises(ValueError):
            CP.build_simulation(cfg)


@pytest.mark.gpu
def test_build_run_and_dump(tmp_path):
    cfg = CP.ConfigParser().parse_text(TEXT)
    sim = CP.build_simulation(cfg, seed=3)
    sim.init()
    sim.step(10)
    sim.sync()
    c = sim.counters()
    assert c["steps"] == 10
    # slots of collected particles stay (dead) until the next sort compacts them
    live = sum(sim.diagnostics()["live"])
    assert live + sum(c["absorbed"]) + sum(c["electrode_absorbed"]) == 100_000
    assert sum(c["electrode_absorbed"]) > 0
    phi = sim.fields()[0].cpu().numpy().reshape(129, 129)
    assert phi[10, 32] == -20.0 and phi[10, 96] == 20.0 and phi[100, 32] != -20.0
    path = tmp_path / "fields.txt"
    CP.save_fields(sim, str(path))
    data = np.loadtxt(path)
    assert data.shape == (129 * 129, 6)
    np.testing.assert_allclose(data[:, 3], phi.reshape(-1), rtol=6e-3, atol=1e-30)
    sim.close()


@pytest.mark.gpu
def test_cylindrical_file_runs_in_rz():
    """Cylindrical = 1 (the reference's shipped input is cylindrical): the two
    electrodes are disks on the axis; the axis row is free, particles stay at
    r >= 0 and charge is conserved between the live particles, the walls and
    the electrodes."""
    cfg = CP.ConfigParser().parse_text(TEXT.replace("Cylindrical = 0", "Cylindrical = 1"))
    sim = CP.build_simulation(cfg, seed=4)
    assert sim.geometry == "rz"
    sim.init()
    sim.step(10)
    sim.sync()
    c = sim.counters()
    live = sum(sim.diagnostics()["live"])
    assert live + sum(c["absorbed"]) + sum(c["electrode_absorbed"]) == 100_000
    assert sum(c["electrode_absorbed"]) > 0
    for s in range(2):
        x, y = (a.cpu().numpy() for a in sim.species_arrays(s)[:2])
        yl = y[np.isfinite(x)]
        assert yl.size and yl.min() >= 0.0 and yl.max() <= 128.0
    phi = sim.fields()[0].cpu().numpy().reshape(129, 129)
    # electrode nodes keep their potentials, the axis nodes between them are free
    assert phi[0, 32] == -20.0 and phi[0, 96] == 20.0
    assert -20.0 < phi[0, 64] < 20.0
    sim.close()
