"""The FP64 CPU restatement behind the adjoint tests (oracle/adjoint_ref.py):
its Poisson solve, its conservation of particles without walls in reach, and
the workload's wall segments and target profile."""
import numpy as np

from oracle import adjoint_ref
from pic_b200 import Consts, adjoint


def test_wall_segments_cover_the_edges():
    mask, seg = adjoint.wall_segments(9, 7)
    m, s = mask.reshape(7, 9), seg.reshape(7, 9)
    assert m[0].all() and m[-1].all() and m[:, 0].all() and m[:, -1].all() and not m[1:-1, 1:-1].any()
    assert (s[:, 0] == 0).all() and (s[:, -1] == 2).all()  # corners with the left and right walls
    assert (s[0, 1:-1] == 1).all() and (s[-1, 1:-1] == 3).all()
    assert (s[1:-1, 1:-1] == -1).all()


def test_target_profile_is_seeded_and_positive():
    a = adjoint.target_density(33, 33, 1e14, 5)
    b = adjoint.target_density(33, 33, 1e14, 5)
    assert np.array_equal(a, b) and (a >= 1e14).all() and a.max() > 1.2e14


def _ref(V_left=10.0, n=0, steps=0):
    nodes = 17
    mask, seg = adjoint.wall_segments(nodes, nodes)
    rng = np.random.default_rng(0)
    x = rng.uniform(6, 10, n)
    y = rng.uniform(6, 10, n)
    sp = [dict(charge=-Consts.qe, mass=Consts.me, np2c=1.0, x=x, y=y, vx=np.zeros(n), vy=np.zeros(n))]
    return adjoint_ref.RefDifferentiable(nodes, nodes, 1e-4, 1e-4, 1e-12, Consts.eps0, sp, mask, seg, 4, steps, 0,
                                         np.zeros(nodes * nodes))


def test_poisson_solve_is_discrete_laplace_with_the_wall_potentials():
    r = _ref()
    G = 17 * 17
    phiB = np.where(r.mask, 0.0, 0.0)
    phiB[r.mask & (r.seg == 0)] = 10.0
    phi = r._solve(np.zeros(G), phiB).reshape(17, 17)
    lap = (phi[1:-1, :-2] + phi[1:-1, 2:] + phi[:-2, 1:-1] + phi[2:, 1:-1] - 4 * phi[1:-1, 1:-1])
    assert np.abs(lap).max() < 1e-10
    assert np.allclose(phi[:, 0], 10.0) and np.allclose(phi[0, 1:], 0.0)
    assert 0.0 < phi[8, 1] < 10.0


def test_particles_far_from_the_walls_are_all_kept():
    r = _ref(n=200, steps=5)
    loss, pos, alive = r.run(np.zeros(4), 0.0)
    assert alive[0].all() and loss >= 0.0
