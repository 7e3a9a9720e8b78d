"""Hand-written adjoint of the collisionless step (pic_adj_*).

Checks: the FP64 forward pass against the CPU restatement (oracle/adjoint_ref.py);
the adjoint gradients against central finite differences of the GPU forward
pass and against the FP64 reference gradient (central differences of the CPU
restatement, 65x65 nodes, 1e4 particles), both within 1e-4 relative; the
torch.autograd.Function wrapper; and the cost of the backward pass against
the forward pass.

The loss is piecewise smooth: CIC weights and the interpolated field's
gradient have kinks at cell boundaries, and a particle that crosses one
between the runs at V - h and V + h moves a central difference by about one
particle's share of the gradient.  With h = 1e-3 V that reaches 1e-3
relative on these small cases, so the 1e-4 comparison uses h = 1e-5 V (the
multigrid tolerance, 1e-12, stays far below that perturbation) and h = 1e-3
V is checked at 1e-2.
"""
import time

import numpy as np
import pytest
import torch

from oracle import adjoint_ref
from pic_b200 import Consts, adjoint, workloads

pytestmark = pytest.mark.gpu
REL = 1e-4


def _case(nodes, n, steps, C, seed=11, Te=2.0):
    w = adjoint.AdjWorkload(nodes=nodes, n=n, steps=steps, checkpoint_every=C, seed=seed, Te=Te)
    return adjoint.build(w)


def _oracle(w_prob_inputs, nodes, steps, V_unused=None):
    prob, V0, A0, inp = w_prob_inputs
    dx = 1e-4
    sp = []
    ex, ey, evx, evy, dvx = inp["e"]
    ix, iy, ivx, ivy = inp["i"]
    for d, arr, dv in ((inp["species"][0], (ex, ey, evx, evy), dvx), (inp["species"][1], (ix, iy, ivx, ivy), None)):
        sp.append(dict(charge=d["charge"], mass=d["mass"], np2c=d["np2c"], x=arr[0], y=arr[1], vx=arr[2], vy=arr[3],
                       dvx=0.0 if dv is None else dv, dvy=0.0))
    return adjoint_ref.RefDifferentiable(nodes, nodes, dx, dx, 1e-11, Consts.eps0, sp, inp["mask"], inp["seg"], 4,
                                         steps, 0, inp["target"])


def test_forward_matches_the_fp64_restatement():
    case = _case(33, 3000, 25, 10)
    prob, V0, A0, inp = case
    loss = prob.forward(V0, A0)
    ref = _oracle(case, 33, 25)
    rloss, pos, alive = ref.run(V0, A0)
    assert loss == pytest.approx(rloss, rel=1e-9)
    x, y, _, _, death, _ = prob.state()
    x, y, death = x.cpu().numpy(), y.cpu().numpy(), death.cpu().numpy()
    n = 3000
    for s in range(2):
        sl = slice(s * n, (s + 1) * n)
        a = death[sl] > 25
        np.testing.assert_array_equal(a, alive[s])
        assert np.abs(x[sl][a] - pos[s][0][a]).max() < 1e-8
        assert np.abs(y[sl][a] - pos[s][1][a]).max() < 1e-8
    prob.close()


def _rel_err(g, ref):
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(np.asarray(g) - np.asarray(ref)).max() / scale


def _gpu_fd(prob, V0, A0, h, hA):
    fd = np.zeros(4)
    for q in range(4):
        e = np.zeros(4)
        e[q] = h
        fd[q] = (prob.forward(V0 + e, A0) - prob.forward(V0 - e, A0)) / (2 * h)
    fdA = (prob.forward(V0, A0 + hA) - prob.forward(V0, A0 - hA)) / (2 * hA)
    return fd, fdA


def test_adjoint_matches_gpu_finite_differences():
    # 40 steps with checkpoints every 7 (a partial last segment)
    prob, V0, A0, _ = _case(65, 10_000, 40, 7)
    prob.forward(V0, A0)
    dV, dA = prob.backward()
    fd, fdA = _gpu_fd(prob, V0, A0, 1e-5, 0.1)
    assert _rel_err(dV, fd) < REL, (dV, fd)
    assert abs(dA - fdA) <= REL * abs(fdA), (dA, fdA)
    fd3, fdA3 = _gpu_fd(prob, V0, A0, 1e-3, 1.0)
    assert _rel_err(dV, fd3) < 1e-2, (dV, fd3)
    assert abs(dA - fdA3) <= 1e-2 * abs(fdA3), (dA, fdA3)
    prob.close()


def test_adjoint_matches_the_fp64_reference_gradient():
    case = _case(65, 5_000, 30, 10, seed=12)
    prob, V0, A0, _ = case
    prob.forward(V0, A0)
    dV, dA = prob.backward()
    ref = _oracle(case, 65, 30)
    rV, rA = ref.gradient_fd(V0, A0, hV=1e-5, hA=0.1)
    assert _rel_err(dV, rV) < REL, (dV, rV)
    assert abs(dA - rA) <= REL * abs(rA), (dA, rA)
    prob.close()


def test_autograd_function_gives_the_adjoint_gradients():
    prob, V0, A0, _ = _case(33, 2000, 12, 5)
    V = torch.tensor(V0, dtype=torch.float64, requires_grad=True)
    A = torch.tensor(A0, dtype=torch.float64, requires_grad=True)
    loss = adjoint.ElectrodeLoss.apply(V, A, prob)
    (3.0 * loss).backward()
    prob.forward(V0, A0)
    dV, dA = prob.backward()
    np.testing.assert_allclose(V.grad.numpy(), 3.0 * dV, rtol=1e-12)
    assert float(A.grad) == pytest.approx(3.0 * dA, rel=1e-12)
    prob.close()


def test_backward_costs_at_most_four_forward_passes():
    prob, V0, A0, _ = _case(129, 100_000, 40, 10)
    prob.forward(V0, A0)
    prob.backward()  # warm-up: graphs captured
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prob.forward(V0, A0)
    t1 = time.perf_counter()
    prob.backward()
    t2 = time.perf_counter()
    assert (t2 - t1) <= 4.0 * (t1 - t0), (t1 - t0, t2 - t1)
    prob.close()
