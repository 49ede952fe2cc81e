"""Time-integration driver checks that need no GPU.

* the dual-time ESDIRK4 / SDIRK4 / backward-Euler steppers reach their orders
  on the harmonic oscillator of test/cpp/Solver/test_ODE.cpp:55-118, 183-200;
* GMRES on a small nonsymmetric system and the reference's own GMRES cases (test/cpp/Solver/test_Linear.cpp:44-150);
* the whole driver (frhs / fdtau / fsolve) running on the oracle advances an
  isentropic vortex stably.
"""
import math

import numpy as np
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.oracle_driver import OracleEval, OracleVR
from tests.util import oracle_for

W = 2 * math.pi


def _oscillator(ode, T, N):
    dt = T / N
    u = torch.tensor([[1.0, 0.0]], dtype=torch.float64)

    def frhs(rhs, x, dtau, it, ct):
        rhs[0, 0] = -W * x[0, 1]
        rhs[0, 1] = W * x[0, 0]

    def fdt(x, dtau, a):
        dtau.fill_(1e100)

    def fsolve(x, rhs, ro, dtau, dt_, a, xinc, it, ct):
        d = 1.0 / float(dtau[0]) + 1.0 / dt_
        aw = a * W
        det = d * d + aw * aw
        r0, r1 = float(rhs[0, 0]), float(rhs[0, 1])
        xinc[0, 0] = (d * r0 - aw * r1) / det
        xinc[0, 1] = (aw * r0 + d * r1) / det

    def fstop(it, res, st):
        return float(torch.linalg.norm(res)) < 1e-13 or it >= 50

    def finc(x, xinc, s):
        x.add_(xinc, alpha=s)

    for _ in range(N):
        ode.step(u, frhs, fdt, fsolve, 50, fstop, finc, dt)
    return math.hypot(float(u[0, 0]) - math.cos(W * T), float(u[0, 1]) - math.sin(W * T))


@pytest.mark.parametrize("scheme,N,lo,hi", [(0, 20, 3.5, 4.5), (1, 20, 3.5, 4.6)])
def test_sdirk_esdirk_order(scheme, N, lo, hi):
    e1 = _oscillator(I.ESDIRK(scheme), 1.0, N)
    e2 = _oscillator(I.ESDIRK(scheme), 1.0, 2 * N)
    assert lo < math.log2(e1 / e2) < hi


def test_backward_euler_order():
    e1 = _oscillator(I.BDF1Stepper(), 1.0, 200)
    e2 = _oscillator(I.BDF1Stepper(), 1.0, 400)
    assert 0.9 < math.log2(e1 / e2) < 1.3


def test_gmres_small_system():
    rng = np.random.default_rng(0)
    A = np.eye(20) * 4 + rng.normal(size=(20, 20)) * 0.3
    b = rng.normal(size=20)
    At = torch.tensor(A)
    g = I.GMRES(10, torch.zeros(20, dtype=torch.float64))
    x = torch.zeros(20, dtype=torch.float64)
    g.solve(lambda v, Av: Av.copy_(At @ v), lambda v, Mv: Mv.copy_(v), lambda a, c: float(a @ c), torch.tensor(b), x, 10,
            lambda i, r, rb: r < 1e-12 * rb)
    np.testing.assert_allclose(x.numpy(), np.linalg.solve(A, b), rtol=1e-9, atol=1e-11)


def _gmres(A, b, k, n_restart, tol, diag_prec=False):
    At = torch.tensor(A)
    dinv = torch.tensor(1.0 / np.diag(A))
    g = I.GMRES(k, torch.zeros(len(b), dtype=torch.float64))
    x = torch.zeros(len(b), dtype=torch.float64)
    seen = []

    def stop(i, r, rb):
        seen.append(i)
        return r < tol * rb
    ok = g.solve(lambda v, Av: Av.copy_(At @ v), (lambda v, Mv: Mv.copy_(dinv * v)) if diag_prec else (lambda v, Mv: Mv.copy_(v)),
                 lambda a, c: float(a @ c), torch.tensor(b, dtype=torch.float64), x, n_restart, stop)
    return ok, x.numpy(), seen[-1]


def test_gmres_reference_3x3_spd():
    # test_Linear.cpp:44-71: GMRES(3), 10 restarts, stop at 1e-14, error below 1e-12
    A = np.array([[4.0, 1, 0], [1, 3, 1], [0, 1, 2]])
    b = np.array([1.0, 2, 3])
    ok, x, _ = _gmres(A, b, 3, 10, 1e-14)
    assert ok and np.linalg.norm(x - np.linalg.solve(A, b)) < 1e-12


def test_gmres_reference_10x10_random_spd():
    # test_Linear.cpp:73-98: A = R^T R + 10 I with R uniform in [-1, 1] (seeded here), GMRES(10), 20 restarts
    R = np.random.default_rng(11).uniform(-1, 1, size=(10, 10))
    A = R.T @ R + 10 * np.eye(10)
    b = np.ones(10)
    ok, x, _ = _gmres(A, b, 10, 20, 1e-12)
    assert ok and np.linalg.norm(x - np.linalg.solve(A, b)) < 1e-10


def test_gmres_reference_diagonal_preconditioner():
    # test_Linear.cpp:100-150: diag (i + 1) 10 with A01 = A10 = 1, GMRES(3), 50 restarts; the diagonal
    # preconditioner converges in no more restarts and to 1e-10
    A = np.diag((np.arange(10) + 1) * 10.0)
    A[0, 1] = A[1, 0] = 1.0
    b = np.ones(10)
    _, _, r_npc = _gmres(A, b, 3, 50, 1e-12)
    ok, x, r_pc = _gmres(A, b, 3, 50, 1e-12, diag_prec=True)
    assert np.linalg.norm(x - np.linalg.solve(A, b)) < 1e-10
    assert r_pc <= r_npc


@pytest.mark.parametrize("gmres", [0, 1])
def test_driver_on_oracle_advances_vortex(gmres):
    m = M.renumber_by_color(M.iv_mesh(12))
    o = oracle_for(m, 2, "Roe", mu=0.0, ignoreVis=1)
    vr, ev = OracleVR(o), OracleEval(o)
    u = torch.tensor(o.init_field(2, 5.0))
    cfg = I.SolverConfig(odeCode=0, dtImplicit=0.01, nTimeStep=2, nTimeStepInternal=6, CFL=10.0, gmresCode=gmres, nGmresSpace=5)
    s = I.ImplicitSolver(vr, ev, cfg)
    u0 = u.clone()
    s.run(u)
    assert torch.isfinite(u).all()
    rel = float(torch.linalg.norm(u - u0) / torch.linalg.norm(u0))
    assert 1e-6 < rel < 0.05
    # the pseudo-time iterations reduce the unsteady residual of each implicit stage
    hist = [r for (_, it, r) in cfg.res_history if it == 1]
    last = [r for (_, it, r) in cfg.res_history if it == cfg.nTimeStepInternal]
    assert len(hist) > 0 and min(last) < max(hist)
