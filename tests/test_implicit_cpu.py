"""Time-integration driver checks that need no GPU.

* the dual-time ESDIRK4 / SDIRK4 / backward-Euler steppers reach their orders
  on the harmonic oscillator of test/cpp/Solver/test_ODE.cpp:55-118, 183-200;
* GMRES on a small nonsymmetric system (test/cpp/Solver/test_Linear.cpp);
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
