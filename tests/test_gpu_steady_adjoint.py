"""Steady adjoint on the GPU: the transposed LU-SGS kernels and the pressure-force objective
against the oracle, and the coupled adjoint solve against the tangent solve.

* LUSGSMatrixVec transposed and one transposed Gauss-Seidel sweep per direction: parity with
  the oracle at 1e-12 on a colour-numbered bump mesh (the colour order is then the oracle's
  sequential order);
* pressure force on the bump and its gradient: parity with the oracle at 1e-12;
* the coupled Jacobian of (EvaluateRHS, VR sweep residual) and its transpose satisfy
  <A^T y, x> = <y, A x> at 1e-12;
* adjoint and tangent GMRES solves reach a 1e-10 residual drop, and the sensitivity of the
  pressure force to a residual source agrees between them, -<psi, s> = <g, d>, at 1e-8.
  The solves run on the system of one implicit Euler step (dt = 5 local CFL-1 time steps): the
  purely steady system of this reflecting channel at a non-steady state is as badly conditioned
  as the primal defect correction, whose residual also levels off.
"""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu

BUMP = M.BUMP_ZONES["bump"]
DRAG = np.array([1.0, 0.0, 0.0])


def _setup(p, mach=0.5):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.bump_channel_tet(8, 4, 3, periodic_z=True))
    o, far, types, vals, w = bump_oracle(m, p, "Roe", 0.0, 1, mach=mach)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    ev.SetBC(types, vals)
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    uRec0 *= 0.1
    return m, o, vr, ev, u0, uRec0, torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")


@pytest.mark.parametrize("p", [1, 2])
def test_transposed_lusgs_and_pressure_force_parity(p):
    m, o, vr, ev, u0, uRec0, u, uRec = _setup(p)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    dt0, _ = o.eval_dt(u0, 5.0)
    jd = ev.BuildJDiag()
    ev.LUSGSMatrixInit(jd, dt, 1e100, 1.0)
    jd0 = o.lusgs_init(dt0, 1e100, 1.0)
    assert relerr(jd.cpu().numpy(), jd0) < 1e-12
    rng = np.random.default_rng(4)
    y0 = rng.normal(size=u0.shape)
    b0 = rng.normal(size=u0.shape)
    y = torch.tensor(y0, device="cuda")
    out = torch.empty_like(y)
    ev.LUSGSMatrixVecT(1.0, u, y, jd, out)
    assert relerr(out.cpu().numpy(), o.lusgs_matvec_t(1.0, u0, y0, jd0)) < 1e-12
    x = torch.tensor(rng.normal(size=u0.shape), device="cuda")
    Ax = torch.empty_like(x)
    ev.LUSGSMatrixVec(1.0, u, x, jd, Ax)
    a, bb = float((Ax * y).sum()), float((x * out).sum())
    assert abs(a - bb) < 1e-12 * (abs(a) + 1)
    for forward in (True, False):
        yn = torch.empty_like(y)
        ev.UpdateSGST(1.0, torch.tensor(b0, device="cuda"), u, y, yn, jd, forward)
        ref = o.update_sgs_t(1.0, b0, u0, y0, y0, jd0, forward)
        assert relerr(yn.cpu().numpy(), ref) < 1e-12
        # the FP32 sweep (float vectors, FP64 operator) of the adjoint preconditioner
        yn32 = torch.empty_like(y, dtype=torch.float32)
        ev.UpdateSGST(1.0, torch.tensor(b0, device="cuda", dtype=torch.float32), u, y.float(), yn32, jd, forward)
        assert relerr(yn32.double().cpu().numpy(), ref) < 1e-6
    J, gU, gR = ev.PressureForce(BUMP, DRAG, u, uRec, grad=True)
    J0, gU0, gR0 = o.pressure_force(BUMP, DRAG, u0, uRec0, grad=True)
    assert abs(J - J0) < 1e-12 * abs(J0)
    assert relerr(gU.cpu().numpy(), gU0) < 1e-12 and relerr(gR.cpu().numpy(), gR0) < 1e-12
    assert ev.PressureForce(BUMP, DRAG, u, uRec) == J


@pytest.mark.parametrize("p", [1, 2])
def test_coupled_adjoint_and_tangent_solves_agree(p):
    from dndsr_b200.adjoint import SteadyAdjoint
    m, o, vr, ev, u0, uRec0, u, uRec = _setup(p)
    dTau = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, u, 1.0)
    adj = SteadyAdjoint(vr, ev, u, uRec, cfl=5.0, dt=5.0 * float(dTau.max()))
    rng = np.random.default_rng(9)
    # the transpose is exact
    x = (torch.tensor(rng.normal(size=u0.shape), device="cuda"), torch.tensor(rng.normal(size=uRec0.shape), device="cuda"))
    y = (torch.tensor(rng.normal(size=u0.shape), device="cuda"), torch.tensor(rng.normal(size=uRec0.shape), device="cuda"))
    Ax, ATy = adj.op(x), adj.op_T(y)
    lhs = sum(float((a * b).sum()) for a, b in zip(ATy, x))
    rhs = sum(float((a * b).sum()) for a, b in zip(y, Ax))
    assert abs(lhs - rhs) < 1e-12 * abs(rhs)
    # adjoint of the pressure force and the tangent response to a residual source
    J, gU, gR = ev.PressureForce(BUMP, DRAG, u, uRec, grad=True)
    psi, lam, h_adj = adj.solve_adjoint(gU, gR, restart=32, max_restarts=60, rtol=1e-10)
    assert h_adj[-1] < 1e-10
    # FP32 transposed LU-SGS inside the FP64 Krylov iteration reaches the same adjoint
    adj32 = SteadyAdjoint(vr, ev, u, uRec, cfl=5.0, dt=5.0 * float(dTau.max()), precision="fp32")
    psi32, lam32, h32 = adj32.solve_adjoint(gU, gR, restart=32, max_restarts=60, rtol=1e-10)
    assert h32[-1] < 1e-10 and relerr(psi32.cpu().numpy(), psi.cpu().numpy()) < 1e-8
    sU = torch.tensor(rng.normal(size=u0.shape), device="cuda")
    sR = torch.zeros_like(uRec)
    du, dRec, h_tan = adj.solve_tangent(sU, sR, restart=32, max_restarts=60, rtol=1e-10)
    assert h_tan[-1] < 1e-10
    via_adjoint = -float((psi * sU).sum())
    via_tangent = float((gU * du).sum() + (gR * dRec).sum())
    assert abs(via_adjoint - via_tangent) < 1e-8 * abs(via_tangent)
