"""The reference's one-Newton-step goldens (test/cpp/Euler/test_EulerEvaluator.cpp:120-330) through the
C-ABI on the GPU, and the operators that sequence adds: the batched mean-value Roe flux
(rsMeanValueEig) and UpdateLUSGSForward / UpdateLUSGSBackward.

Tolerances: the reference's own 1e-6 relative on its golden norms; 1e-12 relative for FP64 operator
parity with the oracle; dual consistency 1e-12.
"""
import numpy as np
import pytest
import torch

import oracle
from dndsr_b200 import mesh as M
from tests.newton_case import CASES, GAS, initial_state, norms
from tests.util import relerr

pytestmark = pytest.mark.gpu


def _t(x):
    return torch.tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")


def _gpu_case(case):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = case["mesh"]()
    vr = VariationalReconstruction(m, case["vr_py"]).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=case["rs"], rsMeanValueEig=case["rsMeanValueEig"], **GAS))
    return m, vr, ev


@pytest.mark.parametrize("name", list(CASES))
def test_newton_step_golden_gpu(name):
    case = CASES[name]
    m, vr, ev = _gpu_case(case)
    u = vr.BuildUDof(5)
    if "chi" in case["gold"]:
        ev.InitializeUDOF(u, 2, case["gold"]["chi"])
    else:
        u.copy_(_t(initial_state(case, vr.get("cellBary").reshape(-1, 3))))
    ev.FixUMaxFilter(u)
    dTau = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, u, case["CFL"], 1e100, True)
    uRec = vr.BuildURec(5)
    rhs = vr.BuildUDof(5)
    ev.EvaluateRHS(rhs, u, uRec)
    l1 = ev.EvaluateNorm(rhs, 1, True)
    jd = ev.BuildJDiag()
    ev.LUSGSMatrixInit(jd, dTau, 1e100, 1.0)
    xinc, xincNew = vr.BuildUDof(5), vr.BuildUDof(5)
    ev.UpdateLUSGSForward(1.0, rhs, u, xinc, jd, xincNew)
    ev.UpdateLUSGSBackward(1.0, rhs, u, xinc, jd, xincNew)
    inc = ev.EvaluateNorm(xincNew, 2, False)
    g = case["gold"]
    assert abs(l1[0] - g["rhsDensityL1"]) <= g["rel_tol"] * g["rhsDensityL1"]
    assert abs(np.linalg.norm(inc) - g["incL2"]) <= g["rel_tol"] * g["incL2"]
    # the same numbers from the arrays (EvaluateNorm's own reductions are checked elsewhere)
    r, i = norms(rhs.cpu().numpy(), xincNew.cpu().numpy(), vr.get("volume"))
    assert abs(r - l1[0]) <= 1e-12 * r and abs(i - np.linalg.norm(inc)) <= 1e-12 * i


def _warped(rs, mve, p=2):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.tgv_mesh(5))
    vro = dict(CASES["iv"]["vr_oracle"], maxOrder=p, intOrder=5)
    es = dict(nVars=5, rsType=oracle.RS[rs], rsFixScale=1.0, rsIncFScale=1.0, ignoreVis=1, rsMeanValueEig=mve, gamma=1.4, Rgas=1.0,
              muGas=0.0, prGas=0.72, TRef=273.15, CSutherland=110.4, muModel=0)
    o = oracle.Oracle(m, vro, es)
    assert o.construct() == 0
    vr = VariationalReconstruction(m, dict(CASES["iv"]["vr_py"], maxOrder=p, intOrder=5)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, rsMeanValueEig=mve, ignoreVis=True, gamma=1.4, Rgas=1.0, muGas=0.0,
                                 muModel=0))
    return m, o, vr, ev


@pytest.mark.parametrize("rs", ["Roe_M1", "Roe_M2", "Roe_M3", "Roe_M4", "Roe_M5"])
def test_mean_value_eig_rhs_parity(rs):
    # warped hexahedra: per-point normals differ from the face's mean normal
    m, o, vr, ev = _warped(rs, 1)
    u0 = o.init_field(3)
    rng = np.random.default_rng(11)
    uRec0 = rng.normal(size=(m.n_cell, o.R, 5)) * 0.02 * np.abs(u0).mean(0)
    dt0, _ = o.eval_dt(u0, 1.0)
    ref = o.eval_rhs(u0, uRec0)
    u, uRec = _t(u0), _t(uRec0)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    assert relerr(rhs.cpu().numpy(), ref) < 1e-12
    # derivatives: the forward-mode face kernel carries the mean normal on every face
    w = _t(rng.normal(size=u0.shape))
    du, duRec = ev.EvaluateRHSVJP(w, u, uRec)
    vu, vRec = _t(rng.normal(size=u0.shape)), _t(rng.normal(size=uRec0.shape))
    jv = ev.EvaluateRHSJVP(vu, vRec, u, uRec)
    lhs = float((w * jv).sum())
    rhs_ = float((du * vu).sum() + (duRec * vRec).sum())
    assert abs(lhs - rhs_) <= 1e-12 * max(abs(lhs), 1e-300) * 10
    # JVP against a central difference of the oracle's residual.  Roe_M1, M2 and M5 switch their
    # eigenvalues by sign and max (Gas.hpp:878-1007: signTol jumps at u.n = 0), so a difference
    # quotient across a switch is not a derivative; their JVP is the forward-mode derivative of the
    # primal code checked above, and the transpose identity covers the VJP
    if rs not in ("Roe_M3", "Roe_M4"):
        return
    h = 1e-6
    fd = (o.eval_rhs(u0 + h * vu.cpu().numpy(), uRec0 + h * vRec.cpu().numpy()) -
          o.eval_rhs(u0 - h * vu.cpu().numpy(), uRec0 - h * vRec.cpu().numpy())) / (2 * h)
    assert relerr(jv.cpu().numpy(), fd) < 1e-6


def test_update_lusgs_parity():
    m, o, vr, ev = _warped("Roe", 0, p=1)
    u0 = o.init_field(3)
    rng = np.random.default_rng(5)
    dt0, _ = o.eval_dt(u0, 2.0)
    rhs0 = rng.normal(size=u0.shape)
    jd0 = o.lusgs_init(dt0, 0.05, 1.0)
    x0 = rng.normal(size=u0.shape) * 0.1
    u, rhs = _t(u0), _t(rhs0)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 2.0)
    jd = ev.BuildJDiag()
    ev.LUSGSMatrixInit(jd, dt, 0.05, 1.0)
    assert relerr(jd.cpu().numpy(), jd0) < 1e-12
    # separate arrays (every cell independent)
    ref = o.update_lusgs(1.0, rhs0, u0, x0, np.zeros_like(u0), jd0, forward=True)
    ref = o.update_lusgs(1.0, rhs0, u0, x0, ref, jd0, forward=False)
    x, xn = _t(x0), torch.zeros_like(u)
    ev.UpdateLUSGSForward(1.0, rhs, u, x, jd, xn)
    ev.UpdateLUSGSBackward(1.0, rhs, u, x, jd, xn)
    assert relerr(xn.cpu().numpy(), ref) < 1e-12
    # in place (uInc is uIncNew): sequential Gauss-Seidel order, exact on the colour-numbered mesh
    ref = o.update_lusgs(1.0, rhs0, u0, None, x0, jd0, forward=True, inplace=True)
    ref = o.update_lusgs(1.0, rhs0, u0, None, ref, jd0, forward=False, inplace=True)
    y = _t(x0)
    ev.UpdateLUSGSForward(1.0, rhs, u, y, jd, y)
    ev.UpdateLUSGSBackward(1.0, rhs, u, y, jd, y)
    assert relerr(y.cpu().numpy(), ref) < 1e-12
