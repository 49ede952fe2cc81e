"""Native linear solve (dndsb_eval_solve_linear) and the implicit driver on the GPU.

The oracle's UpdateSGS / LUSGSMatrixVec, orchestrated by the Python GMRES of
dndsr_b200.implicit exactly as EulerSolver::solveLinear does
(EulerSolver.hxx:1407-1579), is the reference.  Tolerances: 1e-11 relative
for the FP64 solve (a chain of ~100 FP64 operator applications), 1e-5 for the
FP32 preconditioner, whose output feeds the FP64 defect correction.
"""
import numpy as np
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.oracle_driver import OracleEval, OracleVR
from tests.util import VR_HQM_PY, oracle_for, relerr

pytestmark = pytest.mark.gpu

CASES = [
    ("iv-tri-p2-Roe", lambda: M.iv_mesh(10), 2, 2, "Roe", 0.0),
    ("tgv-hex-p1-HLLEP", lambda: M.tgv_mesh(5), 1, 3, "HLLEP", 1 / 1600),
    ("bump-tet-p1-Roe", lambda: M.bump_channel_tet(6, 4, 2), 1, 0, "Roe", 0.0),
]


def _setup(mk, p, rs, mu):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(mk())
    if (m.face2cell[:, 1] < 0).any():
        from tests.bump_case import bump_oracle
        o, far, types, vals, w = bump_oracle(m, p, rs, mu, ignoreVis=int(mu == 0))
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=0, ignoreVis=mu == 0))
        ev.SetBC(types, vals)
        o._far = far
        return m, o, vr, ev
    o = oracle_for(m, p, rs, mu, ignoreVis=int(mu == 0))
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=0, ignoreVis=mu == 0))
    return m, o, vr, ev


def _init(o, kind):
    if kind == 0:
        from tests.bump_case import perturbed_state
        return torch.tensor(perturbed_state(o.mesh, o._far))
    return torch.tensor(o.init_field(kind, 5.0))


def _reference_solve(oe, u, rhs, dTau, dt, alpha, code, jacobi, sgsIter, k, nIter, meanScale=None):
    jd = torch.zeros((u.shape[0], 6) if u.shape[1] == 6 else (u.shape[0],), dtype=torch.float64)
    oe.LUSGSMatrixInit(jd, dTau, dt, alpha)
    tmp = torch.zeros_like(rhs)

    def pair(b, x):
        oe.UpdateSGS(alpha, b, u, x, tmp, jd, True, jacobi == 1, False)
        x.copy_(tmp)
        oe.UpdateSGS(alpha, b, u, x, tmp, jd, False, jacobi == 1, False)
        x.copy_(tmp)

    x = torch.zeros_like(rhs)
    if code in (0, 2):
        for _ in range(1 + sgsIter):
            pair(rhs, x)
    if code:
        s2 = torch.ones(u.shape[1], dtype=torch.float64) if meanScale is None else torch.tensor([1 / (m + 1e-200) ** 2 for m in meanScale])
        g = I.GMRES(k, x)

        def FML(v, Mv):
            Mv.zero_()
            for _ in range(1 + sgsIter):
                pair(v, Mv)

        g.solve(lambda v, Av: oe.LUSGSMatrixVec(alpha, u, v, jd, Av), FML, lambda a, b: float((a * b * s2).sum()), rhs, x, nIter,
                lambda i, r, rb: False)
    return x


@pytest.mark.parametrize("name,mk,p,kind,rs,mu", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("code,jacobi,sgsIter,k,nIter", [(0, 1, 1, 1, 1), (0, 0, 0, 1, 1), (1, 1, 0, 8, 2), (2, 1, 1, 5, 1), (1, 0, 1, 6, 1)])
def test_solve_linear_matches_reference_orchestration(name, mk, p, kind, rs, mu, code, jacobi, sgsIter, k, nIter):
    m, o, vr, ev = _setup(mk, p, rs, mu)
    oe = OracleEval(o)
    u0 = _init(o, kind)
    dTau0 = torch.zeros(m.n_cell, dtype=torch.float64)
    oe.EvaluateDt(dTau0, u0, 1e3)
    rhs0 = torch.tensor(np.random.default_rng(3).normal(size=(m.n_cell, 5)))
    alpha, dt = 0.5, 10.0
    ref = _reference_solve(oe, u0, rhs0, dTau0, dt, alpha, code, jacobi, sgsIter, k, nIter)
    u, rhs = u0.cuda(), rhs0.cuda()
    dTau = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, u, 1e3)
    for prec, tol in [("fp64", 1e-11), ("fp32", 1e-5)]:
        outs = []
        for graph in (True, True, False):
            x = torch.full_like(rhs, 7.0)
            ev.SolveLinear(alpha, dTau, dt, u, rhs, x, gmresCode=code, jacobiCode=jacobi, sgsIter=sgsIter, nGmresSpace=k, nGmresIter=nIter,
                           precision=prec, useGraph=graph)
            outs.append(x.cpu())
        assert relerr(outs[0].numpy(), ref.numpy()) < tol, prec
        # graph capture, graph replay and direct launches give identical bits
        assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])


def test_solve_linear_weighted_dot_and_errors():
    from dndsr_b200.capi import DndsbError
    m, o, vr, ev = _setup(lambda: M.iv_mesh(8), 1, "Roe", 0.0)
    oe = OracleEval(o)
    u0 = torch.tensor(o.init_field(2, 5.0))
    dTau0 = torch.zeros(m.n_cell, dtype=torch.float64)
    oe.EvaluateDt(dTau0, u0, 100.0)
    rhs0 = torch.tensor(np.random.default_rng(5).normal(size=(m.n_cell, 5)))
    ms = [1.0, 1.2, 1.2, 1.2, 2.5]
    ref = _reference_solve(oe, u0, rhs0, dTau0, 1.0, 1.0, 1, 1, 0, 6, 1, meanScale=ms)
    u, rhs = u0.cuda(), rhs0.cuda()
    dTau = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, u, 100.0)
    x = torch.zeros_like(rhs)
    ev.SolveLinear(1.0, dTau, 1.0, u, rhs, x, gmresCode=1, nGmresSpace=6, meanScale=ms)
    # CFL 100 with dt = 1: the operator's conditioning amplifies the FP64 rounding of the
    # differently ordered sums, hence a looser bound than the per-call operator parity
    assert relerr(x.cpu().numpy(), ref.numpy()) < 1e-9
    with pytest.raises(DndsbError):
        ev.SolveLinear(1.0, dTau, 1.0, u, rhs, x, gmresCode=1, nGmresSpace=40)


def test_driver_gpu_matches_oracle_driver():
    """Three ESDIRK4 steps of the isentropic vortex, 4 pseudo iterations each:
    the GPU driver (native linear solve) against the same driver on the oracle."""
    m, o, vr, ev = _setup(lambda: M.iv_mesh(10), 2, "Roe", 0.0)
    kw = dict(odeCode=0, dtImplicit=0.05, nTimeStep=3, nTimeStepInternal=4, CFL=20.0, gmresCode=1, nGmresSpace=5, sgsIter=0)
    u_o = torch.tensor(o.init_field(2, 5.0))
    I.ImplicitSolver(OracleVR(o), OracleEval(o), I.SolverConfig(**kw)).run(u_o)
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 2, 5.0)
    I.ImplicitSolver(vr, ev, I.SolverConfig(**kw)).run(u)
    assert relerr(u.cpu().numpy(), u_o.numpy()) < 1e-10
    # the FP32 linear solve inside the FP64 defect correction stays close to the FP64 trajectory
    u32 = vr.BuildUDof(5)
    ev.InitializeUDOF(u32, 2, 5.0)
    I.ImplicitSolver(vr, ev, I.SolverConfig(linear_precision="fp32", **kw)).run(u32)
    assert relerr(u32.cpu().numpy(), u_o.numpy()) < 1e-5
