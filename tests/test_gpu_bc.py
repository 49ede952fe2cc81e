"""Boundary faces on the GPU against the oracle: the bump channel with far-field,
slip-wall, symmetry and outflow zones, and viscous cases with inflow, pressure-outflow,
no-slip and isothermal walls (setup arrays, VR sweeps with GetBoundaryRHS,
local time step, right-hand side, LU-SGS operators and the native linear solve).
Tolerance 1e-12 relative for FP64 operators."""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12

# (name, p, Riemann solver, mu, ignoreVis, outflow type, intOrder, inflow type, bump-wall type)
CASES = [("p1-Roe-euler", 1, "Roe", 0.0, 1, 1, 5, 1, 3), ("p2-Roe-euler", 2, "Roe", 0.0, 1, 1, 5, 1, 3),
         ("p2-HLLEP-ns-bcout", 2, "HLLEP", 1e-3, 0, 5, 5, 1, 3), ("p3-RoeM1-euler", 3, "Roe_M1", 0.0, 1, 1, 5, 1, 3),
         ("p1-Roe-euler-int2", 1, "Roe", 0.0, 1, 1, 2, 1, 3),
         # viscous boundary fluxes: BCIn inflow, BCOutP pressure outflow, BCWallIsothermal / BCWall no-slip bump
         ("p1-Roe-ns-in-outp-isothermal", 1, "Roe", 1e-3, 0, 6, 5, 7, 4), ("p2-HLLEP-ns-in-outp-wall", 2, "HLLEP", 1e-3, 0, 6, 5, 7, 2)]


def _setup(p, rs, mu, ignoreVis, outflow, intOrder=5, inflow=1, wall=3):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.bump_channel_tet(6, 4, 2))
    o, far, types, vals, w = bump_oracle(m, p, rs, mu, ignoreVis, outflow_type=outflow, intOrder=intOrder, inflow_type=inflow,
                                         wall_type=wall)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p, intOrder=intOrder)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=0, ignoreVis=bool(ignoreVis)))
    ev.SetBC(types, vals)
    return m, o, vr, ev, far


@pytest.mark.parametrize("name,p,rs,mu,iv,outflow,intOrder,inflow,wall", CASES, ids=[c[0] for c in CASES])
def test_boundary_operators(name, p, rs, mu, iv, outflow, intOrder, inflow, wall):
    m, o, vr, ev, far = _setup(p, rs, mu, iv, outflow, intOrder, inflow, wall)
    for nm in ["faceWeight", "matrixA", "matrixAAInvB", "vectorAInvB"]:
        assert relerr(vr.get(nm), o.get(nm)) < TOL, nm
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    new = torch.zeros_like(uRec)
    for kw in [dict(), dict(recordInc=True), dict(recordInc=True, uRecIsZero=True)]:
        vr.DoReconstructionIter(uRec, new, u, putIntoNew=True, **kw)
        assert relerr(new.cpu().numpy(), o.vr_iter(uRec0, u0, **kw)) < TOL, kw
    vr.DoReconstructionIter(uRec, new, u, putIntoNew=True, precision="fp32")
    assert relerr(new.cpu().numpy(), o.vr_iter(uRec0, u0)) < 1e-6
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    d0, _ = o.eval_dt(u0, 5.0)
    assert relerr(dt.cpu().numpy(), d0) < TOL
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    assert relerr(rhs.cpu().numpy(), o.eval_rhs(u0, uRec0)) < TOL
    # LU-SGS operators skip boundary faces like the reference (scalar Jacobian)
    jd = torch.zeros_like(dt)
    ev.LUSGSMatrixInit(jd, dt, 0.1, 0.5)
    assert relerr(jd.cpu().numpy(), o.lusgs_init(d0, 0.1, 0.5)) < TOL
    x0 = np.random.default_rng(9).normal(size=u0.shape)
    Ax = torch.zeros_like(u)
    ev.LUSGSMatrixVec(0.5, u, torch.tensor(x0, device="cuda"), jd, Ax)
    assert relerr(Ax.cpu().numpy(), o.lusgs_matvec(0.5, u0, x0, o.lusgs_init(d0, 0.1, 0.5))) < TOL


def test_boundary_table_is_required_and_checked():
    from dndsr_b200.capi import DndsbError
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.bump_channel_tet(4, 2, 2)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    u, uRec = vr.BuildUDof(5), vr.BuildURec(5)
    u[:, 0], u[:, 4] = 1.0, 2.5
    with pytest.raises(DndsbError):
        ev.EvaluateRHS(torch.zeros_like(u), u, uRec)
    with pytest.raises(DndsbError):
        vr.DoReconstructionIter(uRec, torch.zeros_like(uRec), u)
    with pytest.raises(DndsbError):  # a boundary zone without a type
        ev.SetBC([0, 1, 1, 3, 3, 9, 0], np.zeros((7, 5)))
    with pytest.raises(DndsbError):  # an unknown type
        ev.SetBC([0, 1, 1, 3, 3, 9, 42], np.zeros((7, 5)))
