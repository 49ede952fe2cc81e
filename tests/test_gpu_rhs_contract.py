"""The full EvaluateRHS contract (EulerEvaluator.hpp:399-409, EulerEvaluator_EvaluateRHS.hxx:55-818)
through the C-ABI against the oracle: point values from the limited reconstruction uRec, gradients
from uRecUnlim, cellRHSAlpha on the SA source and JSource, the RHS_Ignore_Viscosity flag, the
wall-flux integral of :599-607, and the deferred error reporting.  Tolerance 1e-12 relative (FP64)."""
import numpy as np
import pytest
import torch

import oracle
from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.plate_case import plate_oracle, plate_perturbed
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _t(x):
    return torch.tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")


def _plate(p, rs="Roe"):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.flat_plate_hex(12, 10, 3, y1=1e-3, growth=1.3))
    o, far, mu, types, vals, w = plate_oracle(m, p, rs)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType=rs, muGas=mu, muModel=0, prGas=0.72))
    ev.SetBC(types, vals)
    ev.SetWallDistance(M.plate_wall_distance(vr.get("cellPP").reshape(m.n_cell, -1, 3)))
    return m, o, vr, ev, far


@pytest.mark.parametrize("p", [1, 2])
def test_limited_unlimited_pair_sa(p):
    m, o, vr, ev, far = _plate(p)
    u0, uRec0 = plate_perturbed(m, far, R=o.R)
    lim0 = uRec0 * np.random.default_rng(2).uniform(0.2, 1.0, size=(m.n_cell, 1, 1))  # a "limited" copy
    alpha0 = np.random.default_rng(3).uniform(0.5, 1.0, size=m.n_cell)
    dt0, _ = o.eval_dt(u0, 5.0)
    ref, js_ref, fw_ref = o.eval_rhs_full(u0, uRec0, lim0, alpha0)
    u, uU, uL, a = _t(u0), _t(uRec0), _t(lim0), _t(alpha0)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    rhs, js = torch.zeros_like(u), torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uL, JSource=js, uRecUnlim=uU, cellRHSAlpha=a)
    assert relerr(rhs.cpu().numpy(), ref) < TOL
    assert relerr(js.cpu().numpy(), js_ref) < TOL
    assert relerr(ev.get("fluxWallSum"), fw_ref) < TOL
    # the unlimited pair collapses to the short form
    ref2, _, _ = o.eval_rhs_full(u0, uRec0, uRec0, None)
    ev.EvaluateRHS(rhs, u, uU)
    assert relerr(rhs.cpu().numpy(), ref2) < TOL
    assert relerr(rhs.cpu().numpy(), o.eval_rhs(u0, uRec0)) < TOL


@pytest.mark.parametrize("p,rs,mu,iv,wall", [(2, "HLLEP", 1e-3, 0, 2), (1, "Roe", 0.0, 1, 3)])
def test_limited_pair_bump_and_wall_flux(p, rs, mu, iv, wall):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.bump_channel_tet(6, 4, 2))
    o, far, types, vals, w = bump_oracle(m, p, rs, mu, iv, outflow_type=6 if wall == 2 else 1, inflow_type=7 if wall == 2 else 1,
                                         wall_type=wall)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=0, ignoreVis=bool(iv)))
    ev.SetBC(types, vals)
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    lim0 = uRec0 * 0.5
    o.eval_dt(u0, 5.0)
    ref, _, fw_ref = o.eval_rhs_full(u0, uRec0, lim0)
    u = _t(u0)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    rhs, js = torch.zeros_like(u), torch.ones_like(u)
    ev.EvaluateRHS(rhs, u, _t(lim0), JSource=js, uRecUnlim=_t(uRec0))
    assert relerr(rhs.cpu().numpy(), ref) < TOL
    assert float(js.abs().max()) == 0.0  # no source Jacobian for 5 variables
    # BCWall (viscous) or BCWallInvis with muGas < 1e-99 enter the wall-flux integral
    assert np.abs(fw_ref).max() > 0
    assert relerr(ev.get("fluxWallSum"), fw_ref) < TOL
    # RHS_Dont_Update_Integration keeps the previous integral
    before = ev.get("fluxWallSum")
    ev.EvaluateRHS(rhs, u, _t(uRec0), uRecUnlim=_t(uRec0), flags=ev.RHS_Dont_Update_Integration)
    assert np.array_equal(ev.get("fluxWallSum"), before)


def test_ignore_viscosity_flag():
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.tgv_mesh(4)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=1 / 1600, muModel=0))
    ev_inv = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=1 / 1600, muModel=0, ignoreVis=True))
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    uRec = _t(np.random.default_rng(1).normal(size=(m.n_cell, vr.R, 5)) * 1e-3)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    ev_inv.EvaluateDt(dt, u, 1.0)
    a, b, c = torch.zeros_like(u), torch.zeros_like(u), torch.zeros_like(u)
    ev.EvaluateRHS(a, u, uRec, flags=ev.RHS_Ignore_Viscosity)
    ev_inv.EvaluateRHS(b, u, uRec)
    ev.EvaluateRHS(c, u, uRec)
    assert torch.equal(a, b)
    assert not torch.equal(a, c)


def test_deferred_error_reporting():
    from dndsr_b200.capi import DndsbError
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.tgv_mesh(4)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=1 / 1600, muModel=0))
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    uRec = vr.BuildURec(5)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    ref = torch.zeros_like(u)
    ev.EvaluateRHS(ref, u, uRec)
    ev.SetDeferredErrors(True)
    out = torch.zeros_like(u)
    ev.EvaluateRHS(out, u, uRec)
    ev.CheckErrors()
    assert torch.equal(out, ref)
    bad = u.clone()
    bad[5, 0] = -1.0  # a negative density, injected on the host side
    ev.EvaluateRHS(out, bad, uRec)  # returns without reading the error back
    ev.EvaluateRHS(out, u, uRec)  # a clean call does not clear the pending report
    with pytest.raises(DndsbError) as ei:
        ev.CheckErrors()
    assert ei.value.code == -4
    ev.CheckErrors()  # cleared
    ev.SetDeferredErrors(False)
    with pytest.raises(DndsbError):
        ev.EvaluateRHS(out, bad, uRec)
