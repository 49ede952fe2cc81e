"""The isentropic vortex configuration end to end on the GPU: VR degree 2 on jittered periodic
triangles, Roe flux, ESDIRK4 dual time (dt 0.01 to t = 1, 20 pseudo-iterations of one SGS pair per
stage), as the reference's IV case runs it (EulerSolver.hxx:147-1001).  The vortex is convected
with the free stream (1, 1), so the exact cell means at t = 1 are those of the initial field over
the cells shifted by (-1, -1); the L2 density error must fall at least as fast as h^2 from 16^2 to
32^2 quads (the scheme is third order in space and fourth in time)."""
import numpy as np
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.util import VR_HQM_PY

pytestmark = pytest.mark.gpu


def _density_error(n):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.iv_mesh(n)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 2, 5.0)
    cfg = I.SolverConfig(odeCode=0, dtImplicit=0.01, nTimeStep=100, nTimeStepInternal=20, nTimeStepInternalMin=20, CFL=10.0, gmresCode=0,
                         jacobiCode=1, sgsIter=0, rhsThresholdInternal=1e-12)
    I.ImplicitSolver(vr, ev, cfg).run(u)
    # exact cell means at t = 1: the initial field over the same cells moved back by the convection
    ms = M.iv_mesh(n)
    ms.coords = ms.coords - np.array([1.0, 1.0, 0.0])
    vs = VariationalReconstruction(ms, dict(VR_HQM_PY, maxOrder=2)).construct()
    es = EulerEvaluator(vs, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    ue = vs.BuildUDof(5)
    es.InitializeUDOF(ue, 2, 5.0)
    vol = torch.tensor(vr.get("volume"), device="cuda")
    return float(torch.sqrt((vol * (u[:, 0] - ue[:, 0]) ** 2).sum() / vol.sum()))


def test_vortex_converges_at_least_second_order():
    e16, e32 = _density_error(16), _density_error(32)
    print(f"isentropic vortex, t = 1: L2 density error {e16:.3e} (16^2 quads), {e32:.3e} (32^2), order {np.log2(e16 / e32):.2f}")
    assert np.isfinite(e16) and np.isfinite(e32)
    assert e32 < 1e-2
    assert e16 / e32 > 4.0, (e16, e32)


def test_taylor_green_dissipation_rate_at_t0():
    """The TGV output quantity: the kinetic-energy dissipation rate -dE_k/dt at t = 0 from the RHS,
    E_k = sum_c V_c |m|^2 / (2 rho) / sum_c V_c, against the oracle's RHS (1e-10).  It is positive and
    above the viscous dissipation of the initial field, 3 mu / 4: at Mach 0.1 the HLLE+ flux adds
    numerical dissipation of the same order on 24^3 cells, identically in the oracle."""
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    from tests.util import oracle_for
    mu, n = 1.0 / 1600, 24
    m = M.tgv_mesh(n)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=mu, muModel=0, prGas=0.72))
    u, uRec, tmp = vr.BuildUDof(5), vr.BuildURec(5), vr.BuildURec(5)
    ev.InitializeUDOF(u, 3)
    for _ in range(20):
        vr.DoReconstructionIter(uRec, tmp, u, putIntoNew=False)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    vol = torch.tensor(vr.get("volume"), device="cuda")

    def dEk(U, R):
        rho, mom = U[:, 0], U[:, 1:4]
        return float((vol * ((mom * R[:, 1:4]).sum(1) / rho - 0.5 * (mom * mom).sum(1) / rho ** 2 * R[:, 0])).sum() / vol.sum())

    rate = -dEk(u, rhs)
    o = oracle_for(m, 2, "HLLEP", mu=mu, ignoreVis=0)
    u0 = u.cpu().numpy()
    o.eval_dt(u0, 1.0)
    r0 = torch.tensor(o.eval_rhs(u0, uRec.cpu().numpy()), device="cuda")
    assert abs(rate - (-dEk(u, r0))) < 1e-10 * abs(rate)
    print(f"TGV -dEk/dt at t = 0 on {n}^3: {rate:.6e} (viscous part of the initial field {0.75 * mu:.6e})")
    assert rate > 0.75 * mu
