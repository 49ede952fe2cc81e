"""WBAP_C limiter on the GPU against the oracle, through the C-ABI: the smooth indicator and the
limited reconstruction (VariationalReconstruction_LimiterProcedure.hxx:40-334 with the
characteristic projections of EulerSolver.hxx:466-505), on tetrahedra (bump channel, far-field /
wall / symmetry faces) and periodic hexahedra, VR degree 1 and 2, with a density and energy jump
across a plane plus random reconstruction noise; with and without ifAll.  Per-call parity 1e-12;
an exactly linear field is left unchanged on the device as in the oracle."""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.util import VR_HQM_PY, oracle_for, relerr

pytestmark = pytest.mark.gpu


def _case(kind, p):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.bump_channel_tet(8, 4, 3) if kind == "tet" else M.tgv_mesh(6)
    o = oracle_for(m, p, "Roe", mu=0.0, ignoreVis=1)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    u = np.tile(np.array([1.0, 0.2, 0.1, 0.05, 3.0]), (m.n_cell, 1))
    X = m.cell_coords().mean(1)
    jump = X[:, 0] > (0.0 if kind == "tet" else np.pi)
    u[jump, 0] *= 3.0
    u[jump, 4] *= 3.0
    uRec = np.random.default_rng(4).normal(size=(m.n_cell, o.R, 5)) * 2e-2
    return m, o, vr, ev, u, uRec


@pytest.mark.parametrize("kind,p", [("tet", 1), ("tet", 2), ("hex", 1), ("hex", 2)])
def test_smooth_indicator_and_wbap_limiter_match_the_oracle(kind, p):
    m, o, vr, ev, u0, uRec0 = _case(kind, p)
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    si = vr.DoCalculateSmoothIndicator(u, uRec)
    si0 = o.smooth_indicator(u0, uRec0)
    assert relerr(si.cpu().numpy(), si0) < 1e-12
    assert int((si0 >= 0.01).sum()) > 0  # at degree 2 the maxOrder^2 factor can put every cell above the threshold
    for ifAll in (False, True):
        out = torch.empty_like(uRec)
        for _ in range(2):  # the second call reuses the device matrixSecondary
            ev.DoLimiterWBAP_C(u, uRec, si, out, 0.01, 10.0, ifAll)
        ref = o.limiter_wbap_c(u0, uRec0, si0, 0.01, 10.0, ifAll)
        assert relerr(out.cpu().numpy(), ref) < 1e-12
        assert not np.array_equal(ref, uRec0)


def test_linear_field_is_left_unchanged_on_the_device():
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.bump_channel_tet(6, 4, 2)
    o = oracle_for(m, 2, "Roe", mu=0.0, ignoreVis=1)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    bary = o.get("cellBary").reshape(-1, 3)
    L = o.get("cellHBox").reshape(-1, 3).max(1)
    g = np.array([[0.1, 0.05, -0.02, 0.0, 0.3], [0.02, -0.1, 0.0, 0.05, 0.2], [0.0, 0.03, 0.1, 0.0, -0.1]])
    u0 = np.array([1.0, 0.2, 0.1, 0.05, 3.0]) + bary @ g
    uRec0 = np.zeros((m.n_cell, o.R, 5))
    for d in range(3):
        uRec0[:, d, :] = g[d] * L[:, None]
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    si = vr.DoCalculateSmoothIndicator(u, uRec)
    out = torch.empty_like(uRec)
    ev.DoLimiterWBAP_C(u, uRec, si, out, 0.01, 10.0, True)
    assert float(si.max()) < 1e-12
    assert relerr(out.cpu().numpy(), uRec0) < 1e-13


def test_implicit_solver_with_the_limiter():
    """useLimiter in the implicit solver: with a threshold no cell reaches, the run equals the
    unlimited one bit for bit; with every cell limited it stays finite and differs."""
    from dndsr_b200 import implicit as I
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.tgv_mesh(6)
    runs = []
    for lim, thr in ((False, 0.01), (True, 1e30), (True, 0.0)):
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1)).construct()
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=0.0, ignoreVis=True))
        u = vr.BuildUDof(5)
        ev.InitializeUDOF(u, 3)
        cfg = I.SolverConfig(odeCode=0, dtImplicit=0.05, nTimeStep=2, nTimeStepInternal=4, useLimiter=lim, smoothThreshold=thr)
        I.ImplicitSolver(vr, ev, cfg).run(u)
        runs.append(u.cpu().numpy())
    assert np.array_equal(runs[0], runs[1])
    assert np.isfinite(runs[2]).all() and not np.array_equal(runs[0], runs[2])
