"""FP32 reconstruction sweeps inside the FP64 defect correction (SolverConfig.vrFP64Below): a dual-time stage
run with FP32 sweep coefficients above the threshold and FP64 ones below it ends on the FP64 fixed point (the
all-FP64 run's state to 1e-9), while FP32 sweeps throughout end measurably further from it."""
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu


def test_fp32_sweeps_finish_on_the_fp64_fixed_point():
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.tgv_mesh(8)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=1.0 / 1600, muModel=0))
    out = {}
    for name, kw in (("fp64", {}), ("switch", dict(linear_precision="fp32", vr_precision="fp32", vrFP64Below=1e-6)),
                     ("fp32", dict(linear_precision="fp32", vr_precision="fp32"))):
        u = vr.BuildUDof(5)
        ev.InitializeUDOF(u, 3)
        cfg = I.SolverConfig(odeCode=0, dtImplicit=0.05, nTimeStep=1, nTimeStepInternal=400, nTimeStepInternalMin=5, CFL=50.0, gmresCode=1,
                             nGmresSpace=30, rhsThresholdInternal=1e-11, **kw)
        I.ImplicitSolver(vr, ev, cfg).run(u)
        out[name] = u.cpu().numpy()
    e_switch, e_fp32 = relerr(out["switch"], out["fp64"]), relerr(out["fp32"], out["fp64"])
    assert e_switch < 1e-9, e_switch
    assert e_fp32 > 10 * e_switch, (e_fp32, e_switch)
