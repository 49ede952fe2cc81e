"""FP32 reconstruction sweeps inside the FP64 defect correction (SolverConfig.vrFP64Below).

The sweep's fixed point with FP32 coefficients differs from the FP64 one by the coefficients' rounding; FP64
sweeps started from the FP32 fixed point return to the FP64 fixed point, which is what switching to FP64
coefficients below the threshold relies on.  The driver switches once the stage residual falls below the
threshold and ends its stages with FP64 sweeps, on a state that agrees with the all-FP64 run as closely as
the all-FP32 one does (the stopping test on the density residual, not the sweep precision, sets that
distance on this case)."""
import numpy as np
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu


def _tgv():
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.tgv_mesh(8)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=1.0 / 1600, muModel=0))
    return m, vr, ev


def test_fp64_sweeps_leave_the_fp32_fixed_point():
    m, vr, ev = _tgv()
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)

    def sweeps(uRec, prec, n):
        new = torch.zeros_like(uRec)
        for _ in range(n):
            vr.DoReconstructionIter(uRec, new, u, putIntoNew=True, precision=prec)
            uRec, new = new, uRec
        return uRec

    r64 = sweeps(vr.BuildURec(5), "fp64", 600)
    r32 = sweeps(vr.BuildURec(5), "fp32", 600)
    # both sequences have converged: one more sweep changes nothing beyond rounding
    assert relerr(sweeps(r64.clone(), "fp64", 1).cpu().numpy(), r64.cpu().numpy()) < 1e-13
    floor = relerr(r32.cpu().numpy(), r64.cpu().numpy())
    assert 1e-10 < floor < 1e-5, floor
    back = relerr(sweeps(r32.clone(), "fp64", 600).cpu().numpy(), r64.cpu().numpy())
    assert back < 1e-12 and back < 1e-3 * floor, (back, floor)


def test_driver_switches_to_fp64_sweeps_below_the_threshold():
    m, vr, ev = _tgv()
    out, prec = {}, {}
    for name, kw in (("fp64", {}), ("switch", dict(linear_precision="fp32", vr_precision="fp32", vrFP64Below=1e-6)),
                     ("fp32", dict(linear_precision="fp32", vr_precision="fp32"))):
        u = vr.BuildUDof(5)
        ev.InitializeUDOF(u, 3)
        cfg = I.SolverConfig(odeCode=0, dtImplicit=0.05, nTimeStep=1, nTimeStepInternal=400, nTimeStepInternalMin=5, CFL=50.0, gmresCode=1,
                             nGmresSpace=30, rhsThresholdInternal=1e-11, **kw)
        s = I.ImplicitSolver(vr, ev, cfg)
        s.run(u)
        out[name], prec[name] = u.cpu().numpy(), s.vrPrec
    assert prec["switch"] == "fp64" and prec["fp32"] == "fp32" and prec["fp64"] == "fp64"
    e_switch, e_fp32 = relerr(out["switch"], out["fp64"]), relerr(out["fp32"], out["fp64"])
    assert e_switch < 1e-7 and e_switch < 2 * e_fp32 + 1e-12, (e_switch, e_fp32)
