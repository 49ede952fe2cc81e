"""The reference's one-Newton-step regression cases (test/cpp/Euler/test_EulerEvaluator.cpp:120-330).

runOneNewtonStep (:120-226) runs InitializeUDOF -> FixUMaxFilter -> EvaluateDt -> EvaluateRHS with
uRec = 0 -> EvaluateNorm(L1, volume-weighted) -> LUSGSMatrixInit(dt = 1e100, alphaDiag = 1) ->
UpdateLUSGSForward + UpdateLUSGSBackward from a zero increment -> EvaluateNorm(L2).  The golden
values sit in tests/golden/reference_goldens.json ("newton_step_iv", "newton_step_box").
"""
import json
import os

import numpy as np

from dndsr_b200 import mesh as M

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_goldens.json")))

# IV10_10 with the case settings of cases/euler/euler_config_IV.json (maxOrder 1, intOrder 3 overrides)
IV = dict(mesh=lambda: M.periodic_quad_2d(10, L=10.0, jitter=0.0), rs="Roe_M1", rsMeanValueEig=1, CFL=100.0,
          vr_oracle=dict(maxOrder=1, intOrder=3, jacobiRelax=1.0, SORInstead=0, scaleType=1, scaleMultiplier=1.0, dirWeightScheme=1,
                         geomWeightScheme=1, geomWeightBias=1.0, geomWeightPower=0.5, bcWeight=1.0),
          vr_py=dict(maxOrder=1, intOrder=3, scaleType="BaryDiff", dirWeightScheme="HQM_OPT", geomWeightScheme="HQM_SD",
                     geomWeightBias=1.0, geomWeightPower=0.5),
          gold=GOLD["newton_step_iv"])
# Uniform32_3D_Periodic with cases/euler3D/euler3D_config_Box.json (maxOrder 1, intOrder 3, default functional)
BOX = dict(mesh=lambda: M.periodic_hex_3d(32, L=1.0, jitter=0.0), rs="HLLC", rsMeanValueEig=0, CFL=10.0,
           vr_oracle=dict(maxOrder=1, intOrder=3, jacobiRelax=1.0, SORInstead=0, scaleType=1, scaleMultiplier=1.0, dirWeightScheme=0,
                          geomWeightScheme=0, geomWeightBias=0.0, geomWeightPower=0.5, bcWeight=1.0),
           vr_py=dict(maxOrder=1, intOrder=3),
           gold=GOLD["newton_step_box"])
CASES = {"iv": IV, "box": BOX}

# idealGasProperty of both cases (muGas 1e-200 with Sutherland's law: inviscid in effect)
GAS = dict(gamma=1.4, Rgas=289.0, muGas=1e-200, prGas=0.72, TRef=273.15, CSutherland=110.4, muModel=1)


def initial_state(case, bary, oracle_obj=None, init_field=None):
    """InitializeUDOF of the case: the PP isentropic vortex 203 (chi = 10.0828, quadrature-averaged) for
    IV; far-field state plus the box initializer (cell barycentre strictly inside) for Box."""
    g = case["gold"]
    if "chi" in g:
        return init_field(2, g["chi"])
    u = np.tile(np.asarray(g["farFieldStaticValue"], dtype=np.float64), (bary.shape[0], 1))
    b = g["boxInitializer"]
    inside = ((bary[:, 0] > b["x0"]) & (bary[:, 0] < b["x1"]) & (bary[:, 1] > b["y0"]) & (bary[:, 1] < b["y1"]) &
              (bary[:, 2] > b["z0"]) & (bary[:, 2] < b["z1"]))
    u[inside] = b["v"]
    return u


def norms(rhs, inc, vol):
    """(rhsDensity: volume-weighted L1 of the density residual, incL2: 2-norm of the per-variable L2
    norms of the increment), as EvaluateNorm(resNorm, rhs, 1, true) and EvaluateNorm(incNorm, xinc, 2, false)."""
    rhs_l1 = (np.abs(rhs) * vol[:, None]).sum(0)
    inc_l2 = np.sqrt((inc * inc).sum(0))
    return float(rhs_l1[0]), float(np.linalg.norm(inc_l2))
