"""Derivatives of the residual for the SA model and for boundary zones with a viscous flux (the forward-mode
kernels of csrc/adjoint_generic.cu), and the wall-flux (skin-friction) objective.

* VJP of EvaluateRHS against central finite differences of the oracle's FP64 residual (step 1e-5 on O(1e-2)
  perturbations, 24 seeded directions), at 1e-6 relative, and the dual-consistency identity
  <w, J v> = <J^T w, v> against the JVP, at 1e-12: the SA flat plate (6 variables: SA convective and
  diffusion fluxes, eddy viscosity, source; no-slip wall, symmetry, far-field) and the Navier-Stokes bump
  channel with no-slip and isothermal walls, inflow and pressure outflow;
* the VR sweep's VJP / JVP for 6 variables (the SA wall condition in its boundary term), the same way;
* the gradient of the wall-flux integral (EvaluateRHS.hxx:599-607, the x force on the wall: pressure
  and skin friction) against finite differences of the oracle's integral;
* the adjoint of that objective on the coupled residual of one implicit step: the transposed solve and
  the tangent solve give the same sensitivity to a residual source (1e-8)."""
import math

import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.plate_case import plate_oracle, plate_perturbed
from tests.util import VR_HQM_PY

pytestmark = pytest.mark.gpu


def _t(x):
    return torch.tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")


def _plate(p=1):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.flat_plate_hex(12, 10, 3, y1=1e-3, growth=1.3)
    o, far, mu, types, vals, w = plate_oracle(m, p, "Roe")
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType="Roe", muGas=mu, muModel=0, prGas=0.72))
    ev.SetBC(types, vals)
    ev.SetWallDistance(M.plate_wall_distance(vr.get("cellPP").reshape(m.n_cell, -1, 3)))
    u0, uRec0 = plate_perturbed(m, far, R=o.R)
    return m, o, vr, ev, u0, uRec0


def _bump_viscous(p=2, wall=2):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.bump_channel_tet(6, 4, 2)
    o, far, types, vals, w = bump_oracle(m, p, "HLLEP", 1e-3, 0, outflow_type=6, inflow_type=7, wall_type=wall)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=1e-3, muModel=0))
    ev.SetBC(types, vals)
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    return m, o, vr, ev, u0, uRec0


CASES = {"sa-plate-p1": lambda: _plate(1), "sa-plate-p2": lambda: _plate(2), "ns-bump-wall-p2": lambda: _bump_viscous(2, 2),
         "ns-bump-isothermal-p1": lambda: _bump_viscous(1, 4)}


def _dirs(rng, u0, uRec0, k):
    return [(rng.normal(size=u0.shape) * np.abs(u0).mean(0) * 1e-2, rng.normal(size=uRec0.shape) * 1e-3 * np.abs(u0).mean(0))
            for _ in range(k)]


@pytest.mark.parametrize("name", list(CASES))
def test_rhs_vjp_against_finite_differences_and_jvp(name):
    m, o, vr, ev, u0, uRec0 = CASES[name]()
    u, uRec = _t(u0), _t(uRec0)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    o.eval_dt(u0, 1.0)
    rng = np.random.default_rng(11)
    W = rng.normal(size=u0.shape)
    du, duRec = ev.EvaluateRHSVJP(_t(W), u, uRec)
    du, duRec = du.cpu().numpy(), duRec.cpu().numpy()
    h = 1e-5
    worst = 0.0
    for vu, vrec in _dirs(rng, u0, uRec0, 24):
        fd = float((W * (o.eval_rhs(u0 + h * vu, uRec0 + h * vrec) - o.eval_rhs(u0 - h * vu, uRec0 - h * vrec)) / (2 * h)).sum())
        adj = float((du * vu).sum() + (duRec * vrec).sum())
        worst = max(worst, abs(adj - fd) / abs(fd))
        jvp = ev.EvaluateRHSJVP(_t(vu), _t(vrec), u, uRec).cpu().numpy()
        assert abs(float((W * jvp).sum()) - adj) <= 1e-12 * max(abs(adj), 1e-300) * 10
    assert worst < 1e-6, worst


@pytest.mark.parametrize("p", [1, 2])
def test_vr_sweep_derivatives_six_variables(p):
    m, o, vr, ev, u0, uRec0 = _plate(p)
    u, uRec = _t(u0), _t(uRec0)
    rng = np.random.default_rng(5)
    C = rng.normal(size=uRec0.shape)
    vRec, vU = vr.DoReconstructionIterVJP(_t(C), uRec, u)
    vRec, vU = vRec.cpu().numpy(), vU.cpu().numpy()
    h = 1e-5
    worst = 0.0
    for vu, vrec in _dirs(rng, u0, uRec0, 16):
        fd = float((C * (o.vr_iter(uRec0 + h * vrec, u0 + h * vu) - o.vr_iter(uRec0 - h * vrec, u0 - h * vu)) / (2 * h)).sum())
        adj = float((vU * vu).sum() + (vRec * vrec).sum())
        worst = max(worst, abs(adj - fd) / abs(fd))
        jvp = vr.DoReconstructionIterJVP(_t(vrec), _t(vu), uRec, u).cpu().numpy()
        assert abs(float((C * jvp).sum()) - adj) <= 1e-12 * abs(adj) * 10
    assert worst < 1e-6, worst


@pytest.mark.parametrize("name", ["sa-plate-p1", "ns-bump-wall-p2"])
def test_wall_flux_gradient(name):
    m, o, vr, ev, u0, uRec0 = CASES[name]()
    nv = u0.shape[1]
    u, uRec = _t(u0), _t(uRec0)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    o.eval_dt(u0, 1.0)
    d = np.zeros(nv)
    d[1] = 1.0  # the x force on the walls
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec, flags=0, JSource=torch.zeros_like(u))
    J = float(d @ ev.get("fluxWallSum"))
    J0 = float(d @ o.eval_rhs_full(u0, uRec0, uRec0)[2])
    assert abs(J - J0) <= 1e-12 * abs(J0)
    gU, gRec = ev.WallFluxVJP(d, u, uRec)
    gU, gRec = gU.cpu().numpy(), gRec.cpu().numpy()
    assert np.abs(gU).max() > 0
    rng = np.random.default_rng(2)
    h = 1e-5
    worst = 0.0
    for vu, vrec in _dirs(rng, u0, uRec0, 16):
        fd = float(d @ (o.eval_rhs_full(u0 + h * vu, uRec0 + h * vrec, uRec0 + h * vrec)[2] -
                        o.eval_rhs_full(u0 - h * vu, uRec0 - h * vrec, uRec0 - h * vrec)[2])) / (2 * h)
        adj = float((gU * vu).sum() + (gRec * vrec).sum())
        worst = max(worst, abs(adj - fd) / max(abs(fd), 1e-300))
    assert worst < 1e-6, worst


def test_skin_friction_adjoint_matches_tangent():
    from dndsr_b200.adjoint import SteadyAdjoint
    m, o, vr, ev, u0, uRec0 = _plate(1)
    u, uRec = _t(u0), _t(uRec0)
    d = np.zeros(6)
    d[1] = 1.0
    adj = SteadyAdjoint(vr, ev, u, uRec, cfl=5.0, dt=0.05)
    gU, gRec = ev.WallFluxVJP(d, u, uRec)
    psi, lam, hist = adj.solve_adjoint(gU, gRec, restart=30, max_restarts=40, rtol=1e-11)
    assert hist[-1] <= 1e-10, hist[-1]
    rng = np.random.default_rng(8)
    sU, sRec = _t(rng.normal(size=u0.shape) * 1e-3), _t(rng.normal(size=uRec0.shape) * 1e-4)
    dU, dRec, hist2 = adj.solve_tangent(sU, sRec, restart=30, max_restarts=40, rtol=1e-11)
    assert hist2[-1] <= 1e-10
    via_adjoint = -float((psi * sU).sum() + (lam * sRec).sum())
    via_tangent = float((gU * dU).sum() + (gRec * dRec).sum())
    assert abs(via_adjoint - via_tangent) <= 1e-8 * abs(via_tangent)
