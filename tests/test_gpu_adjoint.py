"""Derivatives of the residual path on the GPU.

* VJP of EvaluateRHS and of one VR sweep against central finite differences
  (step 1e-5 on O(1e-2) perturbations) of the oracle's FP64 residual, on 64 seeded
  random directions, at 1e-6 relative;
* the dual-consistency identity <w, J v> = <J^T w, v> between the forward
  (JVP) and reverse (VJP) kernels, at 1e-12 relative;
* torch.autograd through two VR sweeps and the RHS, against finite differences
  of the same composition on the oracle.
Inviscid cases on the bump channel and the vortex meshes; Navier-Stokes cases (constant
viscosity and Sutherland's law) on the periodic hex box.
The entropy-fix scale is held fixed (the oracle's EvaluateDt is called once at the
base state).  Riemann solvers with kinks at the tested states (Roe_M1's |u| fix, HLLC's
wave-speed branches) are left to the dual-consistency check.
"""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.util import VR_HQM_PY, oracle_for

pytestmark = pytest.mark.gpu

CASES = [("bump-tet-p2-Roe", "bump", 2, "Roe"), ("bump-tet-p1-HLLEP", "bump", 1, "HLLEP"), ("iv-tri-p2-HLLEP", "iv", 2, "HLLEP"),
         ("iv-quad-p3-Roe", "ivq", 3, "Roe"), ("tgv-hex-p2-HLLEP-viscous", "tgv", 2, "HLLEP"),
         ("tgv-hex-p1-Roe-sutherland", "tgvs", 1, "Roe")]


def _setup(case, p, rs):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    if case == "bump":
        m = M.bump_channel_tet(6, 4, 2)
        o, far, types, vals, w = bump_oracle(m, p, rs, 0.0, 1)
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=0.0, ignoreVis=True))
        ev.SetBC(types, vals)
        u0, uRec0 = perturbed_state(m, far, R=o.R)
    elif case in ("tgv", "tgvs"):
        # Navier-Stokes on the periodic hex box: constant viscosity, or Sutherland's law
        mu, model = (0.02, 0) if case == "tgv" else (0.05, 1)
        m = M.tgv_mesh(4)
        o = oracle_for(m, p, rs, mu=mu, muModel=model, ignoreVis=0)
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=model))
        u0 = o.init_field(3)
        uRec0 = np.random.default_rng(3).normal(size=(m.n_cell, o.R, 5)) * 0.01 * np.abs(u0).mean(0)
    else:
        m = M.iv_mesh(8) if case == "iv" else M.periodic_quad_2d(7, jitter=0.1)
        o = oracle_for(m, p, rs, mu=0.0, ignoreVis=1)
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=0.0, ignoreVis=True))
        u0 = o.init_field(2, 5.0)
        uRec0 = np.random.default_rng(3).normal(size=(m.n_cell, o.R, 5)) * 0.01
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    o.eval_dt(u0, 1.0)
    return m, o, vr, ev, u0, uRec0, u, uRec


def _dirs(rng, u0, uRec0, k):
    return [(rng.normal(size=u0.shape) * np.abs(u0).mean(0) * 1e-2, rng.normal(size=uRec0.shape) * 1e-3) for _ in range(k)]


@pytest.mark.parametrize("name,case,p,rs", CASES, ids=[c[0] for c in CASES])
def test_rhs_vjp_against_finite_differences_and_jvp(name, case, p, rs):
    m, o, vr, ev, u0, uRec0, u, uRec = _setup(case, p, rs)
    rng = np.random.default_rng(11)
    W = rng.normal(size=u0.shape)
    du, duRec = ev.EvaluateRHSVJP(torch.tensor(W, device="cuda"), u, uRec)
    du, duRec = du.cpu().numpy(), duRec.cpu().numpy()
    h = 1e-5
    worst = 0.0
    for vu, vrec in _dirs(rng, u0, uRec0, 64):
        fd = float((W * (o.eval_rhs(u0 + h * vu, uRec0 + h * vrec) - o.eval_rhs(u0 - h * vu, uRec0 - h * vrec)) / (2 * h)).sum())
        adj = float((du * vu).sum() + (duRec * vrec).sum())
        worst = max(worst, abs(adj - fd) / abs(fd))
        jvp = ev.EvaluateRHSJVP(torch.tensor(vu, device="cuda"), torch.tensor(vrec, device="cuda"), u, uRec).cpu().numpy()
        assert abs(float((W * jvp).sum()) - adj) <= 1e-12 * abs(adj)
    assert worst < 1e-6


@pytest.mark.parametrize("name,case,p,rs", CASES, ids=[c[0] for c in CASES])
def test_vr_sweep_vjp_against_finite_differences_and_jvp(name, case, p, rs):
    m, o, vr, ev, u0, uRec0, u, uRec = _setup(case, p, rs)
    rng = np.random.default_rng(5)
    C = rng.normal(size=uRec0.shape)
    vRec, vU = vr.DoReconstructionIterVJP(torch.tensor(C, device="cuda"), uRec, u)
    vRec, vU = vRec.cpu().numpy(), vU.cpu().numpy()
    h = 1e-5
    for vu, vrec in _dirs(rng, u0, uRec0, 8):
        fd = float((C * (o.vr_iter(uRec0 + h * vrec, u0 + h * vu) - o.vr_iter(uRec0 - h * vrec, u0 - h * vu)) / (2 * h)).sum())
        adj = float((vRec * vrec).sum() + (vU * vu).sum())
        assert abs(adj - fd) < 1e-6 * abs(fd)
        jv = vr.DoReconstructionIterJVP(torch.tensor(vrec, device="cuda"), torch.tensor(vu, device="cuda"), uRec, u).cpu().numpy()
        assert abs(float((C * jv).sum()) - adj) <= 1e-12 * abs(adj)


def test_autograd_through_sweeps_and_rhs():
    from dndsr_b200.autograd import residual
    m, o, vr, ev, u0, uRec0, u, uRec = _setup("bump", 2, "Roe")
    rng = np.random.default_rng(2)
    W = torch.tensor(rng.normal(size=u0.shape), device="cuda")
    ut = u.clone().requires_grad_(True)
    rt = uRec.clone().requires_grad_(True)
    J = (residual(ut, rt, vr, ev, n_sweeps=2) * W).sum()
    gu, gr = torch.autograd.grad(J, (ut, rt))

    def R_oracle(uu, rr):
        for _ in range(2):
            rr = o.vr_iter(rr, uu)
        return o.eval_rhs(uu, rr)

    h = 1e-5
    for vu, vrec in _dirs(rng, u0, uRec0, 4):
        fd = float((W.cpu().numpy() * (R_oracle(u0 + h * vu, uRec0 + h * vrec) - R_oracle(u0 - h * vu, uRec0 - h * vrec)) / (2 * h)).sum())
        adj = float((gu.cpu().numpy() * vu).sum() + (gr.cpu().numpy() * vrec).sum())
        assert abs(adj - fd) < 1e-6 * abs(fd)


def test_sa_vjp_without_wall_distance_is_reported_unsupported():
    from dndsr_b200.capi import DndsbError
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    from tests.plate_case import plate_bc, plate_state
    m = M.flat_plate_hex(6, 4, 3, y1=1e-3, growth=1.3)
    far, mu = plate_state()
    types, vals, w = plate_bc(far)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType="Roe", muGas=mu, muModel=0, prGas=0.72))
    ev.SetBC(types, vals)  # the SA source needs the wall distance, which was never set
    u, uRec = vr.BuildUDof(6), vr.BuildURec(6)
    u[:] = torch.tensor(far, device="cuda")
    with pytest.raises(DndsbError):
        ev.EvaluateRHSVJP(torch.ones_like(u), u, uRec)