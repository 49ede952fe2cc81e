"""Derivatives of the residual path with respect to the mesh node coordinates, on the GPU.

The oracle's residual as a function of the node coordinates X is its whole chain run again
from perturbed coordinates: metrics, basis moments, face weights, A^-1 B / A^-1 b (its own
Jacobi-SVD pseudo-inverse), then EvaluateRHS or one VR sweep, with u, uRec and the entropy-fix
scale deltaLambdaCell held at the base state.  Checks:

* VJP (dR/dX)^T w of EvaluateRHS against central differences (step 1e-5 on unit-scale random
  directions times 1e-2 of the smallest edge) of the oracle, on 64 seeded directions, at 1e-6;
* the same for one VR sweep (8 directions);
* dual consistency <w, (dR/dX) v> = <(dR/dX)^T w, v> between the JVP (one thread per cell,
  the direction seeded on every node) and the VJP (one thread per cell and patch node), 1e-12.

Inviscid cases: the bump channel (tetrahedra with far-field, slip-wall and symmetry faces; VR
degree 1 and 2, Roe and HLLE+) and the periodic vortex meshes (triangles and quadrilaterals).
The bump generator leaves its boundary nodes on the grid, so several vertices of a cell share a
coordinate exactly and the half box max_k |x_k - bary| sits at a tie: a kink of the reference's
own geometry, where central differences average the two one-sided slopes.  Every node of the bump
test mesh is therefore moved by a seeded 2 % of the grid step first (generic position).
"""
import dataclasses

import numpy as np
import pytest
import torch

import oracle
from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.util import VR_HQM, VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu

CASES = [("bump-tet-p1-Roe", "bump", 1, "Roe"), ("bump-tet-p2-Roe", "bump", 2, "Roe"), ("bump-tet-p1-HLLEP", "bump", 1, "HLLEP"),
         ("iv-tri-p2-HLLEP", "iv", 2, "HLLEP"), ("iv-quad-p3-Roe", "ivq", 3, "Roe")]


def _oracle(case, m, p, rs):
    if case == "bump":
        o, far, types, vals, w = bump_oracle(m, p, rs, 0.0, 1)
        return o, (far, types, vals, w)
    es = dict(nVars=5, rsType=oracle.RS[rs], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=0.0, prGas=0.72, TRef=273.15,
              CSutherland=110.4, muModel=0, ignoreVis=1)
    o = oracle.Oracle(m, dict(VR_HQM, maxOrder=p), es)
    assert o.construct() == 0
    return o, None


def _setup(case, p, rs):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    if case == "bump":
        m = M.bump_channel_tet(6, 4, 2)
        step = np.array([4.0 / 6, 1.0 / 4, 0.5 / 2])
        m = dataclasses.replace(m, coords=m.coords + np.random.default_rng(23).uniform(-0.02, 0.02, m.coords.shape) * step)
    else:
        m = M.iv_mesh(8) if case == "iv" else M.periodic_quad_2d(7, jitter=0.1)
    o, extra = _oracle(case, m, p, rs)
    if case == "bump":
        far, types, vals, w = extra
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=0.0, ignoreVis=True))
        ev.SetBC(types, vals)
        u0, uRec0 = perturbed_state(m, far, R=o.R)
    else:
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=0.0, ignoreVis=True))
        u0 = o.init_field(2, 5.0)
        uRec0 = np.random.default_rng(3).normal(size=(m.n_cell, o.R, 5)) * 0.01
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    o.eval_dt(u0, 1.0)
    dl = o.get("deltaLambdaCell")

    def at(X):
        """the oracle on the same mesh with node coordinates X, deltaLambdaCell of the base state"""
        oo, _ = _oracle(case, dataclasses.replace(m, coords=X), p, rs)
        oo.set_delta_lambda(dl)
        return oo

    X = m.coords.copy()
    edges = np.linalg.norm(np.diff(m.cell_coords(), axis=1), axis=2)
    scale = 1e-2 * float(edges.min())
    if m.dim == 2:
        scale_vec = np.array([1.0, 1.0, 0.0])
    else:
        scale_vec = np.ones(3)
    return m, o, vr, ev, u0, uRec0, u, uRec, X, at, scale, scale_vec


@pytest.mark.parametrize("name,case,p,rs", CASES, ids=[c[0] for c in CASES])
def test_rhs_coordinate_vjp_against_finite_differences_and_jvp(name, case, p, rs):
    m, o, vr, ev, u0, uRec0, u, uRec, X, at, scale, sv = _setup(case, p, rs)
    rng = np.random.default_rng(17)
    W = rng.normal(size=u0.shape)
    dX = ev.EvaluateRHSVJPCoords(torch.tensor(W, device="cuda"), u, uRec).cpu().numpy()
    assert np.isfinite(dX).all() and np.abs(dX).max() > 0
    h = 1e-5
    worst = 0.0
    for _ in range(64):
        V = rng.normal(size=X.shape) * scale * sv
        fd = float((W * (at(X + h * V).eval_rhs(u0, uRec0) - at(X - h * V).eval_rhs(u0, uRec0))).sum() / (2 * h))
        adj = float((dX * V).sum())
        worst = max(worst, abs(adj - fd) / abs(fd))
        jvp = ev.EvaluateRHSJVPCoords(torch.tensor(V, device="cuda"), u, uRec).cpu().numpy()
        assert abs(float((W * jvp).sum()) - adj) <= 1e-12 * max(abs(adj), np.abs(W * jvp).sum() * 1e-3)
    assert worst < 1e-6, worst


@pytest.mark.parametrize("name,case,p,rs", CASES, ids=[c[0] for c in CASES])
def test_vr_sweep_coordinate_vjp_against_finite_differences_and_jvp(name, case, p, rs):
    m, o, vr, ev, u0, uRec0, u, uRec, X, at, scale, sv = _setup(case, p, rs)
    rng = np.random.default_rng(19)
    C = rng.normal(size=uRec0.shape)
    dX = vr.DoReconstructionIterVJPCoords(torch.tensor(C, device="cuda"), uRec, u).cpu().numpy()
    assert np.isfinite(dX).all() and np.abs(dX).max() > 0
    h = 1e-5
    for _ in range(8):
        V = rng.normal(size=X.shape) * scale * sv
        fd = float((C * (at(X + h * V).vr_iter(uRec0, u0) - at(X - h * V).vr_iter(uRec0, u0))).sum() / (2 * h))
        adj = float((dX * V).sum())
        assert abs(adj - fd) < 1e-6 * abs(fd), (adj, fd)
        jv = vr.DoReconstructionIterJVPCoords(torch.tensor(V, device="cuda"), uRec, u).cpu().numpy()
        assert abs(float((C * jv).sum()) - adj) <= 1e-12 * max(abs(adj), np.abs(C * jv).sum() * 1e-3)
    # the one-pass coupled VJP is the sum of the two
    W = rng.normal(size=u0.shape)
    Ct, Wt = torch.tensor(C, device="cuda"), torch.tensor(W, device="cuda")
    both = ev.ResidualVJPCoords(Wt, Ct, u, uRec).cpu().numpy()
    apart = (ev.EvaluateRHSVJPCoords(Wt, u, uRec) + vr.DoReconstructionIterVJPCoords(Ct, uRec, u)).cpu().numpy()
    assert relerr(both, apart) < 1e-13


def test_coordinate_derivatives_unsupported_cases_fail_loudly():
    """A viscous evaluator has no coordinate derivative yet: the call reports it, computes nothing."""
    from dndsr_b200 import capi
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.tgv_mesh(3)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=0.01))
    u = torch.ones((m.n_cell, 5), dtype=torch.float64, device="cuda")
    u[:, 4] = 3.0
    uRec = torch.zeros((m.n_cell, vr.R, 5), dtype=torch.float64, device="cuda")
    with pytest.raises(capi.DndsbError):
        ev.EvaluateRHSVJPCoords(torch.ones_like(u), u, uRec)


BUMP = M.BUMP_ZONES["bump"]
DRAG = np.array([1.0, 0.0, 0.0])


@pytest.mark.parametrize("p", [1, 2])
def test_pressure_force_coordinate_derivative_against_finite_differences(p):
    m, o, vr, ev, u0, uRec0, u, uRec, X, at, scale, sv = _setup("bump", p, "Roe")
    dX = ev.PressureForceCoords(BUMP, DRAG, u, uRec).cpu().numpy()
    assert np.abs(dX).max() > 0
    rng = np.random.default_rng(29)
    h = 1e-5
    worst = 0.0
    for _ in range(64):
        V = rng.normal(size=X.shape) * scale
        fd = (at(X + h * V).pressure_force(BUMP, DRAG, u0, uRec0) - at(X - h * V).pressure_force(BUMP, DRAG, u0, uRec0)) / (2 * h)
        worst = max(worst, abs(float((dX * V).sum()) - fd) / abs(fd))
    assert worst < 1e-6, worst


def test_shape_gradient_of_the_pressure_drag_against_the_tangent_response():
    """dJ/dX = dJ/dX|_state - psi^T dR_u/dX - lam^T dS/dX from one adjoint solve against
    <dJ/dX|_state, v> + <g, d>, with d the tangent response A d = -(dR/dX) v, in 3 directions."""
    from dndsr_b200.adjoint import SteadyAdjoint
    m, o, vr, ev, u0, uRec0, u, uRec, X, at, scale, sv = _setup("bump", 1, "Roe")
    dTau = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, u, 1.0)
    adj = SteadyAdjoint(vr, ev, u, uRec, cfl=5.0, dt=5.0 * float(dTau.max()))
    J, gU, gR = ev.PressureForce(BUMP, DRAG, u, uRec, grad=True)
    psi, lam, h_adj = adj.solve_adjoint(gU, gR, restart=32, max_restarts=60, rtol=1e-11)
    assert h_adj[-1] < 1e-11
    dJdX = ev.PressureForceCoords(BUMP, DRAG, u, uRec)
    G = adj.shape_gradient(psi, lam, dJdX)
    rng = np.random.default_rng(31)
    for _ in range(3):
        V = torch.tensor(rng.normal(size=X.shape) * scale, device="cuda")
        sU = ev.EvaluateRHSJVPCoords(V, u, uRec)
        sR = vr.DoReconstructionIterJVPCoords(V, uRec, u)
        du, dRec, h_tan = adj.solve_tangent(sU, sR, restart=32, max_restarts=60, rtol=1e-11)
        assert h_tan[-1] < 1e-11
        tangent = float((dJdX * V).sum() + (gU * du).sum() + (gR * dRec).sum())
        assert abs(float((G * V).sum()) - tangent) < 1e-8 * abs(tangent)
