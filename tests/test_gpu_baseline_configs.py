"""The benchmark configurations run end to end on the GPU and on the oracle with the same driver, compared
along the trajectory (the per-call parity tests only cover single operator calls on small meshes).

C1: isentropic vortex (strength 5) on periodic [0,10]^2, 64 x 64 quads split into triangles with +-10 %
    jitter, VR degree 2, Roe, ESDIRK4 with dt = 0.01 and 20 pseudo-iterations of one LU-SGS pair per stage,
    100 steps (t = 1).  The mesh is numbered colour by colour, so the GPU's colour-parallel Gauss-Seidel
    sweep equals the oracle's sequential one.  Checked at steps 0, 50 and 100: the residual at the
    oracle's state (1e-12, the per-call bound) and the state itself (1e-8, the converged-state bound),
    and the L2 density error against the exact convected vortex.
C2: Taylor-Green vortex (Re 1600, Mach 0.1) on 24^3 jittered hexahedra, VR degree 2, HLLE+ with the
    compact viscous flux, ESDIRK4 (dt 0.05, 8 pseudo-iterations of one LU-SGS pair per stage) for 20
    steps: the kinetic-energy history E_k(t) and the dissipation rate -dE_k/dt, GPU against oracle (1e-8).
C3 (reduced): the steady transonic bump of the steady configuration (BCFar in/out, BCWallInvis floor and
    ceiling, BCSym sides, Mach 0.8, VR degree 1, Roe_M2) on 2,304 tetrahedra, BDF1 at CFL 200 with GMRES(30)
    preconditioned by one LU-SGS pair, 4,000 pseudo-iterations from the free stream on each side (a residual
    drop near 1e-10): the GPU's converged state against the oracle's (1e-8, the converged-state bound), the
    GPU solving with its native FP64 and FP32 linear solves, the oracle with the restated GMRES on its own
    operators.
The runs take minutes on the oracle side (OpenMP on the host cores)."""
import dataclasses

import numpy as np
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.oracle_driver import OracleEval, OracleVR
from tests.util import VR_HQM_PY, oracle_for, relerr

pytestmark = pytest.mark.gpu


def _vortex_exact(m):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    ms = dataclasses.replace(m, coords=m.coords - np.array([1.0, 1.0, 0.0]))
    vs = VariationalReconstruction(ms, dict(VR_HQM_PY, maxOrder=2)).construct()
    es = EulerEvaluator(vs, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    ue = vs.BuildUDof(5)
    es.InitializeUDOF(ue, 2, 5.0)
    return ue.cpu().numpy()


def _l2(u, ue, vol):
    return float(np.sqrt((vol * (u[:, 0] - ue[:, 0]) ** 2).sum() / vol.sum()))


def test_c1_vortex_trajectory_matches_oracle():
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.iv_mesh(64))
    o = oracle_for(m, 2, "Roe", 0.0, ignoreVis=1)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
    kw = dict(odeCode=0, dtImplicit=0.01, nTimeStep=50, nTimeStepInternal=20, nTimeStepInternalMin=20, CFL=10.0, gmresCode=0, jacobiCode=1,
              sgsIter=0, rhsThresholdInternal=1e-12)
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 2, 5.0)
    u_o = torch.tensor(o.init_field(2, 5.0))
    assert relerr(u.cpu().numpy(), u_o.numpy()) < 1e-12
    s_g = I.ImplicitSolver(vr, ev, I.SolverConfig(**kw))
    s_o = I.ImplicitSolver(OracleVR(o), OracleEval(o), I.SolverConfig(**kw))
    vol = o.get("volume")
    ue = _vortex_exact(m)
    rhs = torch.zeros_like(u)
    for step in (0, 50, 100):
        if step:
            s_g.run(u)
            s_o.run(u_o)
        # the residual at the oracle's state and reconstruction, GPU against oracle
        uo = u_o.numpy()
        rec = s_o.uRec.numpy()
        o.eval_dt(uo, 10.0)
        ref = o.eval_rhs(uo, rec)
        dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
        ev.EvaluateDt(dt, u_o.cuda(), 10.0)
        ev.EvaluateRHS(rhs, u_o.cuda(), s_o.uRec.cuda())
        assert relerr(rhs.cpu().numpy(), ref) < 1e-12, step
        assert relerr(u.cpu().numpy(), uo) < 1e-8, step
        eg, eo = _l2(u.cpu().numpy(), ue, vol), _l2(uo, ue, vol)
        print(f"C1 step {step}: L2 density error GPU {eg:.6e} oracle {eo:.6e}")
        if step:
            assert abs(eg - eo) <= 1e-8 * eo


def test_c2_tgv_dissipation_history_matches_oracle():
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    mu = 1.0 / 1600
    m = M.renumber_by_color(M.tgv_mesh(24))
    o = oracle_for(m, 2, "HLLEP", mu)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=mu, muModel=0, prGas=0.72))
    kw = dict(odeCode=0, dtImplicit=0.05, nTimeStep=1, nTimeStepInternal=8, nTimeStepInternalMin=8, CFL=10.0, gmresCode=0, jacobiCode=1,
              sgsIter=0, rhsThresholdInternal=1e-12)
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    u_o = torch.tensor(o.init_field(3))
    s_g = I.ImplicitSolver(vr, ev, I.SolverConfig(**kw))
    s_o = I.ImplicitSolver(OracleVR(o), OracleEval(o), I.SolverConfig(**kw))
    vol = o.get("volume")

    def ek(x):
        x = x.cpu().numpy() if torch.is_tensor(x) else x
        return float((vol * (x[:, 1:4] ** 2).sum(1) / (2 * x[:, 0])).sum() / vol.sum())

    hg, ho = [ek(u)], [ek(u_o)]
    for _ in range(20):
        s_g.run(u)
        s_o.run(u_o)
        hg.append(ek(u))
        ho.append(ek(u_o))
    hg, ho = np.array(hg), np.array(ho)
    rate_g, rate_o = -np.diff(hg) / 0.05, -np.diff(ho) / 0.05
    print("C2 E_k", hg[[0, 10, 20]], "dissipation rate", rate_g[[0, 9, 19]])
    assert np.all(np.abs(hg - ho) <= 1e-8 * np.abs(ho))
    assert np.all(np.abs(rate_g - rate_o) <= 1e-8 * np.abs(rate_o).max())
    assert np.all(rate_g > 0)
    assert relerr(u.cpu().numpy(), u_o.numpy()) < 1e-8


def test_c3_converged_state_matches_oracle():
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction, euler_bc_dir_weights
    from tests.bump_case import bump_oracle
    m = M.renumber_by_color(M.bump_channel_tet(16, 8, 3))
    o, far, types, vals, w = bump_oracle(m, 1, "Roe_M2", 0.0, 1, intOrder=2)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1, intOrder=2)).construct(euler_bc_dir_weights(types))
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe_M2", muGas=0.0, ignoreVis=True))
    ev.SetBC(types, vals)
    kw = dict(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=4000, nTimeStepInternalMin=4000, CFL=200.0, gmresCode=1,
              nGmresSpace=30, nGmresIter=1, sgsIter=0, rhsThresholdInternal=1e-10)
    states = {}
    for prec in ("fp64", "fp32"):
        u = vr.BuildUDof(5)
        u[:] = torch.tensor(far, device="cuda")
        cfg = I.SolverConfig(**kw, linear_precision=prec)
        I.ImplicitSolver(vr, ev, cfg).run(u)
        assert cfg.res_history[-1][2] < 1e-9, (prec, cfg.res_history[-1])
        states[prec] = u.cpu().numpy()
    u_o = torch.tensor(np.tile(far, (m.n_cell, 1)))
    cfg_o = I.SolverConfig(**kw, native_linear=False)
    I.ImplicitSolver(OracleVR(o), OracleEval(o), cfg_o).run(u_o)
    assert cfg_o.res_history[-1][2] < 1e-9, cfg_o.res_history[-1]
    for prec, ug in states.items():
        assert relerr(ug, u_o.numpy()) < 1e-8, (prec, relerr(ug, u_o.numpy()))
