"""Block-diagonal and Roe-linearised LU-SGS operators (useScalarJacobian = false, useRoeJacobian) on the GPU
against the oracle: the face eigenvalues lambdaFace0/123/4 recorded by EvaluateDt and EvaluateRHS
(EvaluateRHS.hxx:527-545, interior faces in the tuned and the generic face kernels, boundary faces in the
boundary kernel), the diagonal blocks and their inverses of LUSGSMatrixInit (EulerEvaluator.hxx:37-159,
boundary faces with the linearised ghost), UpdateSGS, UpdateLUSGSForward/Backward and LUSGSMatrixVec with the
Roe form of the neighbour increment, the native linear solve in FP64 and FP32 against the same solve
orchestrated on the oracle's operators, and a few pseudo-time iterations of the implicit driver.
Tolerance 1e-12 relative for single FP64 operators."""
import numpy as np
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.oracle_driver import OracleEval, OracleVR
from tests.util import VR_HQM_PY, oracle_for, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12

# (name, mesh, p, Riemann solver, mu, boundary types: outflow, inflow, wall)
CASES = [("bump-p1-Roe-euler", "bump", 1, "Roe", 0.0, (1, 1, 3)),
         ("bump-p2-RoeM2-euler", "bump", 2, "Roe_M2", 0.0, (1, 1, 3)),
         ("bump-p1-HLLEP-ns-in-outp-isothermal", "bump", 1, "HLLEP", 1e-3, (6, 7, 4)),
         ("bump-p2-Roe-ns-wall", "bump", 2, "Roe", 1e-3, (5, 1, 2)),
         ("tgv-p2-HLLEP-ns", "tgv", 2, "HLLEP", 1 / 1600, None),
         ("iv2d-p2-RoeM1-euler", "iv", 2, "Roe_M1", 0.0, None)]


def _setup(mesh, p, rs, mu, bt):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    iv = mu == 0
    if mesh == "bump":
        m = M.renumber_by_color(M.bump_channel_tet(6, 4, 2))
        o, far, types, vals, w = bump_oracle(m, p, rs, mu, int(iv), outflow_type=bt[0], inflow_type=bt[1], wall_type=bt[2])
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=0, ignoreVis=iv))
        ev.SetBC(types, vals)
        u0, uRec0 = perturbed_state(m, far, R=o.R)
    else:
        m = M.renumber_by_color(M.tgv_mesh(4) if mesh == "tgv" else M.iv_mesh(8))
        o = oracle_for(m, p, rs, mu, ignoreVis=int(iv))
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=0, ignoreVis=iv))
        u0 = o.init_field(3) if mesh == "tgv" else o.init_field(2, 5.0)
        uRec0 = 0.05 * np.random.default_rng(4).normal(size=(m.n_cell, o.R, 5)) * np.abs(u0[:, None, :])
        if mesh == "iv":  # 2-D: no z momentum
            uRec0[:, :, 3] = 0
    return m, o, vr, ev, u0, uRec0


@pytest.mark.parametrize("name,mesh,p,rs,mu,bt", CASES, ids=[c[0] for c in CASES])
def test_roe_jacobian_operators(name, mesh, p, rs, mu, bt):
    m, o, vr, ev, u0, uRec0 = _setup(mesh, p, rs, mu, bt)
    o.set_jacobian_mode(False, True)
    ev.SetJacobianMode(False, True)
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    d0, _ = o.eval_dt(u0, 5.0)
    assert relerr(dt.cpu().numpy(), d0) < TOL
    for nm in ("lambdaFace0", "lambdaFace123", "lambdaFace4"):  # the convective speed after EvaluateDt
        assert relerr(ev.get(nm), o.get(nm)) < TOL, nm
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    rhs0 = o.eval_rhs(u0, uRec0)
    assert relerr(rhs.cpu().numpy(), rhs0) < TOL
    for nm in ("lambdaFace0", "lambdaFace123", "lambdaFace4"):  # the Riemann eigenvalues after EvaluateRHS
        assert relerr(ev.get(nm), o.get(nm)) < TOL, nm
    jd = ev.BuildJDiag()
    assert jd.shape == (m.n_cell, 2, 5, 5)
    ev.LUSGSMatrixInit(jd, dt, 0.1, 0.5, u)
    jd0 = o.lusgs_init_block(d0, 0.1, 0.5, u0)
    assert relerr(jd[:, 0].cpu().numpy(), jd0[:, 0]) < TOL
    assert relerr(jd[:, 1].cpu().numpy(), jd0[:, 1]) < 1e-11  # inverses: different pivoting, same matrix
    x0 = np.random.default_rng(9).normal(size=u0.shape)
    x = torch.tensor(x0, device="cuda")
    Ax = torch.zeros_like(u)
    ev.LUSGSMatrixVec(0.5, u, x, jd, Ax)
    assert relerr(Ax.cpu().numpy(), o.lusgs_matvec(0.5, u0, x0, jd0)) < TOL
    out = torch.zeros_like(u)
    for fwd, gs, zero in [(True, True, False), (False, True, False), (True, False, False), (True, True, True)]:
        s = ev.UpdateSGS(0.5, rhs, u, x, out, jd, fwd, gs, zero)
        ref, s0 = o.update_sgs(0.5, rhs0, u0, x0, np.zeros_like(x0), jd0, fwd, gs, zero)
        assert relerr(out.cpu().numpy(), ref) < 1e-11, (fwd, gs, zero)
    for fwd in (True, False):
        y = torch.zeros_like(u)
        ev.UpdateLUSGSForward(0.5, rhs, u, x, jd, y) if fwd else ev.UpdateLUSGSBackward(0.5, rhs, u, x, jd, y)
        ref = o.update_lusgs(0.5, rhs0, u0, x0, np.zeros_like(x0), jd0, fwd)
        assert relerr(y.cpu().numpy(), ref) < 1e-11, fwd
    # the transposed operators keep the scalar Jacobian
    from dndsr_b200.capi import DndsbError
    with pytest.raises(DndsbError):
        ev.LUSGSMatrixVecT(0.5, u, x, jd, Ax)


def test_block_mode_without_roe_term_equals_scalar():
    m, o, vr, ev, u0, uRec0 = _setup("bump", 1, "Roe", 0.0, (1, 1, 3))
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    x = torch.tensor(np.random.default_rng(2).normal(size=u0.shape), device="cuda")
    res = {}
    for block in (False, True):
        ev.SetJacobianMode(not block, False)
        jd = ev.BuildJDiag()
        ev.LUSGSMatrixInit(jd, dt, 0.1, 0.5)
        Ax, y = torch.zeros_like(u), torch.zeros_like(u)
        ev.LUSGSMatrixVec(0.5, u, x, jd, Ax)
        ev.UpdateSGS(0.5, rhs, u, x, y, jd, True, True, False)
        z = torch.zeros_like(u)
        ev.SolveLinear(0.5, dt, 0.1, u, rhs, z, gmresCode=1, nGmresSpace=6)
        res[block] = (Ax.cpu(), y.cpu(), z.cpu())
    for a, b in zip(res[False], res[True]):
        assert relerr(b.numpy(), a.numpy()) < 1e-13


def _reference_solve(oe, u, rhs, dTau, dt, alpha, code, sgsIter, k, nIter, jacobi=1):
    """EulerSolver::solveLinear (EulerSolver.hxx:1407-1579) with doPrecondition (:1605-1657) on the oracle's operators."""
    jd = oe.BuildJDiag()
    oe.LUSGSMatrixInit(jd, dTau, dt, alpha, u)
    if jacobi == 2:
        oe.LUSGSMatrixToJacobianLU(alpha, u, jd)
    tmp = torch.zeros_like(rhs)

    def pair(b, x, zero):
        if jacobi == 2:
            for it in range(2):
                oe.LUSGSMatrixSolveJacobianLU(alpha, b, u, x, tmp, jd, zero and it == 0)
                x.copy_(tmp)
            return
        oe.UpdateSGS(alpha, b, u, x, tmp, jd, True, True, False)
        x.copy_(tmp)
        oe.UpdateSGS(alpha, b, u, x, tmp, jd, False, True, False)
        x.copy_(tmp)

    x = torch.zeros_like(rhs)
    if code in (0, 2):
        for i in range(1 + sgsIter):
            pair(rhs, x, i == 0)
    if code:
        g = I.GMRES(k, x)

        def FML(v, Mv):
            Mv.zero_()
            for i in range(1 + sgsIter):
                pair(v, Mv, i == 0)

        g.solve(lambda v, Av: oe.LUSGSMatrixVec(alpha, u, v, jd, Av), FML, lambda a, b: float((a * b).sum()), rhs, x, nIter,
                lambda i, r, rb: False)
    return x


@pytest.mark.parametrize("name,mesh,p,rs,mu,bt", [CASES[0], CASES[2], CASES[4], CASES[5]], ids=[CASES[i][0] for i in (0, 2, 4, 5)])
@pytest.mark.parametrize("code,sgsIter,k,nIter,jacobi,roe", [(0, 1, 1, 1, 1, True), (1, 0, 8, 2, 1, True), (2, 1, 5, 1, 1, True),
                                                             (0, 1, 1, 1, 2, True), (1, 0, 8, 1, 2, True), (1, 0, 8, 1, 2, False)])
def test_roe_jacobian_linear_solve(name, mesh, p, rs, mu, bt, code, sgsIter, k, nIter, jacobi, roe):
    """The native solve with the Roe Jacobian (SGS pairs or the local LU), and the local LU with the scalar Jacobian."""
    m, o, vr, ev, u0, uRec0 = _setup(mesh, p, rs, mu, bt)
    oe = OracleEval(o)
    oe.SetJacobianMode(not roe, roe)
    ev.SetJacobianMode(not roe, roe)
    ut, uRt = torch.tensor(u0), torch.tensor(uRec0)
    dTau0 = torch.zeros(m.n_cell, dtype=torch.float64)
    oe.EvaluateDt(dTau0, ut, 1e3)
    oe.EvaluateRHS(torch.zeros_like(ut), ut, uRt)  # records the eigenvalues
    rhs0 = torch.tensor(np.random.default_rng(3).normal(size=(m.n_cell, 5)))
    alpha, dt = 0.5, 10.0
    ref = _reference_solve(oe, ut, rhs0, dTau0, dt, alpha, code, sgsIter, k, nIter, jacobi)
    u, uRec, rhs = ut.cuda(), uRt.cuda(), rhs0.cuda()
    dTau = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, u, 1e3)
    ev.EvaluateRHS(torch.zeros_like(u), u, uRec)
    for prec, tol in [("fp64", 1e-10), ("fp32", 1e-5)]:
        outs = []
        for graph in (True, True, False):
            x = torch.full_like(rhs, 7.0)
            ev.SolveLinear(alpha, dTau, dt, u, rhs, x, gmresCode=code, jacobiCode=jacobi, sgsIter=sgsIter, nGmresSpace=k, nGmresIter=nIter,
                           precision=prec, useGraph=graph)
            outs.append(x.cpu())
        assert relerr(outs[0].numpy(), ref.numpy()) < tol, prec
        assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])


def test_roe_jacobian_driver_matches_oracle_driver():
    """Six BDF1 pseudo-time iterations of the steady bump (Roe, VR degree 1, CFL 50, LU-SGS and GMRES) with the
    Roe Jacobian: the GPU driver (native block linear solve) against the same driver on the oracle."""
    m, o, vr, ev, u0, uRec0 = _setup("bump", 1, "Roe", 0.0, (1, 1, 3))
    far = M.freestream(0.8)
    kw = dict(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=6, nTimeStepInternalMin=6, CFL=50.0, gmresCode=1,
              nGmresSpace=10, sgsIter=0)
    oe = OracleEval(o)
    oe.SetJacobianMode(False, True)
    ev.SetJacobianMode(False, True)
    u_o = torch.tensor(np.tile(far, (m.n_cell, 1)))
    I.ImplicitSolver(OracleVR(o), oe, I.SolverConfig(**kw)).run(u_o)
    u = torch.tensor(np.tile(far, (m.n_cell, 1)), device="cuda")
    I.ImplicitSolver(vr, ev, I.SolverConfig(**kw)).run(u)
    assert relerr(u.cpu().numpy(), u_o.numpy()) < 1e-10


@pytest.mark.parametrize("mode", ["scalar", "block", "roe"])
def test_local_lu_operators(mode):
    """LUSGSMatrixToJacobianLU + LUSGSMatrixSolveJacobianLU (block ILU(0)) against the oracle's natural-order
    factorisation on the colour-numbered bump mesh, with the scalar Jacobian (the reference's RotPeriodicIV
    setting: its diagonal as blocks), the block diagonal and the Roe Jacobian."""
    m, o, vr, ev, u0, uRec0 = _setup("bump", 1, "Roe", 0.0, (1, 1, 3))
    roe = mode == "roe"
    o.set_jacobian_mode(mode == "scalar", roe)
    ev.SetJacobianMode(mode == "scalar", roe)
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 20.0)
    d0, _ = o.eval_dt(u0, 20.0)
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    rhs0 = o.eval_rhs(u0, uRec0)
    jd = ev.BuildJDiag()
    ev.LUSGSMatrixInit(jd, dt, 1e100, 1.0, u)
    jd0 = o.lusgs_init(d0, 1e100, 1.0) if mode == "scalar" else o.lusgs_init_block(d0, 1e100, 1.0, u0)
    ev.LUSGSMatrixToJacobianLU(1.0, u, jd)
    o.jacobian_lu(1.0, u0, jd0)
    x0 = np.random.default_rng(7).normal(size=u0.shape)
    x = torch.tensor(x0, device="cuda")
    out = torch.zeros_like(u)
    for zero in (True, False):
        s = ev.LUSGSMatrixSolveJacobianLU(1.0, rhs, u, x, out, jd, zero)
        ref, s0 = o.solve_jacobian_lu(1.0, rhs0, u0, x0, jd0, zero)
        assert relerr(out.cpu().numpy(), ref) < 1e-11, zero
        assert relerr(np.asarray(s), s0) < 1e-11
    from dndsr_b200.capi import DndsbError
    with pytest.raises(DndsbError):  # uIncNew must not alias uInc
        ev.LUSGSMatrixSolveJacobianLU(1.0, rhs, u, out, out, jd, False)


def test_local_lu_driver_matches_oracle_driver():
    """The reference's Roe-Jacobian configuration (jacobiCode 2 without GMRES): six BDF1 pseudo-time iterations of
    the steady bump at CFL 50, the GPU driver (native block ILU(0) solve) against the same driver on the oracle."""
    m, o, vr, ev, u0, uRec0 = _setup("bump", 1, "Roe", 0.0, (1, 1, 3))
    far = M.freestream(0.8)
    kw = dict(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=6, nTimeStepInternalMin=6, CFL=50.0, gmresCode=0, jacobiCode=2,
              sgsIter=0)
    oe = OracleEval(o)
    oe.SetJacobianMode(False, True)
    ev.SetJacobianMode(False, True)
    u_o = torch.tensor(np.tile(far, (m.n_cell, 1)))
    I.ImplicitSolver(OracleVR(o), oe, I.SolverConfig(**kw)).run(u_o)
    u = torch.tensor(np.tile(far, (m.n_cell, 1)), device="cuda")
    I.ImplicitSolver(vr, ev, I.SolverConfig(**kw)).run(u)
    assert relerr(u.cpu().numpy(), u_o.numpy()) < 1e-10


@pytest.mark.parametrize("roe", [False, True])
def test_sa_block_operators(roe):
    """6 variables (the SA model, no-slip wall, far field): the block diagonal with the SA source Jacobian, with
    and without the Roe term, its products and sweeps, the local LU and the native solve against the oracle."""
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    from tests.plate_case import plate_oracle, plate_perturbed
    m = M.renumber_by_color(M.flat_plate_hex(12, 10, 3, y1=1e-3, growth=1.3))
    o, far, mu, types, vals, w = plate_oracle(m, 1, "Roe", 5)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1, intOrder=5)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType="Roe", muGas=mu, muModel=0, prGas=0.72))
    ev.SetBC(types, vals)
    ev.SetWallDistance(M.plate_wall_distance(vr.get("cellPP").reshape(m.n_cell, -1, 3)))
    o.set_jacobian_mode(False, roe)
    ev.SetJacobianMode(False, roe)
    u0, uRec0 = plate_perturbed(m, far, R=o.R)
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    d0, _ = o.eval_dt(u0, 5.0)
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    r0 = o.eval_rhs(u0, uRec0)
    assert relerr(rhs.cpu().numpy(), r0) < TOL
    if roe:
        for nm in ("lambdaFace0", "lambdaFace123", "lambdaFace4"):
            assert relerr(ev.get(nm), o.get(nm)) < TOL, nm
    jd = ev.BuildJDiag()
    assert jd.shape == (m.n_cell, 2, 6, 6)
    ev.LUSGSMatrixInit(jd, dt, 0.1, 0.5, u)
    jd0 = o.lusgs_init_block(d0, 0.1, 0.5, u0)
    assert relerr(jd[:, 0].cpu().numpy(), jd0[:, 0]) < TOL
    assert relerr(jd[:, 1].cpu().numpy(), jd0[:, 1]) < 1e-11
    x0 = np.random.default_rng(2).normal(size=u0.shape)
    x = torch.tensor(x0, device="cuda")
    Ax = torch.zeros_like(u)
    ev.LUSGSMatrixVec(0.5, u, x, jd, Ax)
    assert relerr(Ax.cpu().numpy(), o.lusgs_matvec(0.5, u0, x0, jd0)) < TOL
    out = torch.zeros_like(u)
    ev.UpdateSGS(0.5, rhs, u, x, out, jd, True, True, False)
    ref, _ = o.update_sgs(0.5, r0, u0, x0, np.zeros_like(x0), jd0, True, True, False)
    assert relerr(out.cpu().numpy(), ref) < 1e-11
    ev.LUSGSMatrixToJacobianLU(0.5, u, jd)
    o.jacobian_lu(0.5, u0, jd0)
    ev.LUSGSMatrixSolveJacobianLU(0.5, rhs, u, x, out, jd, False)
    ref, _ = o.solve_jacobian_lu(0.5, r0, u0, x0, jd0, False)
    assert relerr(out.cpu().numpy(), ref) < 1e-11
    oe = OracleEval(o)
    oe.SetJacobianMode(False, roe)
    refx = _reference_solve(oe, torch.tensor(u0), torch.tensor(r0), torch.tensor(d0), 0.1, 0.5, 1, 0, 6, 1, 2)
    for prec, tol in [("fp64", 1e-10), ("fp32", 1e-5)]:
        xs = torch.zeros_like(u)
        ev.SolveLinear(0.5, dt, 0.1, u, rhs, xs, gmresCode=1, nGmresSpace=6, jacobiCode=2, precision=prec)
        assert relerr(xs.cpu().numpy(), refx.numpy()) < tol, prec


def test_local_lu_with_triangles_in_the_cell_graph():
    """A 3-periodic hexahedral grid: each row of three cells is a triangle of face neighbours, so the ILU(0)
    corrections between neighbours that share a lower neighbour run (standalone local LU and native solve)."""
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.tgv_mesh(3))
    o = oracle_for(m, 1, "Roe", 1e-3, ignoreVis=0)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=1e-3, muModel=0))
    o.set_jacobian_mode(False, True)
    ev.SetJacobianMode(False, True)
    u0 = o.init_field(3)
    uRec0 = 0.02 * np.random.default_rng(1).normal(size=(m.n_cell, o.R, 5))
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 10.0)
    d0, _ = o.eval_dt(u0, 10.0)
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    r0 = o.eval_rhs(u0, uRec0)
    jd = ev.BuildJDiag()
    ev.LUSGSMatrixInit(jd, dt, 1e100, 1.0, u)
    jd0 = o.lusgs_init_block(d0, 1e100, 1.0, u0)
    ev.LUSGSMatrixToJacobianLU(1.0, u, jd)
    o.jacobian_lu(1.0, u0, jd0)
    x0 = np.random.default_rng(3).normal(size=u0.shape)
    out = torch.zeros_like(u)
    for zero in (True, False):
        ev.LUSGSMatrixSolveJacobianLU(1.0, rhs, u, torch.tensor(x0, device="cuda"), out, jd, zero)
        ref, _ = o.solve_jacobian_lu(1.0, r0, u0, x0, jd0, zero)
        assert relerr(out.cpu().numpy(), ref) < 1e-11, zero
    oe = OracleEval(o)
    oe.SetJacobianMode(False, True)
    refx = _reference_solve(oe, torch.tensor(u0), torch.tensor(r0), torch.tensor(d0), 1e100, 1.0, 1, 0, 6, 1, 2)
    xs = torch.zeros_like(u)
    ev.SolveLinear(1.0, dt, 1e100, u, rhs, xs, gmresCode=1, nGmresSpace=6, jacobiCode=2)
    assert relerr(xs.cpu().numpy(), refx.numpy()) < 1e-10
