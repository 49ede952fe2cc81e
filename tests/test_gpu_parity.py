"""GPU kernels vs the CPU oracle, through the C-ABI (include/dndsb.h).

Tolerance: 1e-12 relative for FP64 operators (the per-call residual parity
bound of the target), 1e-6 for FP32-coefficient VR sweeps.
"""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.util import VR_HQM_PY, oracle_for, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12

CASES = [
    ("iv-tri-p2-Roe", lambda: M.iv_mesh(8), 2, 2, "Roe", 1e-3),
    ("iv-tri-p3-HLLC", lambda: M.iv_mesh(6), 3, 2, "HLLC", 0.0),
    ("iv-quad-p1-RoeM1", lambda: M.periodic_quad_2d(7, jitter=0.1), 1, 2, "Roe_M1", 1e-3),
    ("tgv-hex-p2-HLLEP", lambda: M.tgv_mesh(4), 2, 3, "HLLEP", 1 / 1600),
    ("tgv-hex-p1-RoeM1", lambda: M.tgv_mesh(5), 1, 3, "Roe_M1", 0.01),
    ("tgv-hex-p3-Roe", lambda: M.tgv_mesh(4), 3, 3, "Roe", 1 / 1600),
]


def _setup(mk, p, rs, mu):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(mk())
    o = oracle_for(m, p, rs, mu)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=rs, muGas=mu, muModel=0))
    return m, o, vr, ev


def _t(x):
    return torch.tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("name,mk,p,kind,rs,mu", CASES, ids=[c[0] for c in CASES])
def test_setup_arrays(name, mk, p, kind, rs, mu):
    m, o, vr, ev = _setup(mk, p, rs, mu)
    for nm in ["volume", "cellBary", "cellJDet", "faceArea", "faceJDet", "faceNorm", "faceMeanNorm", "smoothRatio", "baseMoment",
               "faceWeight", "matrixA", "matrixAAInvB", "vectorAInvB"]:
        assert relerr(vr.get(nm), o.get(nm)) < TOL, nm


@pytest.mark.parametrize("name,mk,p,kind,rs,mu", CASES, ids=[c[0] for c in CASES])
def test_hot_path_operators(name, mk, p, kind, rs, mu):
    m, o, vr, ev = _setup(mk, p, rs, mu)
    u0 = o.init_field(kind, 5.0)
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, kind, 5.0)
    assert relerr(u.cpu().numpy(), u0) < TOL
    u = _t(u0)
    rng = np.random.default_rng(7)
    uRec0 = rng.normal(size=(m.n_cell, o.R, 5)) * 0.01 * np.abs(u0).mean(0)
    uRec = _t(uRec0)
    new = torch.zeros_like(uRec)
    # VR sweep: plain, recordInc, recordInc from zero, FP32 coefficients
    vr.DoReconstructionIter(uRec, new, u, putIntoNew=True)
    assert relerr(new.cpu().numpy(), o.vr_iter(uRec0, u0)) < TOL
    vr.DoReconstructionIter(uRec, new, u, putIntoNew=True, recordInc=True)
    assert relerr(new.cpu().numpy(), o.vr_iter(uRec0, u0, recordInc=True)) < TOL
    vr.DoReconstructionIter(uRec, new, u, putIntoNew=True, recordInc=True, uRecIsZero=True)
    assert relerr(new.cpu().numpy(), o.vr_iter(uRec0, u0, recordInc=True, uRecIsZero=True)) < TOL
    vr.DoReconstructionIter(uRec, new, u, putIntoNew=True, precision="fp32")
    assert relerr(new.cpu().numpy(), o.vr_iter(uRec0, u0)) < 1e-6
    # putIntoNew = False swaps the buffers like the reference
    a, b = uRec.clone(), torch.zeros_like(uRec)
    vr.DoReconstructionIter(a, b, u, putIntoNew=False)
    assert relerr(a.cpu().numpy(), o.vr_iter(uRec0, u0)) < TOL and relerr(b.cpu().numpy(), uRec0) == 0
    # local time step and spectral radii
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    mn = ev.EvaluateDt(dt, u, 5.0)
    dt0, mn0 = o.eval_dt(u0, 5.0)
    assert relerr(dt.cpu().numpy(), dt0) < TOL and abs(mn - mn0) <= TOL * mn0
    assert relerr(ev.get("lambdaFace"), o.get("lambdaFace")) < TOL
    assert relerr(ev.get("deltaLambdaCell"), o.get("deltaLambdaCell")) < TOL
    # right-hand side
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    r0 = o.eval_rhs(u0, uRec0)
    assert relerr(rhs.cpu().numpy(), r0) < TOL
    # LU-SGS: diagonal, forward sweep from zero, backward sweep, matvec
    jd = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.LUSGSMatrixInit(jd, dt, 0.01, 1.0)
    jd0 = o.lusgs_init(dt0, 0.01, 1.0)
    assert relerr(jd.cpu().numpy(), jd0) < TOL
    z = np.zeros_like(u0)
    x0, xn = _t(z), _t(z)
    s = ev.UpdateSGS(1.0, _t(r0), u, x0, xn, _t(jd0), True, True, True)
    o1, s0 = o.update_sgs(1.0, r0, u0, z, z, jd0, True, True, True)
    assert relerr(xn.cpu().numpy(), o1) < TOL and relerr(s, s0) < TOL
    x1 = xn.clone()
    s = ev.UpdateSGS(1.0, _t(r0), u, x1, xn, _t(jd0), False, True, False)
    o2, s0 = o.update_sgs(1.0, r0, u0, o1, o1, jd0, False, True, False)
    assert relerr(xn.cpu().numpy(), o2) < TOL and relerr(s, s0) < TOL
    Au = torch.zeros_like(u)
    ev.LUSGSMatrixVec(1.0, u, xn, _t(jd0), Au)
    assert relerr(Au.cpu().numpy(), o.lusgs_matvec(1.0, u0, o2, jd0)) < TOL
    nrm = ev.EvaluateNorm(_t(r0), 1, True)
    assert relerr(nrm, (np.abs(r0) * o.get("volume")[:, None]).sum(0)) < TOL


def test_determinism_bitwise():
    """Same inputs twice give bit-identical RHS and reductions (no atomics in the data path)."""
    m, o, vr, ev = _setup(lambda: M.tgv_mesh(6), 2, "HLLEP", 1 / 1600)
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    uRec = vr.BuildURec(5)
    new = torch.zeros_like(uRec)
    vr.DoReconstructionIter(uRec, new, u, putIntoNew=True)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    r1, r2 = torch.zeros_like(u), torch.zeros_like(u)
    ev.EvaluateRHS(r1, u, new)
    ev.EvaluateRHS(r2, u, new)
    assert torch.equal(r1, r2)
    assert np.array_equal(ev.EvaluateNorm(r1, 1, True), ev.EvaluateNorm(r2, 1, True))


def test_nonphysical_state_reports_error():
    """A negative density is reported as DNDSB_E_NONPHYSICAL, not a trap (host-side fault injection)."""
    from dndsr_b200.capi import DndsbError
    m, o, vr, ev = _setup(lambda: M.tgv_mesh(4), 1, "Roe", 0.01)
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    u[3, 0] = -1.0
    rhs = torch.zeros_like(u)
    with pytest.raises(DndsbError) as e:
        ev.EvaluateRHS(rhs, u, vr.BuildURec(5))
    assert e.value.code in (-3, -4)
