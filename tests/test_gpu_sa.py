"""The SA model (6 variables) on the GPU against the oracle: a stretched hexahedral flat-plate
mesh with a no-slip adiabatic plate, symmetry planes, far-field in/outflow and periodic sides.
Covers the cell length scale of the IDDES blend, the VR sweep with the SA wall condition,
the local time step with the eddy viscosity, the RHS (SA convective and diffusion fluxes, the
source integrated at the cell Gauss points), the source Jacobian, the per-variable LU-SGS
diagonal, SGS sweeps, the matrix-vector product and the native linear solve.  The SA
restatement has no reference golden (the reference's RANS tests exclude SA)."""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.oracle_driver import OracleEval
from tests.plate_case import plate_oracle, plate_perturbed
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _setup(p, rs, intOrder=5):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.flat_plate_hex(12, 10, 3, y1=1e-3, growth=1.3))
    o, far, mu, types, vals, w = plate_oracle(m, p, rs, intOrder)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p, intOrder=intOrder)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType=rs, muGas=mu, muModel=0, prGas=0.72))
    ev.SetBC(types, vals)
    ev.SetWallDistance(M.plate_wall_distance(vr.get("cellPP").reshape(m.n_cell, -1, 3)))
    return m, o, vr, ev, far


# p=1 runs the tuned face kernel (4 and 9 points per quadrilateral face); p=2 the generic one
@pytest.mark.parametrize("p,rs,io", [(1, "Roe", 5), (1, "Roe", 3), (2, "HLLEP", 5)])
def test_sa_operators(p, rs, io):
    m, o, vr, ev, far = _setup(p, rs, io)
    assert relerr(vr.get("cellHMax"), o.get("cellHMax")) < TOL
    u0, uRec0 = plate_perturbed(m, far, R=o.R)
    u, uRec = torch.tensor(u0, device="cuda"), torch.tensor(uRec0, device="cuda")
    new = torch.zeros_like(uRec)
    vr.DoReconstructionIter(uRec, new, u, putIntoNew=True)
    assert relerr(new.cpu().numpy(), o.vr_iter(uRec0, u0)) < TOL
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    d0, _ = o.eval_dt(u0, 5.0)
    assert relerr(dt.cpu().numpy(), d0) < TOL
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, uRec)
    r0 = o.eval_rhs(u0, uRec0)
    assert relerr(rhs.cpu().numpy(), r0) < TOL
    assert relerr(rhs.cpu().numpy()[:, 5], r0[:, 5]) < TOL  # the SA equation on its own scale
    assert relerr(ev.get("jSource"), o.get("jSource")) < TOL
    jd = ev.BuildJDiag()
    ev.LUSGSMatrixInit(jd, dt, 0.1, 0.5)
    jd0 = o.lusgs_init(d0, 0.1, 0.5)
    assert jd.shape == (m.n_cell, 6) and relerr(jd.cpu().numpy(), jd0) < TOL
    x0 = np.random.default_rng(2).normal(size=u0.shape)
    Ax = torch.zeros_like(u)
    ev.LUSGSMatrixVec(0.5, u, torch.tensor(x0, device="cuda"), jd, Ax)
    assert relerr(Ax.cpu().numpy(), o.lusgs_matvec(0.5, u0, x0, jd0)) < TOL
    out = torch.zeros_like(u)
    ev.UpdateSGS(0.5, rhs, u, torch.tensor(x0, device="cuda"), out, jd, True, True, False)
    ref, _ = o.update_sgs(0.5, r0, u0, x0, np.zeros_like(x0), jd0, True, True, False)
    assert relerr(out.cpu().numpy(), ref) < TOL
    # native linear solve: FP64 against the oracle's operators, FP32 close to it
    from tests.test_gpu_linear import _reference_solve
    oe = OracleEval(o)
    refx = _reference_solve(oe, torch.tensor(u0), torch.tensor(r0), torch.tensor(d0), 0.1, 0.5, 1, 1, 0, 6, 1)
    for prec, tol in [("fp64", 1e-10), ("fp32", 1e-5)]:
        x = torch.zeros_like(u)
        ev.SolveLinear(0.5, dt, 0.1, u, rhs, x, gmresCode=1, nGmresSpace=6, precision=prec)
        assert relerr(x.cpu().numpy(), refx.numpy()) < tol, prec


def test_sa_needs_wall_distance():
    from dndsr_b200.capi import DndsbError
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.flat_plate_hex(6, 4, 3, y1=1e-3, growth=1.3)
    o, far, mu, types, vals, w = plate_oracle(m, 1)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType="Roe", muGas=mu, muModel=0))
    ev.SetBC(types, vals)
    u = torch.tensor(np.tile(far, (m.n_cell, 1)), device="cuda")
    with pytest.raises(DndsbError):
        ev.EvaluateRHS(torch.zeros_like(u), u, vr.BuildURec(6))
