"""The reconstruction solved by GMRES (recLinearScheme 1, EulerSolver.hxx:270-339): the sweep's residual
(DoReconstructionIter with recordInc) and its linearisation (DoReconstructionIterDiff, the sweep's JVP with
the linearised boundary term) drive GMRES to the fixed point of the Jacobi sweep.  Checked against the
oracle's Jacobi iteration run to its fixed point, on the bump channel with far-field, slip-wall and
symmetry zones.  Tolerance 1e-10 relative (two different iterations reaching one fixed point)."""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p", [1, 2])
def test_rec_gmres_reaches_the_jacobi_fixed_point(p):
    from dndsr_b200 import implicit as I
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.renumber_by_color(M.bump_channel_tet(6, 4, 2))
    o, far, types, vals, w = bump_oracle(m, p, "Roe", 0.0, 1)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, muModel=0, ignoreVis=True))
    ev.SetBC(types, vals)
    u0, _ = perturbed_state(m, far, R=o.R)
    ref = np.zeros((m.n_cell, o.R, 5))
    for _ in range(3000):
        new = o.vr_iter(ref, u0)
        done = np.abs(new - ref).max() <= 1e-15 * np.abs(new).max()
        ref = new
        if done:
            break
    cfg = I.SolverConfig(recLinearScheme=1, nInternalRecStep=4, nGmresSpaceRec=30, nGmresIterRec=4, recThreshold=1e-14)
    s = I.ImplicitSolver(vr, ev, cfg)
    u = torch.tensor(u0, device="cuda")
    s._rec_gmres(u)
    assert relerr(s.uRec.cpu().numpy(), ref) < 1e-10
    # and the residual of the sweep vanishes there
    r = torch.zeros_like(s.uRec)
    vr.DoReconstructionIter(s.uRec, r, u, putIntoNew=True, recordInc=True)
    assert float(r.abs().max()) <= 1e-10 * float(s.uRec.abs().max())
