"""DoReconstructionIter with SORInstead on the GPU against the oracle's sequential SOR sweep
(VariationalReconstruction_Reconstruction.hxx:534-611): in place, colour by colour, on colour-numbered meshes with
boundary faces (tetrahedra, every Euler boundary type of the bump) and periodic hexahedra; putIntoNew semantics;
FP32 coefficients refused.  Tolerance 1e-12 relative."""
import numpy as np
import pytest
import torch

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.util import VR_HQM_PY, oracle_for, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mesh,p", [("bump", 1), ("bump", 2), ("tgv", 2)])
def test_sor_sweep_matches_oracle(mesh, p):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    if mesh == "bump":
        m = M.renumber_by_color(M.bump_channel_tet(6, 4, 2))
        o, far, types, vals, w = bump_oracle(m, p, "Roe", 0.0, 1)
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p, SORInstead=True)).construct(w)
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
        ev.SetBC(types, vals)
        u0, uRec0 = perturbed_state(m, far, R=o.R)
    else:
        m = M.renumber_by_color(M.tgv_mesh(4))
        o = oracle_for(m, p, "HLLEP", 1e-3, ignoreVis=0)
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p, SORInstead=True)).construct()
        u0 = o.init_field(3)
        uRec0 = 0.05 * np.random.default_rng(4).normal(size=(m.n_cell, o.R, 5))
    u = torch.tensor(u0, device="cuda")
    uRec = torch.tensor(uRec0, device="cuda")
    other = torch.full_like(uRec, 3.0)
    ref = uRec0.copy()
    for it in range(5):
        vr.DoReconstructionIter(uRec, other, u, putIntoNew=False)  # in place on uRec, other untouched
        ref = o.vr_iter_sor(ref, u0)
        assert relerr(uRec.cpu().numpy(), ref) < 1e-12, it
    assert torch.all(other == 3.0)
    # putIntoNew: the result lands in uRecNew, uRec takes uRecNew's previous contents (the reference's swap)
    before = uRec.clone()
    vr.DoReconstructionIter(uRec, other, u, putIntoNew=True)
    assert relerr(other.cpu().numpy(), o.vr_iter_sor(before.cpu().numpy(), u0)) < 1e-12
    assert torch.all(uRec == 3.0)
    from dndsr_b200.capi import DndsbError
    with pytest.raises(DndsbError):
        vr.DoReconstructionIter(other, uRec, u, putIntoNew=True, precision="fp32")
