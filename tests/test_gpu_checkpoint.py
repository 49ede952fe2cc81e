"""Resume from a state dump: the implicit solver run for 2N pseudo-iterations equals N iterations, a dump of
(u, uRec), a fresh solver restored from it and N more iterations, bit for bit (the kernels and reductions
are deterministic); the dumped state also feeds the CPU oracle, whose residual matches the GPU's."""
import numpy as np
import pytest
import torch

from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu


def test_resume_is_bit_exact_and_hands_off_to_the_oracle(tmp_path):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction, euler_bc_dir_weights
    from dndsr_b200.checkpoint import load_state
    m = M.bump_channel_tet(12, 6, 2)
    o, far, types, vals, w = bump_oracle(m, 1, "Roe_M2", 0.0, 1, intOrder=2)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1, intOrder=2)).construct(euler_bc_dir_weights(types))
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe_M2", muGas=0.0, ignoreVis=True))
    ev.SetBC(types, vals)
    n = 40

    def cfg():
        return I.SolverConfig(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=n, nTimeStepInternalMin=n, CFL=50.0, gmresCode=1,
                              nGmresSpace=10, rhsThresholdInternal=1e-30)

    u_ref = vr.BuildUDof(5)
    u_ref[:] = torch.tensor(far, device="cuda")
    s_ref = I.ImplicitSolver(vr, ev, cfg())
    s_ref.run(u_ref)
    s_ref.run(u_ref)
    u = vr.BuildUDof(5)
    u[:] = torch.tensor(far, device="cuda")
    s1 = I.ImplicitSolver(vr, ev, cfg())
    s1.run(u)
    p = str(tmp_path / "bump.bin")
    s1.save_state(p, u, iterations=n)
    u2 = vr.BuildUDof(5)
    s2 = I.ImplicitSolver(vr, ev, cfg())
    assert s2.restore_state(p, u2) == {"iterations": n}
    assert torch.equal(u2, u) and torch.equal(s2.uRec, s1.uRec)
    s2.run(u2)
    assert torch.equal(u2, u_ref) and torch.equal(s2.uRec, s_ref.uRec)
    # the dump on the CPU oracle
    a, b, _ = load_state(p)
    rhs = torch.zeros_like(u)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    o.eval_dt(a, 1.0)
    ev.EvaluateRHS(rhs, u, s1.uRec)
    assert relerr(rhs.cpu().numpy(), o.eval_rhs(a, b)) < 1e-12
