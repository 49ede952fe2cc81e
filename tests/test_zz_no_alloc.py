"""The allocation-free RHS entry point against the regular one, through the C-ABI.

dndsb_eval_evaluate_rhs_noalloc serves callers that must not allocate device
memory while they evaluate residuals: its face-flux scratch is a static
device array instead of handle memory.  This file runs last (pytest collects
it after the other test files) and passes alone or after them.
"""
import numpy as np
import pytest
import torch

from dndsr_b200 import capi
from dndsr_b200 import mesh as M
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the FP64 per-call tolerance of the parity tests


def _evaluator(n, p):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.tgv_mesh(n)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=p)).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="HLLEP", muGas=1 / 1600, muModel=0))
    return m, vr, ev


def test_noalloc_rhs_matches_regular_entry_point_twice():
    m, vr, ev = _evaluator(8, 2)
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 5.0)
    rng = np.random.default_rng(3)
    for call in range(2):  # two calls in a row, different reconstructions
        uRec = torch.tensor(rng.normal(size=(m.n_cell, vr.R, 5)) * 1e-2, dtype=torch.float64, device="cuda")
        ref, got = torch.zeros_like(u), torch.full_like(u, np.nan)
        ev.EvaluateRHS(ref, u, uRec)
        handle_scratch = ev.get("faceFlux")  # the regular call's face fluxes, in handle memory
        # the allocation-free call works in the static array: evaluated at another reconstruction it
        # must leave the handle's scratch as the regular call left it
        other = torch.tensor(rng.normal(size=(m.n_cell, vr.R, 5)) * 1e-2, dtype=torch.float64, device="cuda")
        ev.EvaluateRHSNoAlloc(got, u, other)
        assert np.array_equal(ev.get("faceFlux"), handle_scratch), f"call {call}: handle scratch touched"
        ev.EvaluateRHSNoAlloc(got, u, uRec)
        torch.cuda.synchronize()
        assert relerr(got.cpu().numpy(), ref.cpu().numpy()) <= TOL, f"call {call}"


def test_noalloc_rejects_meshes_beyond_the_static_scratch():
    m, vr, ev = _evaluator(42, 1)  # 222,264 faces x 5 variables > 2^20 doubles
    assert m.n_face * 5 > capi.NOALLOC_SCRATCH_DOUBLES
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    rhs = torch.zeros_like(u)
    with pytest.raises(capi.DndsbError) as e:
        ev.EvaluateRHSNoAlloc(rhs, u, vr.BuildURec(5))
    assert e.value.code == -5 and "static scratch" in str(e.value)
