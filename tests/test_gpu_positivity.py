"""Positivity-preserving increment limiting on the GPU against the oracle (EulerEvaluator.hxx
:1938-2140, EulerEvaluator.hpp:1645-1857, Gas.hpp:1750-1860), through the C-ABI:

* per-cell alpha, the count of limited cells and the minimum (relax 0.9 and 1, relaxed floors,
  compress powers, the MIN_IF_NOT_ONE / MIN_ALL flags) and the expansion: alpha to 1e-12, the
  per-call parity bar (the quadratic pressure bound cancels in c1^2 - 4 c0 c2 and -sqrt(.) - c1,
  where fused multiply-adds of the device change the last bits: 5e-14 seen), count exact;
* AddFixedIncrement with 5 and 6 variables: the new state to 1e-12;
* the implicit solver with a far-field state runs the limiting in every increment; on a smooth
  vortex run nothing is limited and the states equal the plain update bit for bit.
"""
import numpy as np
import pytest
import torch

import oracle
from dndsr_b200 import mesh as M
from tests.util import VR_HQM_PY, relerr

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def _state(rng, n, nv=5):
    u = np.zeros((n, nv))
    u[:, 0] = 1 + 0.5 * rng.random(n)
    v = rng.normal(size=(n, 3)) * 0.5
    u[:, 1:4] = u[:, :1] * v
    u[:, 4] = (1 + rng.random(n)) / (GAMMA - 1) + 0.5 * u[:, 0] * (v ** 2).sum(1)
    if nv == 6:
        u[:, 5] = np.abs(rng.normal(size=n))
    return u


def _evaluator(nv, n):
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.periodic_hex_3d(n, jitter=0.05)
    vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=1)).construct()
    return m, EulerEvaluator(vr, dict(nVars=nv, riemannSolverType="Roe", muGas=1e-3))


@pytest.mark.parametrize("relax,relaxed,power", [(0.9, False, 1.0), (1.0, False, 1.0), (0.5, True, 2.0)])
def test_cell_rhs_alpha_and_expansion_match_the_oracle(relax, relaxed, power):
    m, ev = _evaluator(5, 16)
    rng = np.random.default_rng(7)
    u0 = _state(rng, m.n_cell)
    r0 = rng.normal(size=u0.shape) * np.array([0.8, 0.8, 0.8, 0.8, 3.0])
    u, r = torch.tensor(u0, device="cuda"), torch.tensor(r0, device="cuda")
    for flag in (0, 1, 2):
        a = torch.empty(m.n_cell, dtype=torch.float64, device="cuda")
        n, amin = ev.EvaluateCellRHSAlpha(u, r, a, 1.0, 1.0, relax, 2, power, relaxed, flag)
        a0, n0, amin0, bad = oracle.cell_rhs_alpha(u0, r0, 1.0, 1.0, relax=relax, compress=2, compressPower=power,
                                                   ppEpsIsRelaxed=relaxed, flag=flag)
        assert not bad and n == n0 and n > 0
        assert abs(amin - amin0) <= 1e-12 * amin0
        assert relerr(a.cpu().numpy(), a0) < 1e-12
    ones = torch.ones(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateCellRHSAlphaExpansion(u, r, ones, 1.0, 1.0, amin0)
    assert np.array_equal(ones.cpu().numpy(), oracle.cell_rhs_alpha_expansion(u0, r0, np.ones(m.n_cell), 1.0, 1.0, amin0))


@pytest.mark.parametrize("nv", [5, 6])
def test_add_fixed_increment_matches_the_oracle(nv):
    m, ev = _evaluator(nv, 16)
    rng = np.random.default_rng(8)
    u0 = _state(rng, m.n_cell, nv)
    i0 = rng.normal(size=u0.shape) * np.array([2.0, 2.0, 2.0, 2.0, 8.0, 3.0][:nv])
    u, inc = torch.tensor(u0, device="cuda"), torch.tensor(i0, device="cuda")
    fix = ev.AddFixedIncrement(u, inc, 0.7, 1.0, 1.0)
    un0, fix0, bad = oracle.add_fixed_increment(u0, i0, 0.7, 1.0, 1.0)
    assert not bad and fix < 1 and abs(fix - fix0) <= 1e-12 * fix0
    assert relerr(u.cpu().numpy(), un0) < 1e-12


def test_nonphysical_mean_state_is_reported():
    from dndsr_b200 import capi
    m, ev = _evaluator(5, 4)
    rng = np.random.default_rng(9)
    u0 = _state(rng, m.n_cell)
    u0[3, 0] = -1.0
    u = torch.tensor(u0, device="cuda")
    r = torch.zeros_like(u)
    with pytest.raises(capi.DndsbError):
        ev.EvaluateCellRHSAlpha(u, r, torch.empty(m.n_cell, dtype=torch.float64, device="cuda"), 1.0, 1.0)


def test_implicit_solver_with_positivity_limiting_equals_the_plain_update_when_nothing_is_limited():
    from dndsr_b200 import implicit as I
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    m = M.iv_mesh(16)
    far = M.freestream(0.5)
    runs = []
    for pp in ((), tuple(far)):
        vr = VariationalReconstruction(m, dict(VR_HQM_PY, maxOrder=2)).construct()
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
        u = vr.BuildUDof(5)
        ev.InitializeUDOF(u, 2, 5.0)
        cfg = I.SolverConfig(odeCode=0, dtImplicit=0.05, nTimeStep=2, nTimeStepInternal=4, farFieldStaticValue=pp)
        s = I.ImplicitSolver(vr, ev, cfg)
        s.run(u)
        runs.append((u.cpu().numpy(), s))
    assert runs[1][1].pp is not None and runs[1][1].nLimInc == 0
    assert np.array_equal(runs[0][0], runs[1][0])
