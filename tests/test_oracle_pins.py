"""Pins the CPU oracle to the reference's own golden vectors (no GPU needed)."""
import json
import os

import numpy as np
import pytest

import oracle
from dndsr_b200 import mesh as M

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_goldens.json")))


def _prim2cons(r, u, v, w, p, g=1.4):
    return np.array([r, r * u, r * v, r * w, p / (g - 1) + 0.5 * r * (u * u + v * v + w * w)])


@pytest.mark.parametrize("rs", ["Roe", "HLLC", "HLLEP"])
def test_riemann_golden(rs):
    G = GOLD["riemann_mixed_state"]
    UL, UR = _prim2cons(*G["primL"]), _prim2cons(*G["primR"])
    n = np.array(G["normal_unnormalised"]) / np.linalg.norm(G["normal_unnormalised"])
    F, _ = oracle.riemann(rs, UL, UR, n, gamma=G["gamma"])
    np.testing.assert_allclose(F, G["flux"][rs], rtol=G["rel_tol"])


def _exact_flux(U, n, g=1.4):
    v = U[1:4] / U[0]
    p = (g - 1) * (U[4] - 0.5 * U[0] * v @ v)
    vn = v @ n
    return np.array([U[0] * vn, *(U[1:4] * vn + p * n), (U[4] + p) * vn])


@pytest.mark.parametrize("rs", ["Roe", "HLLC", "HLLEP", "Roe_M1", "Roe_M3", "Roe_M4", "Roe_M5", "Roe_M6", "Roe_M7", "Roe_M8"])
def test_riemann_consistency(rs):
    # test_RiemannSolvers.cpp:85-158: identical states give the physical flux
    U = _prim2cons(1.225, 100.0, -50.0, 25.0, 101325.0)
    n = np.array([0.6, -0.8, 0.0])
    F, _ = oracle.riemann(rs, U, U, n)
    np.testing.assert_allclose(F, _exact_flux(U, n), rtol=1e-8, atol=1e-8 * np.abs(_exact_flux(U, n)).max())


@pytest.mark.parametrize("rs", ["Roe", "HLLC", "HLLEP"])
def test_riemann_symmetry(rs):
    # test_RiemannSolvers.cpp:164-200: F(UL,UR,n) = -F(UR,UL,-n)
    UL = _prim2cons(1.0, 100.0, 0.0, 0.0, 100000.0)
    UR = _prim2cons(0.125, 0.0, 0.0, 0.0, 10000.0)
    n = np.array([1.0, 0.0, 0.0])
    F1, _ = oracle.riemann(rs, UL, UR, n)
    F2, _ = oracle.riemann(rs, UR, UL, -n)
    np.testing.assert_allclose(F1, -F2, rtol=1e-10, atol=1e-10 * np.abs(F1).max())


def _approx(a, b, eps):  # doctest's Approx: |a - b| < eps (1 + max(|a|, |b|))
    return np.all(np.abs(a - b) < eps * (1 + np.maximum(np.abs(a), np.abs(b))))


@pytest.mark.parametrize("rs", ["Roe", "HLLC", "HLLEP"])
def test_riemann_sod_flux_finite_and_mass_flux_non_negative(rs):
    # test_RiemannSolvers.cpp:188-238: Sod states (1, 0, 1) | (0.125, 0, 0.1) along x
    F, _ = oracle.riemann(rs, _prim2cons(1.0, 0, 0, 0, 1.0), _prim2cons(0.125, 0, 0, 0, 0.1), np.array([1.0, 0, 0]))
    assert np.all(np.isfinite(F)) and F[0] >= -1e-10


def test_riemann_quiescent_gas_gives_the_pressure_flux():
    # test_RiemannSolvers.cpp:297-313: rho = 1, v = 0, p = 1, every solver gives the exact flux to 1e-12
    U = _prim2cons(1.0, 0, 0, 0, 1.0)
    n = np.array([1.0, 0, 0])
    for rs in ("Roe", "HLLC", "HLLEP"):
        F, _ = oracle.riemann(rs, U, U, n)
        assert _approx(F, _exact_flux(U, n), 1e-12), rs


def test_roe_eigenvalue_output_subsonic():
    # test_RiemannSolvers.cpp:319-336: |u - a|, |u|, |u + a| are non-negative and |u + a| >= |u|
    _, lam = oracle.riemann("Roe", _prim2cons(1.0, 50.0, 0, 0, 100000.0), _prim2cons(1.1, 55.0, 0, 0, 105000.0), np.array([1.0, 0, 0]))
    assert np.all(lam >= 0) and lam[2] >= lam[1]


def test_roe_consistency_on_a_diagonal_normal():
    # test_RiemannSolvers.cpp:342-357
    U = _prim2cons(2.0, 100.0, 200.0, 300.0, 200000.0)
    n = np.ones(3) / np.sqrt(3.0)
    F, _ = oracle.riemann("Roe", U, U, n)
    assert _approx(F, _exact_flux(U, n), 1e-8)


def test_viscous_flux_of_a_zero_gradient_is_zero():
    # test_GasThermo.cpp:479-494: mu 1.8e-5, k 0.025, Cp 1005, n = x
    F = oracle.viscous_flux(_prim2cons(1.225, 100.0, -50.0, 25.0, 101325.0), np.zeros((3, 5)), np.array([1.0, 0, 0]), 1.4, 1.8e-5,
                            0.025, 1005.0)
    assert _approx(F, np.zeros(5), 1e-10)


def _vr_error(n, p, hqm, f, mesh=None):
    m = M.periodic_quad_2d(n, L=10.0, jitter=0.0) if mesh is None else mesh
    vr = dict(maxOrder=p, intOrder=max(p + 2, 5), jacobiRelax=1.0, SORInstead=0, scaleType=1, scaleMultiplier=1.0,
              dirWeightScheme=1 if hqm else 0, geomWeightScheme=1 if hqm else 0, geomWeightBias=1.0,
              geomWeightPower=0.5, bcWeight=1.0)
    o = oracle.Oracle(m, vr, dict(nVars=1, gamma=1.4))
    assert o.construct() == 0
    pp = o.get("cellPP").reshape(m.n_cell, o.nGc, 3)
    jd = o.get("cellJDet").reshape(m.n_cell, o.nGc)
    w = o.cell_quad_weights()
    vol = o.get("volume")
    u = ((f(pp) * jd * w).sum(1) / vol)[:, None]
    uRec = np.zeros((m.n_cell, o.R, 1))
    for _ in range(200):  # test_Reconstruction.cpp:345-375 (Jacobi to an RMS increment below 1e-14)
        new = o.vr_iter(uRec, u)
        inc = np.sqrt(((new - uRec) ** 2).sum() / m.n_cell)
        uRec = new
        if inc < 1e-14:
            break
    vals = o.cell_point_values(u, uRec)[..., 0]
    return (np.abs(vals - f(pp)) * jd * w).sum() / vol.sum()


_K = 2 * np.pi / 10
_FUNCS = {
    "vr_iv10_sincos": lambda x: np.sin(_K * x[..., 0]) * np.cos(_K * x[..., 1]),
    "vr_iv10_cospluscos": lambda x: np.cos(_K * x[..., 0]) + np.cos(_K * x[..., 1]),
}
_CASES = [(key, c, ib) for key in _FUNCS for c in GOLD[key]["cases"] for ib in range(3)]


@pytest.mark.parametrize("key,case,ib", _CASES, ids=[f"{k}-p{c['p']}-{c['weights']}-bis{ib}" for k, c, ib in _CASES])
def test_vr_iv10_golden(key, case, ib):
    err = _vr_error([10, 20, 40][ib], case["p"], case["weights"] == "HQM", _FUNCS[key])
    assert abs(err - case["golden"][ib]) <= GOLD[key]["rel_tol"] * case["golden"][ib]


# ---- one Newton step of the evaluator pipeline (test_EulerEvaluator.cpp:120-330) ----
from tests.newton_case import CASES as NEWTON_CASES, GAS, initial_state, norms  # noqa: E402


def _newton_oracle(case, rsMeanValueEig=None):
    m = case["mesh"]()
    mve = case["rsMeanValueEig"] if rsMeanValueEig is None else rsMeanValueEig
    es = dict(nVars=5, rsType=oracle.RS[case["rs"]], rsFixScale=1.0, rsIncFScale=1.0, ignoreVis=0, rsMeanValueEig=mve, **GAS)
    o = oracle.Oracle(m, case["vr_oracle"], es)
    assert o.construct() == 0
    u = initial_state(case, o.get("cellBary").reshape(-1, 3), init_field=o.init_field)
    dTau, _ = o.eval_dt(u, case["CFL"], 1e100, True)
    rhs = o.eval_rhs(u, np.zeros((m.n_cell, o.R, 5)))
    jd = o.lusgs_init(dTau, 1e100, 1.0)
    x = np.zeros_like(u)
    xn = o.update_lusgs(1.0, rhs, u, x, np.zeros_like(u), jd, forward=True)
    xn = o.update_lusgs(1.0, rhs, u, x, xn, jd, forward=False)
    return norms(rhs, xn, o.get("volume")), (o, u, rhs)


@pytest.mark.parametrize("name", list(NEWTON_CASES))
def test_newton_step_golden(name):
    case = NEWTON_CASES[name]
    (rhs_l1, inc_l2), _ = _newton_oracle(case)
    g = case["gold"]
    assert abs(rhs_l1 - g["rhsDensityL1"]) <= g["rel_tol"] * g["rhsDensityL1"]
    assert abs(inc_l2 - g["incL2"]) <= g["rel_tol"] * g["incL2"]


def test_mean_value_eig_straight_and_curved_faces():
    # straight faces: the batched mean-value Roe flux equals the per-point one (one normal per face)
    (a, _), (_, _, rhs1) = _newton_oracle(NEWTON_CASES["iv"], 1)
    (b, _), (_, _, rhs0) = _newton_oracle(NEWTON_CASES["iv"], 0)
    assert np.abs(rhs1 - rhs0).max() <= 1e-13 * np.abs(rhs0).max()
    # warped hexahedra: per-point normals differ from the face mean, and so do the two fluxes
    m = M.tgv_mesh(4)
    out = []
    for mve in (0, 1):
        es = dict(nVars=5, rsType=oracle.RS["Roe_M1"], rsFixScale=1.0, rsIncFScale=1.0, ignoreVis=1, rsMeanValueEig=mve, gamma=1.4,
                  Rgas=1.0, muGas=0.0, prGas=0.72, TRef=273.15, CSutherland=110.4, muModel=0)
        o = oracle.Oracle(m, dict(NEWTON_CASES["iv"]["vr_oracle"], maxOrder=2, intOrder=5), es)
        assert o.construct() == 0
        u = o.init_field(3)
        uRec = np.random.default_rng(3).normal(size=(m.n_cell, o.R, 5)) * 1e-2
        o.eval_dt(u, 1.0)
        out.append(o.eval_rhs(u, uRec))
    d = np.abs(out[1] - out[0]).max() / np.abs(out[0]).max()
    assert 1e-12 < d < 0.5


def test_update_lusgs_inplace_is_gauss_seidel():
    # uInc aliased with uIncNew: the forward sweep reads the new values of lower cells (sequential
    # Gauss-Seidel); with a separate zero uInc it is D^-1 rhs (the Newton-step sequence above)
    _, (o, u, rhs) = _newton_oracle(NEWTON_CASES["iv"])
    dTau, _ = o.eval_dt(u, 100.0)
    jd = o.lusgs_init(dTau, 1e100, 1.0)
    zero = np.zeros_like(u)
    jac = o.update_lusgs(1.0, rhs, u, zero, zero, jd, forward=True)
    np.testing.assert_allclose(jac, rhs / jd[:, None], rtol=1e-14, atol=0)
    gs = o.update_lusgs(1.0, rhs, u, None, zero, jd, forward=True, inplace=True)
    # reference: an explicit sequential sweep with the matrix-vector operator's off-diagonal part
    ref = np.zeros_like(u)
    for c in range(u.shape[0]):
        x = np.zeros_like(u)
        x[:c] = ref[:c]
        Ax = o.lusgs_matvec(1.0, u, x, jd)  # row c: sum_{o<c} w dF(x_o) (x_c = 0)
        ref[c] = (rhs[c] - Ax[c]) / jd[c]
    np.testing.assert_allclose(gs, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


_K3 = 2 * np.pi
_FUNCS3 = {
    "sinCos3D": lambda x: np.sin(_K3 * x[..., 0]) * np.cos(_K3 * x[..., 1]) * np.cos(_K3 * x[..., 2]),
    "cosPlusCos3D": lambda x: np.cos(_K3 * x[..., 0]) + np.cos(_K3 * x[..., 1]) + np.cos(_K3 * x[..., 2]),
}


@pytest.fixture(scope="module")
def uniform32_3d():
    return M.periodic_hex_3d(32, L=1.0, jitter=0.0)


@pytest.mark.parametrize("case", GOLD["vr_uniform32_3d"]["cases"], ids=lambda c: f"{c['func']}-p{c['p']}")
def test_vr_uniform32_3d_golden(case, uniform32_3d):
    # test_Reconstruction3D.cpp:394-407: VFV HQM (HQM_OPT / HQM_SD, power 0.5, bias 1), intOrder max(p + 2, 5),
    # Jacobi sweeps to an RMS increment below 1e-14 or 200 sweeps, L1 error at the cell quadrature points / volume
    err = _vr_error(None, case["p"], True, _FUNCS3[case["func"]], mesh=uniform32_3d)
    assert abs(err - case["golden"]) <= GOLD["vr_uniform32_3d"]["rel_tol"] * case["golden"], err


@pytest.mark.parametrize("p", [1, 2])
def test_vr_3d_constant_exactness(p, uniform32_3d):
    # test_Reconstruction3D.cpp:347-366: a constant is reconstructed with an error below 1e-12
    assert _vr_error(None, p, True, lambda x: np.ones(x.shape[:-1]), mesh=uniform32_3d) < 1e-12
