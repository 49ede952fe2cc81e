"""The oracle's block / Roe Jacobian restatement (CPU): RoeFluxIncFDiff (Gas.hpp:1149-1243) against the Roe
eigen-structure and against the oracle's Roe flux (pinned to the reference's Riemann goldens), the block
inverse, block mode without the Roe term against the scalar operators, the eigenvalue recording of
EvaluateRHS, and one implicit solve that the Roe Jacobian converges faster than the scalar one."""
import numpy as np
import torch

import oracle
from dndsr_b200 import implicit as I
from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.oracle_driver import OracleEval, OracleVR

G = 1.4


def _state(rho, v, p, extra=()):
    v = np.asarray(v, float)
    return np.array([rho, *(rho * v), p / (G - 1) + 0.5 * rho * v @ v, *extra])


def test_roe_dissipation_matrix_has_the_roe_eigenstructure():
    U = _state(1.2, [0.3, -0.2, 0.1], 0.9)
    n = np.array([0.6, 0.0, 0.8])
    rho, v, p = U[0], U[1:4] / U[0], 0.9
    a = np.sqrt(G * p / rho)
    H = (U[4] + p) / rho
    vn = v @ n
    lam = (0.7, 0.3, 1.9)
    Mx = oracle.roe_fdiff_matrix(U, U, n, lam)
    # right eigenvectors of the flux Jacobian along n (acoustic, entropy, two shear waves, acoustic)
    t1 = np.cross(n, [0, 1, 0])
    t1 /= np.linalg.norm(t1)
    t2 = np.cross(n, t1)
    r0 = np.array([1, *(v - a * n), H - vn * a])
    r4 = np.array([1, *(v + a * n), H + vn * a])
    r1 = np.array([1, *v, 0.5 * v @ v])
    rt1 = np.array([0, *t1, v @ t1])
    rt2 = np.array([0, *t2, v @ t2])
    for r, l in ((r0, lam[0]), (r4, lam[2]), (r1, lam[1]), (rt1, lam[1]), (rt2, lam[1])):
        assert np.allclose(Mx @ r, l * r, rtol=1e-13, atol=1e-13)
    # equal eigenvalues: the identity times the eigenvalue; passive scalars ride with l123
    assert np.allclose(oracle.roe_fdiff_matrix(U, U, n, (0.8, 0.8, 0.8)), 0.8 * np.eye(5), atol=1e-14)
    U6 = np.append(U, 0.05)
    M6 = oracle.roe_fdiff_matrix(U6, U6, n, lam)
    assert abs(M6[5, 5] - lam[1]) < 1e-15 and np.allclose(M6[:5, :5], Mx, atol=1e-15)


def test_roe_dissipation_matches_the_roe_flux():
    """F_Roe = (F(UL) + F(UR)) / 2 - RoeFluxIncFDiff(UR - UL; Roe(UL, UR), l) / 2 with the flux's own eigenvalues."""
    rng = np.random.default_rng(1)
    for _ in range(20):
        UL = _state(1 + 0.3 * rng.random(), rng.normal(size=3) * 0.4, 1 + 0.2 * rng.random())
        UR = _state(1 + 0.3 * rng.random(), rng.normal(size=3) * 0.4, 1 + 0.2 * rng.random())
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        F, lam = oracle.riemann("Roe", UL, UR, n, fixScale=1.0, incFScale=1.0)

        def phys(U):
            v = U[1:4] / U[0]
            p = (G - 1) * (U[4] - 0.5 * U[0] * v @ v)
            vn = v @ n
            return np.array([U[0] * vn, *(U[1:4] * vn + p * n), (U[4] + p) * vn])

        Mx = oracle.roe_fdiff_matrix(UL, UR, n, lam)
        ref = 0.5 * (phys(UL) + phys(UR)) - 0.5 * Mx @ (UR - UL)
        assert np.allclose(F, ref, rtol=1e-12, atol=1e-13)


def _bump():
    m = M.renumber_by_color(M.bump_channel_tet(5, 3, 2))
    o, far, types, vals, w = bump_oracle(m, 1, "Roe", 0.0, 1)
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    return m, o, far, u0, uRec0


def test_block_modes_and_recorded_eigenvalues():
    m, o, far, u0, uRec0 = _bump()
    d0, _ = o.eval_dt(u0, 5.0)
    rhs = o.eval_rhs(u0, uRec0)
    lamConv = o.get("lambdaFace0")
    assert np.array_equal(lamConv, o.get("lambdaFace123")) and np.array_equal(lamConv, o.get("lambdaFace4"))
    jd = o.lusgs_init(d0, 0.1, 0.5)
    x0 = np.random.default_rng(9).normal(size=u0.shape)
    A0 = o.lusgs_matvec(0.5, u0, x0, jd)
    s0, _ = o.update_sgs(0.5, rhs, u0, x0, np.zeros_like(x0), jd, True)
    o.set_jacobian_mode(False, False)
    jb = o.lusgs_init_block(d0, 0.1, 0.5, u0)
    assert np.allclose(jb[:, 0], jd[:, None, None] * np.eye(5), rtol=0, atol=0)
    assert np.allclose(o.lusgs_matvec(0.5, u0, x0, jb), A0, rtol=1e-15, atol=0)
    assert np.allclose(o.update_sgs(0.5, rhs, u0, x0, np.zeros_like(x0), jb, True)[0], s0, rtol=1e-14, atol=1e-15)
    o.set_jacobian_mode(False, True)
    rhs2 = o.eval_rhs(u0, uRec0)
    assert np.array_equal(rhs2, rhs)
    l0, l1, l4 = o.get("lambdaFace0"), o.get("lambdaFace123"), o.get("lambdaFace4")
    assert (l0 >= 0).all() and (l1 >= 0).all() and (l4 >= 0).all() and not np.array_equal(l0, lamConv)
    jr = o.lusgs_init_block(d0, 0.1, 0.5, u0)
    I5 = np.eye(5)
    assert np.abs(np.einsum("cij,cjk->cik", jr[:, 0], jr[:, 1]) - I5).max() < 1e-13
    # the trace of a cell without boundary faces: 5 (1/dTau + 1/dt) plus, per face, (alpha/2)(A_f/V) times the
    # eigenvalue sum l0 + 3 l123 + l4 of the Roe dissipation matrix plus 5 lambdaVis
    area, vol, lv = o.get("faceArea"), o.get("volume"), o.get("lambdaFaceVis")
    f2c = np.asarray(m.face2cell)
    tr = 5 * (1.0 / d0 + 1.0 / 0.1)
    bnd = np.zeros(m.n_cell, bool)
    for f, (c0, c1) in enumerate(f2c):
        t = 0.25 * area[f] * (l0[f] + 3 * l1[f] + l4[f] + 5 * lv[f])
        tr[c0] += t / vol[c0]
        if c1 >= 0:
            tr[c1] += t / vol[c1]
        else:
            bnd[c0] = True
    assert (~bnd).sum() > 10
    got = np.einsum("cii->c", jr[:, 0])
    assert np.allclose(got[~bnd], tr[~bnd], rtol=1e-13, atol=0)


def test_roe_jacobian_converges_faster_on_the_bump():
    m, o, far, u0, uRec0 = _bump()
    drops = {}
    for roe in (False, True):
        oe = OracleEval(o)
        oe.SetJacobianMode(not roe, roe)
        cfg = I.SolverConfig(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=20, nTimeStepInternalMin=20, CFL=50.0, gmresCode=1,
                             nGmresSpace=10)
        u = torch.tensor(np.tile(far, (m.n_cell, 1)))
        I.ImplicitSolver(OracleVR(o), oe, cfg).run(u)
        drops[roe] = cfg.res_history[-1][2]
    assert drops[True] < 0.7 * drops[False], drops


def _dense(o, n, nv, f):
    """The n nv x n nv matrix of the linear map f (column by column)."""
    A = np.zeros((n * nv, n * nv))
    for i in range(n * nv):
        e = np.zeros((n, nv))
        e.flat[i] = 1.0
        A[:, i] = f(e).ravel()
    return A


def test_block_ilu0_factors_match_the_operator_on_its_pattern():
    """JacobianLocalLU with iluCode 0: L U equals the LUSGSMatrixVec operator A on A's block pattern, and the
    LU solve inverts L U exactly; one defect-correction step reduces the residual of A x = b."""
    m = M.renumber_by_color(M.bump_channel_tet(3, 2, 2))
    o, far, types, vals, w = bump_oracle(m, 1, "Roe", 0.0, 1)
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    o.set_jacobian_mode(False, True)
    d0, _ = o.eval_dt(u0, 20.0)
    o.eval_rhs(u0, uRec0)
    jd = o.lusgs_init_block(d0, 1e100, 1.0, u0)
    n, nv = m.n_cell, 5
    A = _dense(o, n, nv, lambda x: o.lusgs_matvec(1.0, u0, x, jd))
    o.jacobian_lu(1.0, u0, jd)
    off = o.get("luOff").reshape(n, -1, nv, nv)
    dinv = o.get("luDinv").reshape(n, nv, nv)
    f2c = np.asarray(m.face2cell)
    c2f = np.asarray(m.cell2face)
    L, U = np.eye(n * nv), np.zeros((n * nv, n * nv))
    pattern = np.zeros((n, n), bool)
    for i in range(n):
        U[i * nv:(i + 1) * nv, i * nv:(i + 1) * nv] = np.linalg.inv(dinv[i])
        pattern[i, i] = True
        for k, f in enumerate(c2f[i]):
            c0, c1 = f2c[f]
            j = c1 if c0 == i else c0
            if j < 0 or j == i:
                continue
            pattern[i, j] = True
            blk = (L if j < i else U)
            blk[i * nv:(i + 1) * nv, j * nv:(j + 1) * nv] = off[i, k]
    LU = L @ U
    mask = np.kron(pattern, np.ones((nv, nv), bool))
    assert np.abs((LU - A)[mask]).max() < 1e-12 * np.abs(A).max()
    assert np.abs(LU[~mask]).max() > 0  # the incomplete factorisation drops fill on this mesh
    b = np.random.default_rng(5).normal(size=(n, nv))
    x, s = o.solve_jacobian_lu(1.0, b, u0, np.zeros_like(b), jd, uIncIsZero=True)
    assert np.allclose(LU @ x.ravel(), b.ravel(), rtol=0, atol=1e-12 * np.abs(b).max())
    assert np.allclose(s, np.abs(x).sum(0))
    x2, _ = o.solve_jacobian_lu(1.0, b, u0, x, jd, uIncIsZero=False)
    r1 = np.linalg.norm(b.ravel() - A @ x.ravel())
    r2 = np.linalg.norm(b.ravel() - A @ x2.ravel())
    assert r2 < 0.5 * r1, (r1, r2)


def test_local_lu_with_the_scalar_jacobian_equals_block_mode():
    """LUSGSMatrixToJacobianLU takes JDiag.getValue: with the scalar Jacobian the diagonal blocks are the scalar
    diagonal, so its local LU equals the one of the block mode without the Roe term."""
    m = M.renumber_by_color(M.bump_channel_tet(3, 2, 2))
    o, far, types, vals, w = bump_oracle(m, 1, "Roe", 0.0, 1)
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    d0, _ = o.eval_dt(u0, 20.0)
    rhs = o.eval_rhs(u0, uRec0)
    b = np.random.default_rng(6).normal(size=rhs.shape)
    out = {}
    for block in (False, True):
        o.set_jacobian_mode(not block, False)
        jd = o.lusgs_init_block(d0, 1e100, 1.0, u0) if block else o.lusgs_init(d0, 1e100, 1.0)
        o.jacobian_lu(1.0, u0, jd)
        out[block] = (o.get("luOff"), o.get("luDinv"), o.solve_jacobian_lu(1.0, b, u0, np.zeros_like(b), jd, True)[0],
                      o.solve_jacobian_lu(1.0, b, u0, 0.1 * b, jd, False)[0])
    for a, c in zip(out[False], out[True]):
        assert np.allclose(a, c, rtol=1e-14, atol=1e-14 * np.abs(c).max())


def test_block_ilu0_with_triangles_in_the_cell_graph():
    """On a 3-periodic hexahedral grid each row of three cells is a triangle of face neighbours, so the ILU(0)
    updates between two neighbours that share a lower neighbour (L_ij -= L_ik U_kj, U_ij -= L_ik U_kj) run; the
    factors still reproduce A on its pattern."""
    import oracle
    from tests.util import VR_HQM
    m = M.renumber_by_color(M.tgv_mesh(3))
    es = dict(nVars=5, rsType=oracle.RS["Roe"], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=1e-3, prGas=0.72, TRef=273.15,
              CSutherland=110.4, muModel=0, ignoreVis=0)
    o = oracle.Oracle(m, dict(VR_HQM, maxOrder=1), es)
    assert o.construct() == 0
    u0 = o.init_field(3)
    uRec0 = 0.02 * np.random.default_rng(1).normal(size=(m.n_cell, o.R, 5))
    o.set_jacobian_mode(False, True)
    d0, _ = o.eval_dt(u0, 10.0)
    o.eval_rhs(u0, uRec0)
    jd = o.lusgs_init_block(d0, 1e100, 1.0, u0)
    n, nv = m.n_cell, 5
    A = _dense(o, n, nv, lambda x: o.lusgs_matvec(1.0, u0, x, jd))
    o.jacobian_lu(1.0, u0, jd)
    off = o.get("luOff").reshape(n, -1, nv, nv)
    dinv = o.get("luDinv").reshape(n, nv, nv)
    f2c, c2f = np.asarray(m.face2cell), np.asarray(m.cell2face)
    L, U = np.eye(n * nv), np.zeros((n * nv, n * nv))
    pattern = np.zeros((n, n), bool)
    tri = 0
    nb = [set() for _ in range(n)]
    for i in range(n):
        U[i * nv:(i + 1) * nv, i * nv:(i + 1) * nv] = np.linalg.inv(dinv[i])
        pattern[i, i] = True
        for k, f in enumerate(c2f[i]):
            c0, c1 = f2c[f]
            j = c1 if c0 == i else c0
            if j < 0 or j == i:
                continue
            nb[i].add(j)
            pattern[i, j] = True
            (L if j < i else U)[i * nv:(i + 1) * nv, j * nv:(j + 1) * nv] = off[i, k]
    for i in range(n):
        for j in nb[i]:
            tri += len(nb[i] & nb[j])
    assert tri > 0  # the cell graph has triangles
    mask = np.kron(pattern, np.ones((nv, nv), bool))
    assert np.abs((L @ U - A)[mask]).max() < 1e-12 * np.abs(A).max()
