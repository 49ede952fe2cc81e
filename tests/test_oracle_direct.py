"""The oracle's block ILU(0) (JacobianLocalLU::InPlaceDecompose with iluCode 0 and Solve, Solver/Direct.hpp:312-405,
487-540) on the reference's own unit case of the local LU and against the oracle's Euler-operator factorisation.

test/cpp/Solver/test_Direct.cpp builds a 2-D periodic Laplacian on a 4 x 4 grid with 2 x 2 blocks (:70-129):
diagonal 4 I + delta diag(i, 2 i) with delta 0.1, -I for each of the four neighbours (r -+ 1, c), (r, c -+ 1) with
wrap-around.  Its ILU(0) assertions are restated here with the same inputs: one ILU(0) solve of A x = b leaves a
relative residual below 0.5 and above 1e-14 (:199-258), and ten fixed-point iterations preconditioned by ILU(0)
bring the error below 1e-3 (:270-352).  The product check of :160-189 pins the matrix this file builds.  The
oracle's factorisation of the Euler operator (Oracle::jacobianLU, the one the GPU local LU is compared with) is
then shown to equal the general-pattern routine on the operator's own blocks."""
import numpy as np

import oracle
from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.test_oracle_roe_jacobian import _dense

G, BS = 4, 2  # grid side, block size (test_Direct.cpp:36, 72)


def _cell(r, c):
    return ((r % G) + G) % G * G + ((c % G) + G) % G


def _laplacian(delta=0.1):
    """nbr [16][4], off [16][4][2][2], diag [16][2][2] of test_Direct.cpp's fill2DLaplacian (:100-129)."""
    n = G * G
    nbr = np.zeros((n, 4), np.int64)
    for r in range(G):
        for c in range(G):
            nbr[_cell(r, c)] = [_cell(r - 1, c), _cell(r + 1, c), _cell(r, c - 1), _cell(r, c + 1)]
    off = np.broadcast_to(-np.eye(BS), (n, 4, BS, BS)).copy()
    diag = np.array([4 * np.eye(BS) + delta * np.diag([i, 2 * i]) for i in range(n)])
    return nbr, off, diag


def _matmul(nbr, off, diag, x):
    y = np.einsum("irc,ic->ir", diag, x)
    for k in range(nbr.shape[1]):
        y += np.einsum("irc,ic->ir", off[:, k], x[nbr[:, k]])
    return y


def _x_known(n):
    i = np.arange(n)
    return np.stack([np.sin(0.7 * i + 0.1), np.cos(0.4 * i + 0.2)], 1)


def test_product_of_the_reference_matrix():
    nbr, off, diag = _laplacian()
    i = np.arange(G * G)
    x = np.stack([np.sin(0.5 * i), np.cos(0.3 * i)], 1)
    y = _matmul(nbr, off, diag, x)
    expected = diag[0] @ x[0] - sum(x[j] for j in (_cell(-1, 0), _cell(1, 0), _cell(0, -1), _cell(0, 1)))
    assert np.abs(y[0] - expected).max() < 1e-14


def test_ilu0_solve_reduces_the_residual_but_is_not_exact():
    nbr, off, diag = _laplacian()
    n = G * G
    xk = _x_known(n)
    b = _matmul(nbr, off, diag, xk)
    fac, dinv = oracle.block_ilu0(nbr, off, diag)
    x = oracle.block_ilu0_solve(nbr, fac, dinv, b)
    rel = np.linalg.norm(b - _matmul(nbr, off, diag, x)) / np.linalg.norm(b)
    assert 1e-14 < rel < 0.5, rel


def test_ilu0_preconditioned_iteration_converges():
    nbr, off, diag = _laplacian()
    n = G * G
    xk = _x_known(n)
    b = _matmul(nbr, off, diag, xk)
    fac, dinv = oracle.block_ilu0(nbr, off, diag)
    x = np.zeros_like(b)
    for _ in range(10):  # x += M^-1 (b - A x), test_Direct.cpp:270-308
        x += oracle.block_ilu0_solve(nbr, fac, dinv, b - _matmul(nbr, off, diag, x))
    assert np.linalg.norm(x - xk) < 1e-3


def test_ilu0_factors_reproduce_the_matrix_on_its_pattern():
    """(L + I)(D + U) = A on the block pattern; off the pattern the dropped fill is non-zero on this grid."""
    nbr, off, diag = _laplacian()
    n = G * G
    fac, dinv = oracle.block_ilu0(nbr, off, diag)
    A = np.zeros((n * BS, n * BS))
    L, U = np.eye(n * BS), np.zeros((n * BS, n * BS))
    pattern = np.eye(n, dtype=bool)
    for i in range(n):
        A[i * BS:(i + 1) * BS, i * BS:(i + 1) * BS] = diag[i]
        U[i * BS:(i + 1) * BS, i * BS:(i + 1) * BS] = np.linalg.inv(dinv[i])
        for k, j in enumerate(nbr[i]):
            A[i * BS:(i + 1) * BS, j * BS:(j + 1) * BS] += off[i, k]
            pattern[i, j] = True
            (L if j < i else U)[i * BS:(i + 1) * BS, j * BS:(j + 1) * BS] = fac[i, k]
    mask = np.kron(pattern, np.ones((BS, BS), bool))
    LU = L @ U
    assert np.abs((LU - A)[mask]).max() < 1e-13
    assert np.abs((LU - A)[~mask]).max() > 1e-3


def test_ilu0_is_exact_without_fill():
    """On a path graph ILU(0) drops nothing: the solve is exact (the role of the complete-LU case of
    test_Direct.cpp:160-197, whose fill levels are out of scope here)."""
    n = 12
    rng = np.random.default_rng(7)
    nbr = np.array([[i - 1 if i > 0 else -1, i + 1 if i < n - 1 else -1] for i in range(n)], np.int64)
    off = rng.normal(size=(n, 2, 3, 3)) * 0.3
    diag = np.array([4 * np.eye(3) + 0.2 * rng.normal(size=(3, 3)) for _ in range(n)])
    xk = rng.normal(size=(n, 3))
    b = np.einsum("irc,ic->ir", diag, xk)
    for k in range(2):
        has = nbr[:, k] >= 0
        b[has] += np.einsum("irc,ic->ir", off[has, k], xk[nbr[has, k]])
    fac, dinv = oracle.block_ilu0(nbr, off, diag)
    assert np.abs(oracle.block_ilu0_solve(nbr, fac, dinv, b) - xk).max() < 1e-12


def test_euler_operator_factorisation_equals_the_general_routine():
    """Oracle::jacobianLU on the block Roe operator of a bump mesh equals the general-pattern block ILU(0) of the
    same operator's blocks, so the reference's unit case above pins the factorisation the GPU is compared with."""
    m = M.renumber_by_color(M.bump_channel_tet(3, 2, 2))
    o, far, types, vals, w = bump_oracle(m, 1, "Roe", 0.0, 1)
    u0, uRec0 = perturbed_state(m, far, R=o.R)
    o.set_jacobian_mode(False, True)
    d0, _ = o.eval_dt(u0, 20.0)
    o.eval_rhs(u0, uRec0)
    jd = o.lusgs_init_block(d0, 1e100, 1.0, u0)
    n, nv = m.n_cell, 5
    A = _dense(o, n, nv, lambda x: o.lusgs_matvec(1.0, u0, x, jd)).reshape(n, nv, n, nv)
    f2c, c2f = np.asarray(m.face2cell), np.asarray(m.cell2face)
    nf = c2f.shape[1]
    nbr = np.full((n, nf), -1, np.int64)
    off = np.zeros((n, nf, nv, nv))
    for i in range(n):
        for k, f in enumerate(c2f[i]):
            c0, c1 = f2c[f]
            j = c1 if c0 == i else c0
            if j >= 0 and j != i:
                nbr[i, k] = j
                off[i, k] = A[i, :, j, :]
    assert all(len(set(r[r >= 0])) == len(r[r >= 0]) for r in nbr)  # one slot per neighbour
    diag = np.array([A[i, :, i, :] for i in range(n)])
    fac, dinv = oracle.block_ilu0(nbr, off, diag)
    o.jacobian_lu(1.0, u0, jd)
    scale = np.abs(A).max()
    got = o.get("luOff").reshape(n, nf, nv, nv)
    assert np.abs(got - np.where((nbr >= 0)[:, :, None, None], fac, 0.0)).max() < 1e-12 * scale
    gdinv = o.get("luDinv").reshape(n, nv, nv)
    assert np.abs(gdinv - dinv).max() < 1e-12 * np.abs(dinv).max()
    b = np.random.default_rng(3).normal(size=(n, nv))
    x, _ = o.solve_jacobian_lu(1.0, b, u0, np.zeros_like(b), jd, uIncIsZero=True)
    assert np.abs(x - oracle.block_ilu0_solve(nbr, fac, dinv, b)).max() < 1e-12 * np.abs(x).max()
