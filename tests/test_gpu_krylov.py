"""The device Krylov primitives of the C-ABI (dndsb_krylov_*) and the flexible GMRES of dndsr_b200/adjoint.py
built on them: the Arnoldi relation A V_k = V_{k+1} H against numpy, FP32 and FP64 columns; the GMRES solves
nonsymmetric systems on tuples of tensors to the requested drop with a fixed and with a varying
preconditioner, and returns its residual history."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _system(n=60, seed=0):
    rng = np.random.default_rng(seed)
    A = np.eye(n) * 4 + rng.normal(size=(n, n)) * 0.3
    B = rng.normal(size=(n // 2, n // 2)) * 0.2 + np.eye(n // 2) * 2
    return torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n", [37, 1000])
def test_arnoldi_relation(dtype, n):
    from dndsr_b200.solver import _C
    C = _C()
    k = 6
    rng = np.random.default_rng(n)
    A = np.eye(n) * 3 + rng.normal(size=(n, n)) / np.sqrt(n)
    b = rng.normal(size=n)
    ld = C.krylov_ld(n)
    assert ld % 4 == 0 and ld >= n
    f64 = dict(dtype=torch.float64, device="cuda")
    V = torch.zeros((k + 1, ld), dtype=dtype, device="cuda")
    H, gsc, cs = torch.zeros(k * (k + 1), **f64), torch.zeros(8 + k, **f64), torch.zeros(k + 1, **f64)
    res = torch.zeros(k, **f64)
    work = torch.zeros(C.krylov_work_bytes(), dtype=torch.uint8, device="cuda")
    At = torch.tensor(A, dtype=dtype, device="cuda")
    C.krylov_start(torch.tensor(b, dtype=dtype, device="cuda"), V, gsc, cs, work, k)
    for j in range(k):
        V[j + 1, :n] = At @ (V[j, :n] * cs[j].to(dtype))
        C.krylov_arnoldi(n, j, k, V, H, cs, gsc, res[j:j + 1], work)
    Vn = (V[:, :n].double() * cs[:, None]).cpu().numpy()
    Hm = H.cpu().numpy().reshape(k, k + 1).T  # column j at j * (k + 1)
    tol = 1e-12 if dtype == torch.float64 else 2e-5
    assert abs(float(gsc[1]) - np.linalg.norm(b)) <= tol * np.linalg.norm(b)
    np.testing.assert_allclose(Vn[0], b / np.linalg.norm(b), atol=tol)
    np.testing.assert_allclose(A @ Vn[:k].T, Vn.T @ Hm, atol=tol * 10)
    np.testing.assert_allclose(Vn @ Vn.T, np.eye(k + 1), atol=tol * 10)
    assert float(V[:, n:].abs().max() if ld > n else 0.0) == 0.0
    # the least squares after k columns: residual of min |beta e1 - H y| and the update x = V y
    beta = np.linalg.norm(b)
    e1 = np.zeros(k + 1)
    e1[0] = beta
    y, *_ = np.linalg.lstsq(Hm, e1, rcond=None)
    assert abs(float(res[-1]) - np.linalg.norm(e1 - Hm @ y)) <= tol * beta * 10
    x = torch.zeros(ld, dtype=dtype, device="cuda")
    C.krylov_update(n, k, V, gsc, cs, x)
    np.testing.assert_allclose(x[:n].double().cpu().numpy(), Vn[:k].T @ y, atol=tol * 100)


def test_gmres_solves_a_two_block_system():
    from dndsr_b200.adjoint import gmres
    A, B = _system()
    n, m = A.shape[0], B.shape[0]

    def op(x):
        return (A @ x[0] + 0.1 * torch.cat([x[1], x[1]]), B @ x[1])

    prec = lambda r: (r[0] / 4, r[1] / 2)
    rng = np.random.default_rng(1)
    b = (torch.tensor(rng.normal(size=n), device="cuda"), torch.tensor(rng.normal(size=m), device="cuda"))
    x, hist = gmres(op, prec, b, restart=8, max_restarts=50, rtol=1e-12)
    r = tuple(bi - oi for bi, oi in zip(b, op(x)))
    rn = float(sum((ri * ri).sum() for ri in r)) ** 0.5
    bn = float(sum((bi * bi).sum() for bi in b)) ** 0.5
    assert hist[-1] <= 1e-12 and rn <= 1e-11 * bn
    assert hist[0] == 1.0 and all(h >= 0 for h in hist)


def test_gmres_with_a_varying_preconditioner():
    from dndsr_b200.adjoint import gmres
    A, _ = _system(40, seed=3)
    calls = [0]

    def prec(r):
        calls[0] += 1
        return (r[0] * (0.2 + 0.05 * (calls[0] % 3)),)  # a different scaling every application

    b = (torch.ones(40, dtype=torch.float64, device="cuda"),)
    x, hist = gmres(lambda v: (A @ v[0],), prec, b, restart=10, max_restarts=30, rtol=1e-10)
    assert float(torch.linalg.norm(A @ x[0] - b[0])) <= 1e-9 * float(torch.linalg.norm(b[0]))


def test_gmres_zero_right_hand_side():
    from dndsr_b200.adjoint import gmres
    A, _ = _system(10)
    x, hist = gmres(lambda v: (A @ v[0],), lambda r: r, (torch.zeros(10, dtype=torch.float64, device="cuda"),))
    assert float(x[0].abs().max()) == 0.0 and hist == [1.0]
