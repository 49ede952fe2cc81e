"""Host-side pieces of the adjoint driver (dndsr_b200/adjoint.py) on CPU tensors: the right-
preconditioned restarted GMRES on tuples of tensors solves nonsymmetric systems to the requested
drop, with a fixed and with a varying (flexible) preconditioner, and returns its residual history."""
import numpy as np
import torch

from dndsr_b200.adjoint import gmres


def _system(n=60, seed=0):
    rng = np.random.default_rng(seed)
    A = np.eye(n) * 4 + rng.normal(size=(n, n)) * 0.3
    B = rng.normal(size=(n // 2, n // 2)) * 0.2 + np.eye(n // 2) * 2
    return torch.tensor(A), torch.tensor(B)


def test_gmres_solves_a_two_block_system():
    A, B = _system()
    n, m = A.shape[0], B.shape[0]

    def op(x):
        return (A @ x[0] + 0.1 * torch.cat([x[1], x[1]]), B @ x[1])

    prec = lambda r: (r[0] / 4, r[1] / 2)
    rng = np.random.default_rng(1)
    b = (torch.tensor(rng.normal(size=n)), torch.tensor(rng.normal(size=m)))
    x, hist = gmres(op, prec, b, restart=8, max_restarts=50, rtol=1e-12)
    r = tuple(bi - oi for bi, oi in zip(b, op(x)))
    rn = float(sum((ri * ri).sum() for ri in r)) ** 0.5
    bn = float(sum((bi * bi).sum() for bi in b)) ** 0.5
    assert hist[-1] <= 1e-12 and rn <= 1e-11 * bn
    assert hist[0] == 1.0 and all(h >= 0 for h in hist)


def test_gmres_with_a_varying_preconditioner():
    A, _ = _system(40, seed=3)
    calls = [0]

    def prec(r):
        calls[0] += 1
        return (r[0] * (0.2 + 0.05 * (calls[0] % 3)),)  # a different scaling every application

    b = (torch.ones(40, dtype=torch.float64),)
    x, hist = gmres(lambda v: (A @ v[0],), prec, b, restart=10, max_restarts=30, rtol=1e-10)
    assert float(torch.linalg.norm(A @ x[0] - b[0])) <= 1e-9 * float(torch.linalg.norm(b[0]))


def test_gmres_zero_right_hand_side():
    A, _ = _system(10)
    x, hist = gmres(lambda v: (A @ v[0],), lambda r: r, (torch.zeros(10, dtype=torch.float64),))
    assert float(x[0].abs().max()) == 0.0 and hist == [1.0]
