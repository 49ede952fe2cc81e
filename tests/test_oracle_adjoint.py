"""The oracle's adjoint building blocks, pinned by properties that hold whatever the mesh:
the transposed LU-SGS operator is the transpose of LUSGSMatrixVec (EulerEvaluator.hxx:175-274),
Gauss-Seidel sweeps on it solve the transposed system, and the gradient of the pressure-force
objective matches central differences of the objective itself."""
import numpy as np
import pytest

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state

BUMP_WALL = M.BUMP_ZONES["bump"]


def _case(p=1, seed=0):
    m = M.bump_channel_tet(6, 3, 3, periodic_z=True)
    o, far, *_ = bump_oracle(m, p, "Roe", mach=0.5, intOrder=4)
    u, uRec = perturbed_state(m, far, seed=seed, R=o.R)
    return m, o, u, uRec


@pytest.mark.parametrize("cfl", [0.5, 50.0])
def test_transposed_matvec_is_the_transpose(cfl):
    m, o, u, uRec = _case()
    dTau, _ = o.eval_dt(u, cfl)
    jd = o.lusgs_init(dTau, 1e100, 1.0)
    rng = np.random.default_rng(7)
    for _ in range(3):
        x, y = rng.normal(size=u.shape), rng.normal(size=u.shape)
        lhs = float(np.sum(o.lusgs_matvec(1.0, u, x, jd) * y))
        rhs = float(np.sum(x * o.lusgs_matvec_t(1.0, u, y, jd)))
        assert abs(lhs - rhs) < 1e-12 * (abs(lhs) + 1.0)


def test_transposed_gauss_seidel_solves_the_transposed_system():
    m, o, u, uRec = _case()
    dTau, _ = o.eval_dt(u, 2.0)
    jd = o.lusgs_init(dTau, 1e100, 1.0)
    b = np.random.default_rng(3).normal(size=u.shape)
    y = np.zeros_like(b)
    r0 = np.linalg.norm(b)
    for _ in range(30):
        y = o.update_sgs_t(1.0, b, u, y, y, jd, True)
        y = o.update_sgs_t(1.0, b, u, y, y, jd, False)
    assert np.linalg.norm(o.lusgs_matvec_t(1.0, u, y, jd) - b) < 1e-10 * r0


@pytest.mark.parametrize("p", [1, 2])
def test_pressure_force_gradient_matches_central_differences(p):
    m, o, u, uRec = _case(p, seed=5)
    d = np.array([1.0, 0.0, 0.0])
    J, gU, gR = o.pressure_force(BUMP_WALL, d, u, uRec, grad=True)
    assert np.count_nonzero(np.abs(gU).sum(1)) > 0
    # only the cells of the bump faces carry a gradient
    bump_cells = set(m.face2cell[(m.face_zone == BUMP_WALL) & (m.face2cell[:, 1] < 0), 0])
    assert set(np.nonzero(np.abs(gU).sum(1))[0]) <= bump_cells
    rng = np.random.default_rng(11)
    h = 1e-6
    for _ in range(4):
        du = rng.normal(size=u.shape) * np.abs(u).mean(0)
        dr = rng.normal(size=uRec.shape) * 0.1 * np.abs(u).mean(0)
        fd = (o.pressure_force(BUMP_WALL, d, u + h * du, uRec + h * dr) - o.pressure_force(BUMP_WALL, d, u - h * du, uRec - h * dr)) / (2 * h)
        an = float(np.sum(gU * du) + np.sum(gR * dr))
        assert abs(fd - an) < 1e-7 * abs(an)
    # a uniform pressure on the closed bump-plus-floor surface gives no net force along x only when
    # the wall is flat: the bump's projected area makes J of the freestream p * (projected area) = 0
    far = M.freestream(0.5)
    u0 = np.tile(far, (m.n_cell, 1))
    J0 = o.pressure_force(BUMP_WALL, d, u0, np.zeros_like(uRec))
    assert abs(J0) < 1e-12
