"""Boundary conditions of the CPU oracle: properties that hold for the reference's
generateBoundaryValue / GetBoundaryRHS (EulerEvaluator_EvaluateDt.hxx:1743-2468,
VariationalReconstruction_Reconstruction.hxx:19-176) whatever the mesh.  No reference
golden covers boundary faces, so these properties pin the restatement."""
import numpy as np
import pytest

from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state


def test_bump_mesh_is_valid():
    m = M.bump_channel_tet(8, 4, 3)
    X = m.cell_coords()
    v6 = np.einsum("ij,ij->i", np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), X[:, 3] - X[:, 0])
    assert m.n_cell == 6 * 8 * 4 * 3 and v6.min() > 0
    # boundary nodes are not jittered: the volume is the channel minus the piecewise-linear bump
    x = np.linspace(-2, 2, 9)
    bump = np.trapezoid(M.bump_height(x), x) * 0.5
    assert abs(v6.sum() / 6 - (2.0 - bump)) < 1e-12
    bnd = m.face2cell[:, 1] < 0
    assert set(np.unique(m.face_zone[bnd])) == set(M.BUMP_ZONES.values()) and np.all(m.face_zone[~bnd] == 0)


def test_bump_mesh_with_periodic_sides():
    m = M.bump_channel_tet(8, 4, 3, periodic_z=True)
    X = m.cell_coords()
    v6 = np.einsum("ij,ij->i", np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), X[:, 3] - X[:, 0])
    x = np.linspace(-2, 2, 9)
    assert v6.min() > 0 and abs(v6.sum() / 6 - (2.0 - np.trapezoid(M.bump_height(x), x) * 0.5)) < 1e-12
    bnd = m.face2cell[:, 1] < 0
    assert set(np.unique(m.face_zone[bnd])) == {1, 2, 3, 4}
    per = np.abs(m.face_pshift[:, 2]) > 0
    assert np.allclose(np.abs(m.face_pshift[per, 2]), 0.5) and per.sum() == 2 * 8 * 4


@pytest.mark.parametrize("p", [1, 2])
def test_freestream_is_preserved_in_a_flat_channel(p):
    m = M.bump_channel_tet(6, 3, 2, amp=0.0)
    o, far, *_ = bump_oracle(m, p)
    u = np.tile(far, (m.n_cell, 1))
    uRec = np.zeros((m.n_cell, o.R, 5))
    o.eval_dt(u, 1.0)
    assert np.abs(o.eval_rhs(u, uRec)).max() < 1e-12
    assert np.abs(o.vr_iter(uRec, u)).max() == 0


def test_slip_walls_carry_no_mass_flux():
    m = M.bump_channel_tet(6, 4, 2)
    o, far, *_ = bump_oracle(m, 2)
    u, uRec = perturbed_state(m, far, R=o.R)
    o.eval_dt(u, 1.0)
    _, ff = o.eval_rhs(u, uRec, want_face_flux=True)
    wall = np.isin(m.face_zone, [M.BUMP_ZONES[k] for k in ("bump", "top", "side0", "side1")])
    assert np.abs(ff[wall, 0]).max() < 1e-12 * np.abs(ff[:, 0]).max()
    assert np.abs(ff[wall, 1:4]).max() > 0  # pressure acts on the walls


def test_supersonic_outflow_copies_the_inner_state():
    m = M.bump_channel_tet(6, 4, 2)
    o1, far, *_ = bump_oracle(m, 1, mach=0.8, outflow_type=5)
    u = np.tile(far, (m.n_cell, 1))
    uRec = np.zeros((m.n_cell, o1.R, 5))
    o1.eval_dt(u, 1.0)
    _, ff = o1.eval_rhs(u, uRec, want_face_flux=True)
    out = m.face_zone == M.BUMP_ZONES["outflow"]
    # UR = UL: the Riemann flux is the physical flux of the inner state
    n = o1.get("faceMeanNorm").reshape(-1, 3)[out]
    A = o1.get("faceArea")[out]
    rho_un = (far[1:4] @ n.T)
    assert np.allclose(-ff[out, 0], rho_un * A, rtol=1e-12)
