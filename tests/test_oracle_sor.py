"""The oracle's SOR reconstruction sweep (SORInstead, VariationalReconstruction_Reconstruction.hxx:534-611) on CPU.

On a periodic mesh its fixed point is the Jacobi sweep's (both solve the same VR system) and it gets there in
fewer sweeps.  On a mesh with boundary faces the reference's in-place update evaluates GetBoundaryRHS from the
cell's partially updated row (with jacobiRelax 1 the row holds only the terms of the faces before the boundary
face in the cell's face order), so the SOR sweep converges to a different fixed point there; the oracle keeps
that behaviour, and the test records that it converges and that the two fixed points differ."""
import numpy as np

import oracle
from dndsr_b200 import mesh as M
from tests.bump_case import bump_oracle, perturbed_state
from tests.util import VR_HQM


def _iterate(o, u0, R, n):
    rj = np.zeros((u0.shape[0], R, u0.shape[1]))
    rs = rj.copy()
    hj, hs = [], []
    for _ in range(n):
        nj, ns = o.vr_iter(rj, u0), o.vr_iter_sor(rs, u0)
        hj.append(np.abs(nj - rj).max())
        hs.append(np.abs(ns - rs).max())
        rj, rs = nj, ns
    return rj, rs, hj, hs


def test_sor_fixed_point_on_a_periodic_mesh():
    m = M.renumber_by_color(M.tgv_mesh(4))
    es = dict(nVars=5, rsType=oracle.RS["HLLEP"], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=1e-3, prGas=0.72, TRef=273.15,
              CSutherland=110.4, muModel=0, ignoreVis=0)
    o = oracle.Oracle(m, dict(VR_HQM, maxOrder=2), es)
    assert o.construct() == 0
    u0 = o.init_field(3)
    rj, rs, hj, hs = _iterate(o, u0, o.R, 300)
    assert hs[-1] < 1e-13 * np.abs(rs).max() and hj[-1] < 1e-10 * np.abs(rj).max(), (hs[-1], hj[-1])
    assert np.abs(rs - rj).max() < 1e-9 * np.abs(rj).max()
    assert hs[20] < 0.2 * hj[20], (hs[20], hj[20])  # Gauss-Seidel ahead of Jacobi


def test_sor_with_boundary_faces_reads_the_partial_row():
    m = M.renumber_by_color(M.bump_channel_tet(4, 3, 2))
    o, far, types, vals, w = bump_oracle(m, 2, "Roe", 0.0, 1)
    u0, _ = perturbed_state(m, far, R=o.R)
    rj, rs, hj, hs = _iterate(o, u0, o.R, 400)
    assert hs[-1] < 1e-12 * np.abs(rs).max(), hs[-1]
    assert np.abs(o.vr_iter_sor(rs, u0) - rs).max() < 1e-12 * np.abs(rs).max()
    # cells without a boundary face see no difference in their own update rule; the boundary term differs
    assert np.abs(rs - rj).max() > 1e-3 * np.abs(rj).max()
