"""The oracle's WBAP_C limiter (VariationalReconstruction_LimiterProcedure.hxx:40-334, Limiters.hpp
:361-470, VariationalReconstruction.cpp:840-866, Gas.hpp:120-200): properties the reference's
procedure guarantees, with no mesh file needed.

* an exactly linear field (cell means and reconstruction of rho, rho v, E linear in x; on a mesh
  periodic in z, linear in x and y) has a zero
  smooth indicator, and limiting every cell leaves it unchanged: matrixSecondary maps each
  neighbour's gradient into this cell's basis exactly, the left and right eigenvector matrices are
  inverse, and WBAP of equal candidates returns them;
* at a discontinuity the indicator is large and limiting shrinks the reconstruction (a WBAP
  average of the candidates, zero where their signs disagree);
* cells below the threshold are copied."""
import numpy as np

from dndsr_b200 import mesh as M
from tests.util import oracle_for


def _linear(o, m, z_gradient=True):
    bary = o.get("cellBary").reshape(-1, 3)
    L = o.get("cellHBox").reshape(-1, 3).max(1)
    g = np.array([[0.1, 0.05, -0.02, 0.0, 0.3], [0.02, -0.1, 0.0, 0.05, 0.2], [0.0, 0.03, 0.1, 0.0, -0.1]])
    if not z_gradient:  # periodic in z: a field linear in x and y only stays continuous across it
        g[2] = 0
    u = np.array([1.0, 0.2, 0.1, 0.05, 3.0]) + bary @ g
    uRec = np.zeros((m.n_cell, o.R, 5))
    for d in range(3):
        uRec[:, d, :] = g[d] * L[:, None]
    return u, uRec


def test_linear_field_is_left_unchanged():
    # tetrahedra in the bump channel (no periodic faces); hexahedra of the plate (periodic in z)
    for m, zg in ((M.bump_channel_tet(6, 4, 2), True), (M.flat_plate_hex(8, 6, 3), False)):
        for p in (1, 2):
            o = oracle_for(m, p, "Roe", mu=0.0, ignoreVis=1)
            u, uRec = _linear(o, m, zg)
            si = o.smooth_indicator(u, uRec)
            assert si.max() < 1e-12
            out = o.limiter_wbap_c(u, uRec, si, ifAll=True)
            assert np.abs(out - uRec).max() < 1e-13 * np.abs(uRec).max()


def test_discontinuity_is_detected_and_limited():
    m = M.tgv_mesh(6)
    for p in (1, 2):
        o = oracle_for(m, p, "Roe", mu=0.0, ignoreVis=1)
        u = np.tile(np.array([1.0, 0.2, 0.1, 0.05, 3.0]), (m.n_cell, 1))
        X = m.cell_coords().mean(1)
        jump = X[:, 0] > np.pi
        u[jump, 0] *= 3.0
        u[jump, 4] *= 3.0
        rng = np.random.default_rng(4)
        uRec = rng.normal(size=(m.n_cell, o.R, 5)) * 1e-3
        si = o.smooth_indicator(u, uRec)
        assert si.max() > 0.1 and si.min() < 0.01
        out = o.limiter_wbap_c(u, uRec, si)
        smooth = si < 0.01
        assert np.array_equal(out[smooth], uRec[smooth])
        assert np.abs(out[~smooth]).sum() < np.abs(uRec[~smooth]).sum()
