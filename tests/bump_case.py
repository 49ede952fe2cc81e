"""The transonic bump channel set-up shared by the boundary-condition tests."""
import numpy as np

import oracle
from dndsr_b200 import mesh as M
from tests.util import VR_HQM

# EulerEvaluator.hpp:138-152: Dirichlet-type VR weights {1,0,0,0} on far-field, walls, symmetry
# and inflow (the default below); zero weight on supersonic outflow (BCOut); interior zones keep 1
BC_DIR_WEIGHT = {1: (1, 0, 0, 0), 3: (1, 0, 0, 0), 9: (1, 0, 0, 0), 5: (0, 0, 0, 0)}


def bump_bc(far, outflow_type=1, inflow_type=1, wall_type=3):
    types = np.zeros(7, np.int32)
    vals = np.zeros((7, len(far)))
    for z, tp in M.BUMP_BC_TYPES.items():
        types[z] = tp
        vals[z] = far
    types[M.BUMP_ZONES["outflow"]] = outflow_type
    types[M.BUMP_ZONES["inflow"]] = inflow_type
    types[M.BUMP_ZONES["bump"]] = wall_type  # an isothermal wall (4) takes its temperature from value[0]
    w = np.ones((7, 4))
    for z in range(1, 7):
        w[z] = BC_DIR_WEIGHT.get(int(types[z]), (1, 0, 0, 0))
    return types, vals, w


def bump_oracle(m, p, rs="Roe", mu=0.0, ignoreVis=1, mach=0.8, outflow_type=1, intOrder=5, inflow_type=1, wall_type=3):
    far = M.freestream(mach)
    types, vals, w = bump_bc(far, outflow_type, inflow_type, wall_type)
    es = dict(nVars=5, rsType=oracle.RS[rs], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=mu, prGas=0.72, TRef=273.15,
              CSutherland=110.4, muModel=0, ignoreVis=ignoreVis)
    o = oracle.Oracle(m, dict(VR_HQM, maxOrder=p, intOrder=intOrder), es)
    assert o.construct(w) == 0
    o.set_bc(types, vals)
    return o, far, types, vals, w


def perturbed_state(m, far, seed=3, R=None):
    """Freestream with smooth density, energy and vertical-velocity perturbations; optional random uRec."""
    X = m.cell_coords().mean(1)
    u = np.tile(far, (m.n_cell, 1))
    u[:, 0] *= 1 + 0.1 * np.sin(3 * X[:, 0]) * np.cos(2 * X[:, 1])
    u[:, 4] *= 1 + 0.05 * np.cos(2 * X[:, 0] + X[:, 2])
    u[:, 2] += 0.05 * np.sin(2 * X[:, 0])
    if R is None:
        return u
    rng = np.random.default_rng(seed)
    return u, rng.normal(size=(m.n_cell, R, 5)) * 0.01 * np.abs(u).mean(0)
