"""The SA flat-plate set-up shared by the turbulence-model tests: Re_L = 5e6, Mach 0.2,
nuTilde_inf = 3 nu (SA variable U5 = rho nuTilde / mu = 3), constant viscosity."""
import numpy as np

import oracle
from dndsr_b200 import mesh as M
from tests.util import VR_HQM

RE_L, MACH = 5e6, 0.2


def plate_state():
    far5 = M.freestream(MACH)
    mu = np.linalg.norm(far5[1:4]) / far5[0] * 1.0 / RE_L
    return np.concatenate([far5, [3.0 * far5[0]]]), mu


def plate_bc(far):
    types = np.zeros(6, np.int32)
    vals = np.zeros((6, len(far)))
    for z, tp in M.PLATE_BC_TYPES.items():
        types[z] = tp
        vals[z] = far
    w = np.ones((6, 4))
    for z in range(1, 6):
        w[z] = (1, 0, 0, 0)
    return types, vals, w


def plate_oracle(m, p, rs="Roe", intOrder=5):
    far, mu = plate_state()
    types, vals, w = plate_bc(far)
    es = dict(nVars=6, rsType=oracle.RS[rs], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=mu, prGas=0.72, TRef=273.15,
              CSutherland=110.4, muModel=0, ignoreVis=0)
    o = oracle.Oracle(m, dict(VR_HQM, maxOrder=p, intOrder=intOrder), es)
    assert o.construct(w) == 0
    o.set_bc(types, vals)
    o.set_wall_distance(M.plate_wall_distance(o.get("cellPP").reshape(m.n_cell, -1, 3)))
    return o, far, mu, types, vals, w


def plate_perturbed(m, far, R=None, seed=4):
    """Freestream with a boundary-layer-like velocity deficit and a smooth nuTilde profile."""
    X = m.cell_coords().mean(1)
    u = np.tile(far, (m.n_cell, 1))
    y = np.maximum(X[:, 1], 0)
    prof = 1 - np.exp(-y / 0.01) * (X[:, 0] > 0)
    u[:, 1:4] *= (0.3 + 0.7 * prof)[:, None]
    u[:, 5] *= 0.5 + 0.5 * prof + 2.0 * np.exp(-((y - 0.01) / 0.01) ** 2) * (X[:, 0] > 0)
    if R is None:
        return u
    rng = np.random.default_rng(seed)
    return u, rng.normal(size=(m.n_cell, R, 6)) * 1e-3 * np.abs(u).mean(0)
