"""Algorithmic flops per cell (F_alg) of the hot-path operators, counted by the op-counting build of the
oracle (oracle/opcount.hpp: +, -, *, / and sqrt one each; exp / pow / log / trigonometric one call each).

Test infrastructure: it runs the oracle's restatement of the reference algorithm (basis values recomputed
from the point coordinates, as in the reference with cacheDiffBase off) on a small mesh of each workload;
on periodic meshes every cell sees the same work, so the count per cell is that of the full-size workload.
Usage: python -m oracle.falg  (prints JSON)
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from dndsr_b200 import mesh as M  # noqa: E402

VR_HQM = dict(maxOrder=2, intOrder=5, jacobiRelax=1.0, SORInstead=0, scaleType=1, scaleMultiplier=1.0, dirWeightScheme=1,
              geomWeightScheme=1, geomWeightBias=1.0, geomWeightPower=0.5, bcWeight=1.0)


def _total(c):
    return sum(c.values())


def tgv(n=6, p=2):
    """The TGV workload: periodic hexahedra, VR degree p (intOrder 5), HLLE+ with the compact viscous flux."""
    m = M.tgv_mesh(n)
    es = dict(nVars=5, rsType=oracle.RS["HLLEP"], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=1 / 1600, prGas=0.71,
              TRef=273.15, CSutherland=110.4, muModel=0, ignoreVis=0)
    o = oracle.Oracle(m, dict(VR_HQM, maxOrder=p), es, opcount=True)
    assert o.construct() == 0
    u = o.init_field(3)
    uRec = np.random.default_rng(0).normal(size=(m.n_cell, o.R, 5)) * 1e-3
    o.eval_dt(u, 1.0)
    o.op_counts(reset=True)
    o.vr_iter(uRec, u)
    vr = o.op_counts(reset=True)
    o.eval_rhs(u, uRec)
    rhs = o.op_counts(reset=True)
    jd = o.lusgs_init(np.full(m.n_cell, 0.1), 1e100, 1.0)
    o.op_counts(reset=True)
    x0 = np.zeros_like(u)
    o.update_sgs(1.0, u, u, x0, x0, jd, True, True, False)
    sgs = o.op_counts(reset=True)
    return dict(workload=f"TGV hex, VR degree {p}, HLLE+ and compact viscous flux, intOrder 5", cells=m.n_cell,
                evaluate_rhs=dict(per_cell=_total(rhs) / m.n_cell, ops=rhs),
                vr_sweep=dict(per_cell=_total(vr) / m.n_cell, ops=vr),
                sgs_sweep_forward=dict(per_cell=_total(sgs) / m.n_cell, ops=sgs))


if __name__ == "__main__":
    out = dict(tgv_p2=tgv(6, 2), tgv_p1=tgv(6, 1))
    print(json.dumps(out, indent=1))
