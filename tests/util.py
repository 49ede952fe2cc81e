"""Shared configuration of the parity tests."""
import numpy as np

import oracle

VR_HQM = dict(maxOrder=2, intOrder=5, jacobiRelax=1.0, SORInstead=0, scaleType=1, scaleMultiplier=1.0, dirWeightScheme=1,
              geomWeightScheme=1, geomWeightBias=1.0, geomWeightPower=0.5, bcWeight=1.0)
VR_HQM_PY = dict(maxOrder=2, intOrder=5, dirWeightScheme="HQM_OPT", geomWeightScheme="HQM_SD", geomWeightBias=1.0, geomWeightPower=0.5)


def oracle_for(mesh, p, rs="Roe", mu=1e-3, muModel=0, nv=5, ignoreVis=0):
    vr = dict(VR_HQM, maxOrder=p)
    es = dict(nVars=nv, rsType=oracle.RS[rs], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=mu, prGas=0.72,
              TRef=273.15, CSutherland=110.4, muModel=muModel, ignoreVis=ignoreVis)
    o = oracle.Oracle(mesh, vr, es)
    assert o.construct() == 0
    return o


def relerr(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
