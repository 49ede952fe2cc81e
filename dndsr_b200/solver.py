"""Python mirror of the reference's VR / Euler evaluator call surface on torch CUDA tensors.

Class and method names follow CFV::VariationalReconstruction
(src/CFV/VariationalReconstruction.hpp:108-1114, bound in
src/CFV/VariationalReconstruction_bind.hpp:19-145) and
Euler::EulerEvaluator (src/Euler/EulerEvaluator.hpp:76-1980).  State arrays
are caller-owned contiguous float64 CUDA tensors.  Every call goes through the
pybind11 module ``dndsr_b200._C`` (csrc/pybind.cpp), which calls the C-ABI of
include/dndsb.h on torch's current stream; this layer adds the reference's
setting names and defaults and allocates result tensors.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from .mesh import Mesh

# reference setting names -> C struct codes
_SCALE = {"MeanAACBB": 0, "BaryDiff": 1}
_DIRW = {"Factorial": 0, "HQM_OPT": 1, "ManualDirWeight": 999}
_GEOMW = {"GWNone": 0, "HQM_SD": 1, "SD_Power": 2}
RS = dict(Roe=1, HLLC=2, HLLEP=3, HLLEP_V1=21, Roe_M1=11, Roe_M2=12, Roe_M3=13, Roe_M4=14, Roe_M5=15, Roe_M6=16, Roe_M7=17,
          Roe_M8=18)

VR_DEFAULTS = dict(maxOrder=1, intOrder=1, jacobiRelax=1.0, SORInstead=False, anisotropicLengths=False, scaleType="BaryDiff",
                   scaleMultiplier=1.0, dirWeightScheme="Factorial", manualDirWeights=(1, 1, 0.5, 1.0 / 6), geomWeightScheme="GWNone",
                   geomWeightBias=0.0, geomWeightPower=0.5, geomWeightPower1=0.0, geomWeightPower2=0.0, bcWeight=1.0)
EULER_DEFAULTS = dict(nVars=5, riemannSolverType="Roe", rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=1.0, prGas=0.72,
                      TRef=273.15, CSutherland=110.4, muModel=1, ignoreVis=False, rsMeanValueEig=0, useScalarJacobian=True,
                      useRoeJacobian=False)


# boundary condition codes, Euler/EulerBC.hpp:35-48
BC = dict(BCFar=1, BCWall=2, BCWallInvis=3, BCWallIsothermal=4, BCOut=5, BCOutP=6, BCIn=7, BCSym=9)


def euler_bc_dir_weights(types, maxOrder=3):
    """Per-zone VR face weights of the Euler boundary types (EulerEvaluator.hpp:138-152, the
    callback InitializeFV passes to ConstructBaseAndWeight): Dirichlet-type {1, 0, 0, 0} for
    far-field, walls, symmetry and inflow, nothing for outflow; interior zones keep 1."""
    w = np.ones((len(types), 4))
    for z, t in enumerate(types):
        t = BC[t] if isinstance(t, str) else int(t)
        if t == 0:
            continue
        if t == BC["BCOut"]:
            w[z] = 0.0
        else:
            w[z] = (1.0, 0.0, 0.0, 0.0)
    return w


def _C():
    """The pybind11 module; there is no CPU path, so a host without a CUDA device is refused here."""
    if not torch.cuda.is_available():
        raise RuntimeError("dndsr_b200 needs a CUDA device; there is no CPU path")
    from . import build as _b
    if not os.path.exists(_b.LIB):
        raise ImportError("dndsr_b200/libdndsb.so is missing: run dndsr_b200/build.py (nvcc, sm_100a)")
    from . import _C as mod
    return mod


class DeviceMesh:
    """Uploads a :class:`dndsr_b200.mesh.Mesh` (replaces Geom::UnstructuredMesh as the VR input)."""

    def __init__(self, mesh: Mesh):
        C = _C()
        self.mesh = mesh
        a = mesh.arrays()
        self._c = C.Mesh(mesh.dim, mesh.cell_type, mesh.face_type, a["coords"], a["cell2node"], a["cell_shift"], a["face2node"],
                         a["face_shift"], a["face2cell"], a["face_zone"], a["face_pshift"], a["cell2face"])

    def colors(self):
        return self._c.colors()


def _code(table, x):
    return table[x] if isinstance(x, str) else int(x)


class VariationalReconstruction:
    """CFV::VariationalReconstruction<dim> on the GPU."""

    def __init__(self, mesh, settings: dict | None = None):
        self.dmesh = mesh if isinstance(mesh, DeviceMesh) else DeviceMesh(mesh)
        self.mesh = self.dmesh.mesh
        s = dict(VR_DEFAULTS)
        s.update(settings or {})
        self.settings = s
        cs = dict(maxOrder=int(s["maxOrder"]), intOrder=int(s["intOrder"]), jacobiRelax=float(s["jacobiRelax"]),
                  SORInstead=int(bool(s["SORInstead"])), anisotropicLengths=int(bool(s["anisotropicLengths"])),
                  scaleType=_code(_SCALE, s["scaleType"]), scaleMultiplier=float(s["scaleMultiplier"]),
                  dirWeightScheme=_code(_DIRW, s["dirWeightScheme"]), manualDirWeights=[float(x) for x in s["manualDirWeights"]][:4],
                  geomWeightScheme=_code(_GEOMW, s["geomWeightScheme"]), geomWeightBias=float(s["geomWeightBias"]),
                  geomWeightPower=float(s["geomWeightPower"]), geomWeightPower1=float(s["geomWeightPower1"]),
                  geomWeightPower2=float(s["geomWeightPower2"]), bcWeight=float(s["bcWeight"]))
        self._c = _C().VariationalReconstruction(self.dmesh._c, cs)

    # VariationalReconstruction.cpp:10-43, :56-498, :507-872
    def ConstructMetrics(self):
        self._c.ConstructMetrics()

    def ConstructBaseAndWeight(self, bc_dir_weight=None):
        self._c.ConstructBaseAndWeight(None if bc_dir_weight is None else np.ascontiguousarray(bc_dir_weight, dtype=np.float64).reshape(-1, 4))

    def ConstructRecCoeff(self):
        self._c.ConstructRecCoeff()
        self.NDOF, self.R, self.nGf, self.nGc = [int(x) for x in self._c.sizes()]

    def construct(self, bc_dir_weight=None):
        self.ConstructMetrics()
        self.ConstructBaseAndWeight(bc_dir_weight)
        self.ConstructRecCoeff()
        return self

    def get(self, name):
        return self._c.get(name)

    # VariationalReconstruction.hpp:920-1000 BuildURec / FiniteVolume BuildUDof
    def BuildURec(self, nVars):
        return torch.zeros((self.mesh.n_cell, self.R, nVars), dtype=torch.float64, device="cuda")

    def BuildUDof(self, nVars):
        return torch.zeros((self.mesh.n_cell, nVars), dtype=torch.float64, device="cuda")

    def DoReconstructionIter(self, uRec, uRecNew, u, putIntoNew=False, recordInc=False, uRecIsZero=False, precision="fp64"):
        """VariationalReconstruction_Reconstruction.hxx:485-615 (Jacobi sweep)."""
        self._c.DoReconstructionIter(uRec, uRecNew, u, u.shape[1], bool(putIntoNew), bool(recordInc), bool(uRecIsZero),
                                     1 if precision == "fp32" else 0)

    def DoReconstructionIterVJP(self, cot, uRec, u):
        """Vector-Jacobian product of one Jacobi sweep uRecNew = S(uRec, u): returns
        ((dS/duRec)^T cot, (dS/du)^T cot)."""
        vRec, vU = torch.empty_like(uRec), torch.empty_like(u)
        self._c.DoReconstructionIterVJP(cot, uRec, u, u.shape[1], vRec, vU)
        return vRec, vU

    def DoReconstructionIterJVP(self, dRec, du, uRec, u):
        """Jacobian-vector product of one Jacobi sweep (DoReconstructionIterDiff with the
        linearised boundary term): dS/duRec dRec + dS/du du."""
        out = torch.empty_like(uRec)
        self._c.DoReconstructionIterJVP(dRec, du, uRec, u, u.shape[1], out)
        return out

    def DoCalculateSmoothIndicator(self, u, uRec):
        """VariationalReconstruction_LimiterProcedure.hxx:40-108 (procedure 0, density and energy): si [nCell]."""
        si = torch.empty(self.mesh.n_cell, dtype=torch.float64, device="cuda")
        self._c.DoCalculateSmoothIndicator(u, uRec, u.shape[1], si)
        return si

    def DoReconstructionIterVJPCoords(self, cot, uRec, u):
        """(dS/dX)^T cot for one Jacobi sweep uRecNew = S(uRec, u; X), X the node coordinates
        [nNode][3]: the geometry, basis moments, weights and A^-1 B / A^-1 b are differentiated."""
        dX = torch.empty((self.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        self._c.DoReconstructionIterVJPCoords(cot, uRec, u, u.shape[1], dX)
        return dX

    def DoReconstructionIterJVPCoords(self, dX, uRec, u):
        """dS/dX dX for one Jacobi sweep along the node displacement dX [nNode][3]."""
        out = torch.empty_like(uRec)
        self._c.DoReconstructionIterJVPCoords(dX, uRec, u, u.shape[1], out)
        return out


class EulerEvaluator:
    """Euler::EulerEvaluator<model> on the GPU (models NS / NS_3D with 5 variables, NS_SA with 6)."""

    # EvaluateRHS flags, EulerEvaluator.hpp:370-378
    RHS_No_Flags, RHS_Ignore_Viscosity, RHS_Dont_Update_Integration, RHS_Dont_Record_Bud_Flux = 0, 1, 2, 4

    def __init__(self, vr: VariationalReconstruction, settings: dict | None = None):
        self.vr = vr
        s = dict(EULER_DEFAULTS)
        s.update(settings or {})
        self.settings = s
        cs = dict(nVars=int(s["nVars"]), rsType=_code(RS, s["riemannSolverType"]), rsFixScale=float(s["rsFixScale"]),
                  rsIncFScale=float(s["rsIncFScale"]), gamma=float(s["gamma"]), Rgas=float(s["Rgas"]), muGas=float(s["muGas"]),
                  prGas=float(s["prGas"]), TRef=float(s["TRef"]), CSutherland=float(s["CSutherland"]), muModel=int(s["muModel"]),
                  ignoreVis=int(bool(s["ignoreVis"])), rsMeanValueEig=int(s["rsMeanValueEig"]))
        self._c = _C().EulerEvaluator(vr._c, cs)
        self.nVars = cs["nVars"]
        self.SetJacobianMode(bool(s["useScalarJacobian"]) and not bool(s["useRoeJacobian"]), bool(s["useRoeJacobian"]))

    def SetJacobianMode(self, useScalarJacobian=True, useRoeJacobian=False):
        """EulerEvaluatorSettings useScalarJacobian / useRoeJacobian (EulerEvaluatorSettings.hpp:53-54): the scalar
        diagonal, block diagonal blocks, or block diagonal blocks with the Roe term; BuildJDiag follows the mode."""
        self._c.SetJacobianMode(bool(useScalarJacobian), bool(useRoeJacobian))
        self.blockJacobian = not useScalarJacobian
        self.useRoeJacobian = bool(useRoeJacobian)

    def SetBC(self, types, values):
        """BoundaryHandler of the evaluator (Euler/EulerBC.hpp) as a per-zone table: types[zone]
        (EulerBC.hpp codes or names, 0 for interior zones) and values[zone] (far-field / inflow
        state, or wall temperature first).  Also the reconstruction's FBoundary."""
        t = np.array([BC[x] if isinstance(x, str) else int(x) for x in types], dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(len(t), self.nVars)
        self._bc = (t, v)
        self._c.SetBC(t, v)

    def SetWallDistance(self, d):
        """dWall of the SA model at every cell Gauss point, [nCell][nGc] host array."""
        self._c.SetWallDistance(np.ascontiguousarray(d, dtype=np.float64))

    def InitializeUDOF(self, u, kind, chi=5.0):
        self._c.InitializeUDOF(u, int(kind), float(chi))

    def EvaluateDt(self, dt, u, CFL, MaxDt=1e100, UseLocaldt=True, want_min=True):
        """Returns the global minimum of dt (want_min=False with UseLocaldt: no host synchronisation, None)."""
        return self._c.EvaluateDt(dt, u, float(CFL), float(MaxDt), bool(UseLocaldt), bool(want_min))

    def EvaluateRHS(self, rhs, u, uRec, JSource=None, uRecUnlim=None, uRecBeta=None, cellRHSAlpha=None, onlyOnHalfAlpha=False, t=0.0,
                    flags=0):
        """EvaluateRHS (EulerEvaluator_EvaluateRHS.hxx:55-818).  The short form (rhs, u, uRec) evaluates with
        the reconstruction uRec for values and gradients.  The keyword form is the reference's full
        contract: uRecUnlim gives the gradients (uRec the limited point values), cellRHSAlpha scales the
        SA source, JSource [nCell][nVars] receives the source Jacobian diagonal, flags are RHS_* bits;
        uRecBeta, onlyOnHalfAlpha and t are accepted and not read, as in the reference's body."""
        if JSource is None and uRecUnlim is None and cellRHSAlpha is None and flags == 0:
            self._c.EvaluateRHS(rhs, u, uRec)
            return
        self._c.EvaluateRHSFull(rhs, JSource, u, uRecUnlim if uRecUnlim is not None else uRec, uRec, uRecBeta, cellRHSAlpha,
                                bool(onlyOnHalfAlpha), float(t), int(flags))

    def SetDeferredErrors(self, deferred=True):
        """EvaluateRHS stops reading its error word back on every call; CheckErrors reads it."""
        self._c.SetDeferredErrors(bool(deferred))

    def CheckErrors(self):
        """Reads and clears the deferred error word of EvaluateRHS (raises DndsbError on a non-physical or
        non-finite state seen since the last check)."""
        self._c.CheckErrors()

    def EvaluateRHSNoAlloc(self, rhs, u, uRec):
        """EvaluateRHS without any device allocation: the face-flux scratch is a
        static 8 MiB device array (nFace * nVars <= capi.NOALLOC_SCRATCH_DOUBLES).
        For callers that cannot allocate device memory when they evaluate a
        residual; calls that overlap on the same GPU share the array and race."""
        self._c.EvaluateRHSNoAlloc(rhs, u, uRec)

    def EvaluateRHSVJP(self, w, u, uRec):
        """(dR/du)^T w and (dR/duRec)^T w of EvaluateRHS at (u, uRec), deltaLambdaCell held fixed."""
        du, duRec = torch.empty_like(u), torch.empty_like(uRec)
        self._c.EvaluateRHSVJP(w, u, uRec, du, duRec)
        return du, duRec

    def WallFluxVJP(self, direction, u, uRec):
        """(dJ/du, dJ/duRec) of the wall-flux integral J = direction . fluxWallSum (EvaluateRHS.hxx:599-607; the x
        force on the walls for direction (0, 1, 0, 0, 0[, 0])), deltaLambdaCell held fixed.  J itself is
        direction . get("fluxWallSum") after an EvaluateRHS at (u, uRec)."""
        du, duRec = torch.empty_like(u), torch.empty_like(uRec)
        self._c.WallFluxVJP(np.ascontiguousarray(direction, dtype=np.float64), u, uRec, du, duRec)
        return du, duRec

    def EvaluateRHSJVP(self, du, duRec, u, uRec):
        """dR/du du + dR/duRec duRec of EvaluateRHS at (u, uRec), deltaLambdaCell held fixed."""
        out = torch.empty_like(u)
        self._c.EvaluateRHSJVP(du, duRec, u, uRec, out)
        return out

    def EvaluateRHSVJPCoords(self, w, u, uRec):
        """(dR/dX)^T w of EvaluateRHS with respect to the node coordinates X [nNode][3] (u, uRec
        and deltaLambdaCell held fixed)."""
        dX = torch.empty((self.vr.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        self._c.EvaluateRHSVJPCoords(w, u, uRec, dX)
        return dX

    def ResidualVJPCoords(self, w, cot, u, uRec):
        """(dR/dX)^T w + (dS/dX)^T cot in one pass (S: one VR sweep of this evaluator's reconstruction)."""
        dX = torch.empty((self.vr.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        self._c.ResidualVJPCoords(w, cot, u, uRec, dX)
        return dX

    def EvaluateRHSJVPCoords(self, dX, u, uRec):
        """dR/dX dX of EvaluateRHS along the node displacement dX [nNode][3]."""
        out = torch.empty_like(u)
        self._c.EvaluateRHSJVPCoords(dX, u, uRec, out)
        return out

    def BuildJDiag(self):
        """Diagonal array of LUSGSMatrixInit: [nCell] (one value per cell), or [nCell][nVars] for the SA model; in block
        mode [nCell][2][nVars][nVars], the blocks and their inverses."""
        n = self.vr.mesh.n_cell
        if self.blockJacobian:
            return torch.zeros((n, 2, self.nVars, self.nVars), dtype=torch.float64, device="cuda")
        return torch.zeros((n, self.nVars) if self.nVars == 6 else (n,), dtype=torch.float64, device="cuda")

    def _jd(self, jdiag):
        """jdiag must have the layout of the Jacobian mode (the library reads it with that size)."""
        n = self.vr.mesh.n_cell
        want = n * 2 * self.nVars * self.nVars if self.blockJacobian else n * (self.nVars if self.nVars == 6 else 1)
        if jdiag.numel() != want or jdiag.dtype != torch.float64:
            raise ValueError(f"jdiag: {want} float64 values expected for this Jacobian mode (BuildJDiag), got {jdiag.numel()}")
        return jdiag

    def LUSGSMatrixInit(self, jdiag, dTau, dt, alphaDiag, u=None, uRec=None, jacobianCode=0, t=0.0):
        """EulerEvaluator.hxx:37-159; u is needed by the Roe Jacobian."""
        self._jd(jdiag)
        if u is None and not self.useRoeJacobian:
            self._c.LUSGSMatrixInit(jdiag, dTau, float(dt), float(alphaDiag))
        else:
            self._c.LUSGSMatrixInitFull(jdiag, dTau, float(dt), float(alphaDiag), u, uRec, int(jacobianCode), float(t))

    def UpdateSGS(self, alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward, gsUpdate=True, uIncIsZero=False, want_sum=True):
        s = self._c.UpdateSGS(float(alphaDiag), rhs, u, uInc, uIncNew, self._jd(jdiag), bool(forward), bool(gsUpdate), bool(uIncIsZero), bool(want_sum))
        return s if want_sum else np.zeros(self.nVars)

    def LUSGSMatrixToJacobianLU(self, alphaDiag, u, jdiag):
        """EulerEvaluator.hxx:290-359 + JacobianLocalLU::InPlaceDecompose (iluCode 0): the evaluator keeps the factors."""
        self._c.LUSGSMatrixToJacobianLU(float(alphaDiag), u, self._jd(jdiag))

    def LUSGSMatrixSolveJacobianLU(self, alphaDiag, rhs, u, uInc, uIncNew, jdiag, uIncIsZero=False, want_sum=True):
        """EulerEvaluator.hxx:838-927: uIncNew = (LU)^-1 (rhs - A uInc) + uInc; returns sumInc."""
        s = self._c.LUSGSMatrixSolveJacobianLU(float(alphaDiag), rhs, u, uInc, uIncNew, self._jd(jdiag), bool(uIncIsZero), bool(want_sum))
        return s if want_sum else np.zeros(self.nVars)

    def UpdateLUSGSForward(self, alphaDiag, rhs, u, uInc, jdiag, uIncNew):
        """EulerEvaluator.hxx:376-451: uIncNew = D^-1 (rhs - lower-neighbour flux increments of uInc).
        uInc may be uIncNew itself (the in-place sweep of the reference's callers)."""
        self._c.UpdateLUSGSForward(float(alphaDiag), rhs, u, uInc, self._jd(jdiag), uIncNew)

    def UpdateLUSGSBackward(self, alphaDiag, rhs, u, uInc, jdiag, uIncNew):
        """EulerEvaluator.hxx:453-529: uIncNew += D^-1 (- upper-neighbour flux increments of uInc)."""
        self._c.UpdateLUSGSBackward(float(alphaDiag), rhs, u, uInc, self._jd(jdiag), uIncNew)

    def FixUMaxFilter(self, u):
        """EulerEvaluator.hxx:1318-1323: the reference's filter returns without changing u."""
        self._c.FixUMaxFilter(u)

    def LUSGSMatrixVec(self, alphaDiag, u, uInc, jdiag, AuInc):
        self._c.LUSGSMatrixVec(float(alphaDiag), u, uInc, self._jd(jdiag), AuInc)

    def LUSGSMatrixVecT(self, alphaDiag, u, y, jdiag, ATy):
        """ATy = A^T y for the operator A of LUSGSMatrixVec (same lambdaFace, jdiag, alphaDiag)."""
        self._c.LUSGSMatrixVecT(float(alphaDiag), u, y, jdiag, ATy)

    def UpdateSGST(self, alphaDiag, b, u, y, yNew, jdiag, forward, gsUpdate=True):
        """One Gauss-Seidel sweep on A^T y = b (the transpose of UpdateSGS), colour by colour; b, y and
        yNew are all float64 or all float32 (the FP32 preconditioner)."""
        fp32 = b.dtype == torch.float32
        if any((t.dtype == torch.float32) != fp32 for t in (y, yNew)):
            raise TypeError("UpdateSGST: b, y and yNew must share one precision")
        self._c.UpdateSGST(float(alphaDiag), b, u, y, yNew, jdiag, bool(forward), bool(gsUpdate), bool(fp32))

    def PressureForce(self, zone, direction, u, uRec, grad=False):
        """Pressure force along direction on boundary zone; with grad also (dJ/du, dJ/duRec) as device tensors."""
        d = np.ascontiguousarray(direction, dtype=np.float64)
        gU = torch.empty_like(u) if grad else None
        gR = torch.empty_like(uRec) if grad else None
        J = self._c.PressureForce(int(zone), d, u, uRec, gU, gR)
        return (J, gU, gR) if grad else J

    def DoLimiterWBAP_C(self, u, uRec, si, uRecNew, smoothThreshold=0.01, WBAP_nStd=10.0, ifAll=False):
        """VariationalReconstruction_LimiterProcedure.hxx:188-334 with the characteristic projections of
        EulerSolver.hxx:466-505: the limited reconstruction into uRecNew (putIntoNew)."""
        self._c.DoLimiterWBAP_C(u, uRec, si, uRecNew, float(smoothThreshold), float(WBAP_nStd), bool(ifAll))

    # positivity-preserving increment limiting (EulerSolver.hxx:696-738)
    def EvaluateCellRHSAlpha(self, u, res, alpha, refRho, refP, relax=0.9, compress=2, compressPower=1.0, ppEpsIsRelaxed=False, flag=0):
        """EulerEvaluator.hxx:1938-2062: alpha [nCell] (written in place) so that u + alpha res keeps the
        relaxed density and pressure floors; returns (nLim, alphaMin).  refRho, refP: far-field density
        and pressure (refUPrim); flag 1 = MIN_IF_NOT_ONE, 2 = MIN_ALL."""
        n, amin = self._c.EvaluateCellRHSAlpha(u, res, alpha, float(refRho), float(refP), float(relax), int(compress), float(compressPower),
                                               bool(ppEpsIsRelaxed), int(flag))
        return int(n), float(amin)

    def EvaluateCellRHSAlphaExpansion(self, u, res, alpha, refRho, refP, alphaMin):
        """EulerEvaluator.hxx:2064-2140: alpha = alphaMin where u + res leaves the floors."""
        self._c.EvaluateCellRHSAlphaExpansion(u, res, alpha, float(refRho), float(refP), float(alphaMin))

    def AddFixedIncrement(self, u, inc, alpha, refRho, refP, ppEpsIsRelaxed=False):
        """EulerEvaluator.hpp:1795-1857: u += CompressInc(u, alpha inc) in place; returns the smallest
        density-increment ratio the compression applied."""
        return float(self._c.AddFixedIncrement(u, inc, float(alpha), float(refRho), float(refP), bool(ppEpsIsRelaxed)))

    def PressureForceCoords(self, zone, direction, u, uRec):
        """Derivative of PressureForce with respect to the node coordinates [nNode][3] (u, uRec held fixed)."""
        dX = torch.empty((self.vr.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        self._c.PressureForceCoords(int(zone), np.ascontiguousarray(direction, dtype=np.float64), u, uRec, dX)
        return dX

    def SolveLinear(self, alphaDiag, dTau, dt, u, rhs, xInc, gmresCode=0, jacobiCode=1, sgsIter=0, nGmresSpace=5, nGmresIter=1,
                    precision="fp64", meanScale=None, useGraph=True):
        """EulerSolver::solveLinear with LUSGSMatrixInit (EulerSolver.hxx:1407-1579, EulerEvaluator.hxx:37-159):
        xInc = M^-1 rhs by LU-SGS pairs (gmresCode 0), GMRES preconditioned by SGS pairs (1), or both (2),
        in FP64 or FP32; all on the device, no host synchronisation."""
        ls = dict(gmresCode=int(gmresCode), jacobiCode=int(jacobiCode), sgsIter=int(sgsIter), nGmresSpace=int(nGmresSpace),
                  nGmresIter=int(nGmresIter), precision=1 if precision == "fp32" else 0, useGraph=int(bool(useGraph)),
                  meanScale=[float(x) for x in (meanScale if meanScale is not None else [])])
        self._c.SolveLinear(ls, float(alphaDiag), dTau, float(dt), u, rhs, xInc)

    def EvaluateNorm(self, x, P=1, volWise=True):
        return self._c.EvaluateNorm(x, int(P), bool(volWise))

    def get(self, name):
        return self._c.get(name)

    def SetDeltaLambda(self, dl):
        self._c.SetDeltaLambda(dl)
