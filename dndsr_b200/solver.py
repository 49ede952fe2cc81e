"""Python mirror of the reference's VR / Euler evaluator call surface on torch CUDA tensors.

Class and method names follow CFV::VariationalReconstruction
(src/CFV/VariationalReconstruction.hpp:108-1114, bound in
src/CFV/VariationalReconstruction_bind.hpp:19-145) and
Euler::EulerEvaluator (src/Euler/EulerEvaluator.hpp:76-1980).  State arrays
are caller-owned contiguous float64 CUDA tensors; every call goes through the
C-ABI of include/dndsb.h on torch's current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import capi
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
                      TRef=273.15, CSutherland=110.4, muModel=1, ignoreVis=False, rsMeanValueEig=0)


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


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor, nm="tensor", fp32=False):
    dt = torch.float32 if fp32 else torch.float64
    if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
        raise ValueError(f"{nm} must be a contiguous {'float32' if fp32 else 'float64'} CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


class Handle:
    _destroy = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h and self._destroy:
            try:
                capi.load(require_device=False)
                getattr(capi._lib, self._destroy)(h)
            except Exception:
                pass
            self.h = None


class DeviceMesh(Handle):
    """Uploads a :class:`dndsr_b200.mesh.Mesh` (replaces Geom::UnstructuredMesh as the VR input)."""
    _destroy = "dndsb_mesh_destroy"

    def __init__(self, mesh: Mesh):
        capi.load()
        self.mesh = mesh
        a = mesh.arrays()
        self._keep = a
        h = ctypes.c_void_p()
        D = capi.dptr
        I64 = lambda x: x.ctypes.data_as(capi._I64)
        capi.call("dndsb_mesh_create", ctypes.byref(h), mesh.dim, mesh.cell_type, mesh.face_type, mesh.n_node, D(a["coords"]), mesh.n_cell,
                  a["cell2node"].shape[1], I64(a["cell2node"]), D(a["cell_shift"]), mesh.n_face, a["face2node"].shape[1],
                  I64(a["face2node"]), D(a["face_shift"]), I64(a["face2cell"]), a["face_zone"].ctypes.data_as(capi._I32), D(a["face_pshift"]),
                  a["cell2face"].shape[1], I64(a["cell2face"]))
        self.h = h

    def colors(self):
        n = ctypes.c_int()
        col = np.zeros(self.mesh.n_cell, dtype=np.int32)
        capi.call("dndsb_mesh_colors", self.h, ctypes.byref(n), col.ctypes.data_as(capi._I32))
        return n.value, col


class VariationalReconstruction(Handle):
    """CFV::VariationalReconstruction<dim> on the GPU."""
    _destroy = "dndsb_vr_destroy"

    def __init__(self, mesh, settings: dict | None = None):
        self.dmesh = mesh if isinstance(mesh, DeviceMesh) else DeviceMesh(mesh)
        self.mesh = self.dmesh.mesh
        s = dict(VR_DEFAULTS)
        s.update(settings or {})
        self.settings = s
        cs = capi.VRSettings()
        cs.maxOrder, cs.intOrder, cs.jacobiRelax = int(s["maxOrder"]), int(s["intOrder"]), float(s["jacobiRelax"])
        cs.SORInstead, cs.anisotropicLengths = int(bool(s["SORInstead"])), int(bool(s["anisotropicLengths"]))
        cs.scaleType = _SCALE[s["scaleType"]] if isinstance(s["scaleType"], str) else int(s["scaleType"])
        cs.scaleMultiplier = float(s["scaleMultiplier"])
        cs.dirWeightScheme = _DIRW[s["dirWeightScheme"]] if isinstance(s["dirWeightScheme"], str) else int(s["dirWeightScheme"])
        for i, x in enumerate(s["manualDirWeights"][:4]):
            cs.manualDirWeights[i] = float(x)
        cs.geomWeightScheme = _GEOMW[s["geomWeightScheme"]] if isinstance(s["geomWeightScheme"], str) else int(s["geomWeightScheme"])
        cs.geomWeightBias, cs.geomWeightPower = float(s["geomWeightBias"]), float(s["geomWeightPower"])
        cs.geomWeightPower1, cs.geomWeightPower2, cs.bcWeight = float(s["geomWeightPower1"]), float(s["geomWeightPower2"]), float(s["bcWeight"])
        h = ctypes.c_void_p()
        capi.call("dndsb_vr_create", ctypes.byref(h), self.dmesh.h, ctypes.byref(cs))
        self.h = h
        self._cs = cs

    # VariationalReconstruction.cpp:10-43, :56-498, :507-872
    def ConstructMetrics(self):
        capi.call("dndsb_vr_construct_metrics", self.h)

    def ConstructBaseAndWeight(self, bc_dir_weight=None):
        if bc_dir_weight is None:
            capi.call("dndsb_vr_construct_base_and_weight", self.h, None, 0)
        else:
            w = np.ascontiguousarray(bc_dir_weight, dtype=np.float64).reshape(-1, 4)
            capi.call("dndsb_vr_construct_base_and_weight", self.h, capi.dptr(w), w.shape[0])

    def ConstructRecCoeff(self):
        capi.call("dndsb_vr_construct_rec_coeff", self.h)
        out = np.zeros(4, dtype=np.int64)
        capi.call("dndsb_vr_sizes", self.h, out.ctypes.data_as(capi._I64))
        self.NDOF, self.R, self.nGf, self.nGc = [int(x) for x in out]

    def construct(self, bc_dir_weight=None):
        self.ConstructMetrics()
        self.ConstructBaseAndWeight(bc_dir_weight)
        self.ConstructRecCoeff()
        return self

    def get(self, name):
        n = ctypes.c_int64()
        capi.call("dndsb_vr_get_array", self.h, name.encode(), None, 0, ctypes.byref(n))
        out = np.zeros(n.value)
        capi.call("dndsb_vr_get_array", self.h, name.encode(), capi.dptr(out), n.value, ctypes.byref(n))
        return out

    # VariationalReconstruction.hpp:920-1000 BuildURec / FiniteVolume BuildUDof
    def BuildURec(self, nVars):
        return torch.zeros((self.mesh.n_cell, self.R, nVars), dtype=torch.float64, device="cuda")

    def BuildUDof(self, nVars):
        return torch.zeros((self.mesh.n_cell, nVars), dtype=torch.float64, device="cuda")

    def DoReconstructionIter(self, uRec, uRecNew, u, putIntoNew=False, recordInc=False, uRecIsZero=False, precision="fp64"):
        """VariationalReconstruction_Reconstruction.hxx:485-615 (Jacobi sweep)."""
        nv = u.shape[1]
        capi.call("dndsb_vr_do_reconstruction_iter", self.h, _ptr(uRec, "uRec"), _ptr(uRecNew, "uRecNew"), _ptr(u, "u"), nv,
                  int(putIntoNew), int(recordInc), int(uRecIsZero), 1 if precision == "fp32" else 0, _stream())


    def DoReconstructionIterVJP(self, cot, uRec, u):
        """Vector-Jacobian product of one Jacobi sweep uRecNew = S(uRec, u): returns
        ((dS/duRec)^T cot, (dS/du)^T cot)."""
        vRec, vU = torch.empty_like(uRec), torch.empty_like(u)
        capi.call("dndsb_vr_iter_vjp", self.h, _ptr(cot, "cot"), _ptr(uRec, "uRec"), _ptr(u, "u"), u.shape[1], _ptr(vRec, "vRec"),
                  _ptr(vU, "vU"), _stream())
        return vRec, vU

    def DoReconstructionIterJVP(self, dRec, du, uRec, u):
        """Jacobian-vector product of one Jacobi sweep (DoReconstructionIterDiff with the
        linearised boundary term): dS/duRec dRec + dS/du du."""
        out = torch.empty_like(uRec)
        capi.call("dndsb_vr_iter_jvp", self.h, _ptr(dRec, "dRec"), _ptr(du, "du"), _ptr(uRec, "uRec"), _ptr(u, "u"), u.shape[1],
                  _ptr(out, "dRecNew"), _stream())
        return out

    def DoCalculateSmoothIndicator(self, u, uRec):
        """VariationalReconstruction_LimiterProcedure.hxx:40-108 (procedure 0, density and energy): si [nCell]."""
        si = torch.empty(self.mesh.n_cell, dtype=torch.float64, device="cuda")
        capi.call("dndsb_vr_smooth_indicator", self.h, _ptr(u, "u"), _ptr(uRec, "uRec"), u.shape[1], _ptr(si, "si"), _stream())
        return si

    def DoReconstructionIterVJPCoords(self, cot, uRec, u):
        """(dS/dX)^T cot for one Jacobi sweep uRecNew = S(uRec, u; X), X the node coordinates
        [nNode][3]: the geometry, basis moments, weights and A^-1 B / A^-1 b are differentiated."""
        dX = torch.empty((self.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        capi.call("dndsb_vr_iter_vjp_coords", self.h, _ptr(cot, "cot"), _ptr(uRec, "uRec"), _ptr(u, "u"), u.shape[1], _ptr(dX, "dX"),
                  _stream())
        return dX

    def DoReconstructionIterJVPCoords(self, dX, uRec, u):
        """dS/dX dX for one Jacobi sweep along the node displacement dX [nNode][3]."""
        out = torch.empty_like(uRec)
        capi.call("dndsb_vr_iter_jvp_coords", self.h, _ptr(dX, "dX"), _ptr(uRec, "uRec"), _ptr(u, "u"), u.shape[1], _ptr(out, "dRecNew"),
                  _stream())
        return out


class EulerEvaluator(Handle):
    """Euler::EulerEvaluator<model> on the GPU (models NS / NS_3D with 5 variables)."""
    _destroy = "dndsb_eval_destroy"

    def __init__(self, vr: VariationalReconstruction, settings: dict | None = None):
        self.vr = vr
        s = dict(EULER_DEFAULTS)
        s.update(settings or {})
        self.settings = s
        cs = capi.EulerSettings()
        cs.nVars = int(s["nVars"])
        rs = s["riemannSolverType"]
        cs.rsType = RS[rs] if isinstance(rs, str) else int(rs)
        cs.rsFixScale, cs.rsIncFScale = float(s["rsFixScale"]), float(s["rsIncFScale"])
        cs.gamma, cs.Rgas, cs.muGas, cs.prGas = float(s["gamma"]), float(s["Rgas"]), float(s["muGas"]), float(s["prGas"])
        cs.TRef, cs.CSutherland, cs.muModel, cs.ignoreVis = float(s["TRef"]), float(s["CSutherland"]), int(s["muModel"]), int(bool(s["ignoreVis"]))
        cs.rsMeanValueEig = int(s["rsMeanValueEig"])
        h = ctypes.c_void_p()
        capi.call("dndsb_eval_create", ctypes.byref(h), vr.h, ctypes.byref(cs))
        self.h = h
        self.nVars = cs.nVars
        self._cs = cs

    def SetBC(self, types, values):
        """BoundaryHandler of the evaluator (Euler/EulerBC.hpp) as a per-zone table: types[zone]
        (EulerBC.hpp codes or names, 0 for interior zones) and values[zone] (far-field / inflow
        state, or wall temperature first).  Also the reconstruction's FBoundary."""
        t = np.array([BC[x] if isinstance(x, str) else int(x) for x in types], dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(len(t), self.nVars)
        self._bc = (t, v)
        capi.call("dndsb_eval_set_bc", self.h, len(t), t.ctypes.data_as(capi._I32), capi.dptr(v))

    def SetWallDistance(self, d):
        """dWall of the SA model at every cell Gauss point, [nCell][nGc] host array."""
        d = np.ascontiguousarray(d, dtype=np.float64)
        capi.call("dndsb_eval_set_wall_distance", self.h, capi.dptr(d))

    def InitializeUDOF(self, u, kind, chi=5.0):
        capi.call("dndsb_eval_initialize_udof", self.h, kind, float(chi), _ptr(u, "u"), _stream())

    def EvaluateDt(self, dt, u, CFL, MaxDt=1e100, UseLocaldt=True, want_min=True):
        """Returns the global minimum of dt (want_min=False with UseLocaldt: no host synchronisation, None)."""
        mn = ctypes.c_double()
        ask = want_min or not UseLocaldt
        capi.call("dndsb_eval_evaluate_dt", self.h, _ptr(u, "u"), float(CFL), float(MaxDt), int(UseLocaldt), _ptr(dt, "dt"),
                  ctypes.byref(mn) if ask else None, _stream())
        return mn.value if ask else None

    # EvaluateRHS flags, EulerEvaluator.hpp:370-378
    RHS_No_Flags, RHS_Ignore_Viscosity, RHS_Dont_Update_Integration, RHS_Dont_Record_Bud_Flux = 0, 1, 2, 4

    def EvaluateRHS(self, rhs, u, uRec, JSource=None, uRecUnlim=None, uRecBeta=None, cellRHSAlpha=None, onlyOnHalfAlpha=False, t=0.0,
                    flags=0):
        """EvaluateRHS (EulerEvaluator_EvaluateRHS.hxx:55-818).  The short form (rhs, u, uRec) evaluates with
        the reconstruction uRec for values and gradients.  The keyword form is the reference's full
        contract: uRecUnlim gives the gradients (uRec the limited point values), cellRHSAlpha scales the
        SA source, JSource [nCell][nVars] receives the source Jacobian diagonal, flags are RHS_* bits;
        uRecBeta, onlyOnHalfAlpha and t are accepted and not read, as in the reference's body."""
        if JSource is None and uRecUnlim is None and cellRHSAlpha is None and flags == 0:
            capi.call("dndsb_eval_evaluate_rhs", self.h, _ptr(rhs, "rhs"), _ptr(u, "u"), _ptr(uRec, "uRec"), _stream())
            return
        capi.call("dndsb_eval_evaluate_rhs_full", self.h, _ptr(rhs, "rhs"), _ptr(JSource, "JSource") if JSource is not None else None,
                  _ptr(u, "u"), _ptr(uRecUnlim if uRecUnlim is not None else uRec, "uRecUnlim"), _ptr(uRec, "uRec"),
                  _ptr(uRecBeta, "uRecBeta") if uRecBeta is not None else None,
                  _ptr(cellRHSAlpha, "cellRHSAlpha") if cellRHSAlpha is not None else None, int(bool(onlyOnHalfAlpha)), float(t),
                  int(flags), _stream())

    def SetDeferredErrors(self, deferred=True):
        """EvaluateRHS stops reading its error word back on every call; CheckErrors reads it."""
        capi.call("dndsb_eval_set_deferred_errors", self.h, int(bool(deferred)))

    def CheckErrors(self):
        """Reads and clears the deferred error word of EvaluateRHS (raises DndsbError on a non-physical or
        non-finite state seen since the last check)."""
        capi.call("dndsb_eval_check_errors", self.h, _stream())

    def EvaluateRHSNoAlloc(self, rhs, u, uRec):
        """EvaluateRHS without any device allocation: the face-flux scratch is a
        static 8 MiB device array (nFace * nVars <= capi.NOALLOC_SCRATCH_DOUBLES).
        For callers that cannot allocate device memory when they evaluate a
        residual; calls that overlap on the same GPU share the array and race."""
        capi.call("dndsb_eval_evaluate_rhs_noalloc", self.h, _ptr(rhs, "rhs"), _ptr(u, "u"), _ptr(uRec, "uRec"), _stream())

    def EvaluateRHSVJP(self, w, u, uRec):
        """(dR/du)^T w and (dR/duRec)^T w of EvaluateRHS at (u, uRec), deltaLambdaCell held fixed."""
        du, duRec = torch.empty_like(u), torch.empty_like(uRec)
        capi.call("dndsb_eval_rhs_vjp", self.h, _ptr(w, "w"), _ptr(u, "u"), _ptr(uRec, "uRec"), _ptr(du, "du"), _ptr(duRec, "duRec"),
                  _stream())
        return du, duRec

    def EvaluateRHSJVP(self, du, duRec, u, uRec):
        """dR/du du + dR/duRec duRec of EvaluateRHS at (u, uRec), deltaLambdaCell held fixed."""
        out = torch.empty_like(u)
        capi.call("dndsb_eval_rhs_jvp", self.h, _ptr(du, "du"), _ptr(duRec, "duRec"), _ptr(u, "u"), _ptr(uRec, "uRec"), _ptr(out, "dRhs"),
                  _stream())
        return out

    def EvaluateRHSVJPCoords(self, w, u, uRec):
        """(dR/dX)^T w of EvaluateRHS with respect to the node coordinates X [nNode][3] (u, uRec
        and deltaLambdaCell held fixed)."""
        dX = torch.empty((self.vr.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        capi.call("dndsb_eval_rhs_vjp_coords", self.h, _ptr(w, "w"), _ptr(u, "u"), _ptr(uRec, "uRec"), _ptr(dX, "dX"), _stream())
        return dX

    def ResidualVJPCoords(self, w, cot, u, uRec):
        """(dR/dX)^T w + (dS/dX)^T cot in one pass (S: one VR sweep of this evaluator's reconstruction)."""
        dX = torch.empty((self.vr.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        capi.call("dndsb_eval_residual_vjp_coords", self.h, _ptr(w, "w"), _ptr(cot, "cot"), _ptr(u, "u"), _ptr(uRec, "uRec"), _ptr(dX, "dX"),
                  _stream())
        return dX

    def EvaluateRHSJVPCoords(self, dX, u, uRec):
        """dR/dX dX of EvaluateRHS along the node displacement dX [nNode][3]."""
        out = torch.empty_like(u)
        capi.call("dndsb_eval_rhs_jvp_coords", self.h, _ptr(dX, "dX"), _ptr(u, "u"), _ptr(uRec, "uRec"), _ptr(out, "dRhs"), _stream())
        return out

    def BuildJDiag(self):
        """Diagonal array of LUSGSMatrixInit: [nCell] (one value per cell), or [nCell][nVars] for the SA model."""
        n = self.vr.mesh.n_cell
        return torch.zeros((n, self.nVars) if self.nVars == 6 else (n,), dtype=torch.float64, device="cuda")

    def LUSGSMatrixInit(self, jdiag, dTau, dt, alphaDiag):
        capi.call("dndsb_eval_lusgs_matrix_init", self.h, _ptr(dTau, "dTau"), float(dt), float(alphaDiag), _ptr(jdiag, "jdiag"), _stream())

    def UpdateSGS(self, alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward, gsUpdate=True, uIncIsZero=False, want_sum=True):
        s = np.zeros(self.nVars)
        capi.call("dndsb_eval_update_sgs", self.h, float(alphaDiag), _ptr(rhs, "rhs"), _ptr(u, "u"), _ptr(uInc, "uInc"),
                  _ptr(uIncNew, "uIncNew"), _ptr(jdiag, "jdiag"), int(forward), int(gsUpdate), int(uIncIsZero),
                  capi.dptr(s) if want_sum else None, _stream())
        return s

    def UpdateLUSGSForward(self, alphaDiag, rhs, u, uInc, jdiag, uIncNew):
        """EulerEvaluator.hxx:376-451: uIncNew = D^-1 (rhs - lower-neighbour flux increments of uInc).
        uInc may be uIncNew itself (the in-place sweep of the reference's callers)."""
        capi.call("dndsb_eval_update_lusgs_forward", self.h, float(alphaDiag), _ptr(rhs, "rhs"), _ptr(u, "u"), _ptr(uInc, "uInc"),
                  _ptr(jdiag, "jdiag"), _ptr(uIncNew, "uIncNew"), _stream())

    def UpdateLUSGSBackward(self, alphaDiag, rhs, u, uInc, jdiag, uIncNew):
        """EulerEvaluator.hxx:453-529: uIncNew += D^-1 (- upper-neighbour flux increments of uInc)."""
        capi.call("dndsb_eval_update_lusgs_backward", self.h, float(alphaDiag), _ptr(rhs, "rhs"), _ptr(u, "u"), _ptr(uInc, "uInc"),
                  _ptr(jdiag, "jdiag"), _ptr(uIncNew, "uIncNew"), _stream())

    def FixUMaxFilter(self, u):
        """EulerEvaluator.hxx:1318-1323: the reference's filter returns without changing u."""
        capi.call("dndsb_eval_fix_umax_filter", self.h, _ptr(u, "u"), _stream())

    def LUSGSMatrixVec(self, alphaDiag, u, uInc, jdiag, AuInc):
        capi.call("dndsb_eval_lusgs_matrix_vec", self.h, float(alphaDiag), _ptr(u, "u"), _ptr(uInc, "uInc"), _ptr(jdiag, "jdiag"),
                  _ptr(AuInc, "AuInc"), _stream())

    def LUSGSMatrixVecT(self, alphaDiag, u, y, jdiag, ATy):
        """ATy = A^T y for the operator A of LUSGSMatrixVec (same lambdaFace, jdiag, alphaDiag)."""
        capi.call("dndsb_eval_lusgs_matrix_vec_t", self.h, float(alphaDiag), _ptr(u, "u"), _ptr(y, "y"), _ptr(jdiag, "jdiag"),
                  _ptr(ATy, "ATy"), _stream())

    def UpdateSGST(self, alphaDiag, b, u, y, yNew, jdiag, forward, gsUpdate=True):
        """One Gauss-Seidel sweep on A^T y = b (the transpose of UpdateSGS), colour by colour; b, y and
        yNew are all float64 or all float32 (the FP32 preconditioner)."""
        fp32 = b.dtype == torch.float32
        if any((t.dtype == torch.float32) != fp32 for t in (y, yNew)):
            raise TypeError("UpdateSGST: b, y and yNew must share one precision")
        capi.call("dndsb_eval_update_sgs_t", self.h, float(alphaDiag), _ptr(b, "b", fp32), _ptr(u, "u"), _ptr(y, "y", fp32),
                  _ptr(yNew, "yNew", fp32), _ptr(jdiag, "jdiag"), int(forward), int(gsUpdate), int(fp32), _stream())

    def PressureForce(self, zone, direction, u, uRec, grad=False):
        """Pressure force along direction on boundary zone; with grad also (dJ/du, dJ/duRec) as device tensors."""
        d = np.ascontiguousarray(direction, dtype=np.float64)
        J = np.zeros(1)
        gU = torch.empty_like(u) if grad else None
        gR = torch.empty_like(uRec) if grad else None
        capi.call("dndsb_eval_pressure_force", self.h, int(zone), capi.dptr(d), _ptr(u, "u"), _ptr(uRec, "uRec"), capi.dptr(J),
                  _ptr(gU, "dJdu") if grad else None, _ptr(gR, "dJduRec") if grad else None, _stream())
        return (float(J[0]), gU, gR) if grad else float(J[0])

    def DoLimiterWBAP_C(self, u, uRec, si, uRecNew, smoothThreshold=0.01, WBAP_nStd=10.0, ifAll=False):
        """VariationalReconstruction_LimiterProcedure.hxx:188-334 with the characteristic projections of
        EulerSolver.hxx:466-505: the limited reconstruction into uRecNew (putIntoNew)."""
        capi.call("dndsb_eval_limiter_wbap_c", self.h, _ptr(u, "u"), _ptr(uRec, "uRec"), _ptr(si, "si"), _ptr(uRecNew, "uRecNew"),
                  float(smoothThreshold), float(WBAP_nStd), int(bool(ifAll)), _stream())

    # positivity-preserving increment limiting (EulerSolver.hxx:696-738)
    def EvaluateCellRHSAlpha(self, u, res, alpha, refRho, refP, relax=0.9, compress=2, compressPower=1.0, ppEpsIsRelaxed=False, flag=0):
        """EulerEvaluator.hxx:1938-2062: alpha [nCell] (written in place) so that u + alpha res keeps the
        relaxed density and pressure floors; returns (nLim, alphaMin).  refRho, refP: far-field density
        and pressure (refUPrim); flag 1 = MIN_IF_NOT_ONE, 2 = MIN_ALL."""
        n, amin = ctypes.c_int64(), ctypes.c_double()
        capi.call("dndsb_eval_cell_rhs_alpha", self.h, _ptr(u, "u"), _ptr(res, "res"), _ptr(alpha, "alpha"), float(refRho), float(refP),
                  float(relax), int(compress), float(compressPower), int(bool(ppEpsIsRelaxed)), int(flag), ctypes.addressof(n),
                  ctypes.addressof(amin), _stream())
        return int(n.value), float(amin.value)

    def EvaluateCellRHSAlphaExpansion(self, u, res, alpha, refRho, refP, alphaMin):
        """EulerEvaluator.hxx:2064-2140: alpha = alphaMin where u + res leaves the floors."""
        capi.call("dndsb_eval_cell_rhs_alpha_expansion", self.h, _ptr(u, "u"), _ptr(res, "res"), _ptr(alpha, "alpha"), float(refRho),
                  float(refP), float(alphaMin), _stream())

    def AddFixedIncrement(self, u, inc, alpha, refRho, refP, ppEpsIsRelaxed=False):
        """EulerEvaluator.hpp:1795-1857: u += CompressInc(u, alpha inc) in place; returns the smallest
        density-increment ratio the compression applied."""
        amin = ctypes.c_double()
        capi.call("dndsb_eval_add_fixed_increment", self.h, _ptr(u, "u"), _ptr(inc, "inc"), float(alpha), float(refRho), float(refP),
                  int(bool(ppEpsIsRelaxed)), ctypes.addressof(amin), _stream())
        return float(amin.value)

    def PressureForceCoords(self, zone, direction, u, uRec):
        """Derivative of PressureForce with respect to the node coordinates [nNode][3] (u, uRec held fixed)."""
        d = np.ascontiguousarray(direction, dtype=np.float64)
        dX = torch.empty((self.vr.mesh.n_node, 3), dtype=torch.float64, device="cuda")
        capi.call("dndsb_eval_pressure_force_coords", self.h, int(zone), capi.dptr(d), _ptr(u, "u"), _ptr(uRec, "uRec"), _ptr(dX, "dJdX"),
                  _stream())
        return dX

    def SolveLinear(self, alphaDiag, dTau, dt, u, rhs, xInc, gmresCode=0, jacobiCode=1, sgsIter=0, nGmresSpace=5, nGmresIter=1,
                    precision="fp64", meanScale=None, useGraph=True):
        """EulerSolver::solveLinear with LUSGSMatrixInit (EulerSolver.hxx:1407-1579, EulerEvaluator.hxx:37-159):
        xInc = M^-1 rhs by LU-SGS pairs (gmresCode 0), GMRES preconditioned by SGS pairs (1), or both (2),
        in FP64 or FP32; all on the device, no host synchronisation."""
        ls = capi.LinearSettings()
        ls.gmresCode, ls.jacobiCode, ls.sgsIter = int(gmresCode), int(jacobiCode), int(sgsIter)
        ls.nGmresSpace, ls.nGmresIter = int(nGmresSpace), int(nGmresIter)
        ls.precision = 1 if precision == "fp32" else 0
        ls.useGraph = int(bool(useGraph))
        for i, x in enumerate(meanScale if meanScale is not None else []):
            ls.meanScale[i] = float(x)
        capi.call("dndsb_eval_solve_linear", self.h, ctypes.byref(ls), float(alphaDiag), _ptr(dTau, "dTau"), float(dt), _ptr(u, "u"),
                  _ptr(rhs, "rhs"), _ptr(xInc, "xInc"), _stream())

    def EvaluateNorm(self, x, P=1, volWise=True):
        out = np.zeros(self.nVars)
        capi.call("dndsb_eval_evaluate_norm", self.h, _ptr(x, "x"), int(P), int(volWise), capi.dptr(out), _stream())
        return out

    def get(self, name):
        n = ctypes.c_int64()
        capi.call("dndsb_eval_get_array", self.h, name.encode(), None, 0, ctypes.byref(n))
        out = np.zeros(n.value)
        capi.call("dndsb_eval_get_array", self.h, name.encode(), capi.dptr(out), n.value, ctypes.byref(n))
        return out

    def SetDeltaLambda(self, dl):
        capi.call("dndsb_eval_set_delta_lambda", self.h, _ptr(dl, "deltaLambdaCell"), _stream())
