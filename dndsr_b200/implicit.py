"""Implicit time marching on top of the GPU operators.

Restates the reference's dual-time machinery:

* ``ESDIRK``  -- Solver/ODE.hpp:122-360 ImplicitSDIRK4DualTimeStep (scheme 1 =
  6-stage ESDIRK4 with explicit first stage, scheme 0 = 3-stage SDIRK4);
* ``BDF1``    -- the backward-Euler member of ImplicitVBDFDualTimeStep
  (ODE.hpp:601-915), used for steady runs;
* ``GMRES``   -- Solver/Linear.hpp:11-133 GMRES_LeftPreconditioned (restarted,
  classical Gram-Schmidt, least-squares Hessenberg solve);
* ``ImplicitSolver`` -- the frhs / fdtau / fsolve / fincrement closures of
  Euler/EulerSolver.hxx:147-997 with solveLinear / doPrecondition
  (:1407-1658): LU-SGS (gmresCode 0) or GMRES preconditioned by SGS sweeps
  (gmresCode 1), optionally in FP32 inside the FP64 defect correction.

Vectors are torch CUDA tensors; every spatial operator is a call into the
CUDA library (include/dndsb.h).  Host code only orchestrates and does the
small dense least-squares solve of GMRES.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

VERY_SMALL = 1e-200


class ESDIRK:
    """ODE.hpp:122-360.  scheme 1: ESDIRK4 (odeCode 0 of the solver), scheme 0: SDIRK4."""

    def __init__(self, scheme=1):
        if scheme == 0:
            z = 0.128886400515
            self.A = np.array([[z, 0, 0], [0.5 - z, z, 0], [2 * z, 1 - 4 * z, z]])
            self.c = np.array([z, 0.5, 1 - z])
            self.b = np.array([1 / (6 * (2 * z - 1) ** 2), (4 * z * z - 4 * z + 2 / 3) / (2 * z - 1) ** 2, 1 / (6 * (2 * z - 1) ** 2)])
            self.explicit_first = False
        else:
            self.A = np.array([
                [VERY_SMALL, 0, 0, 0, 0, 0],
                [0.25, 0.25, 0, 0, 0, 0],
                [0.137776, -0.055776, 0.25, 0, 0, 0],
                [0.1446368660269822, -0.2239319076133447, 0.4492950415863626, 0.25, 0, 0],
                [0.09825878328356477, -0.5915442428196704, 0.8101210205756877, 0.283164405707806, 0.25, 0],
                [0.1579162951616714, 0, 0.1867589405240008, 0.6805652953093346, -0.2752405309950067, 0.25]])
            self.b = self.A[-1].copy()
            self.c = np.array([0, 0.5, 0.332, 0.62, 0.849999966747388, 1])
            self.explicit_first = True
        self.n = len(self.c)
        self.rhsbuf = None
        self.has_last_end_rhs = False

    def step(self, x, frhs, fdt, fsolve, max_iter, fstop, fincrement, dt):
        """One physical step; x is updated in place (ODE.hpp:271-343)."""
        if self.rhsbuf is None:
            self.rhsbuf = [torch.zeros_like(x) for _ in range(self.n)]
        x_last = x.clone()
        dtau = torch.zeros(x.shape[0], dtype=x.dtype, device=x.device)
        xinc = torch.zeros_like(x)
        for iB in range(self.n):
            x.copy_(x_last)
            it = 1
            while it <= max_iter:
                if self.explicit_first and iB == 0:
                    if self.has_last_end_rhs:
                        self.rhsbuf[0].copy_(self.rhsbuf[self.n - 1])
                    else:
                        frhs(self.rhsbuf[0], x, dtau, 1 << 30, self.c[0])
                    break
                fdt(x, dtau, self.A[iB, iB])
                frhs(self.rhsbuf[iB], x, dtau, it, self.c[iB])
                rhs = x_last * (1.0 / dt)
                for jB in range(iB):
                    rhs.add_(self.rhsbuf[jB], alpha=self.A[iB, jB])
                res_other = rhs.clone()
                rhs.add_(x, alpha=-1.0 / dt)
                rhs.add_(self.rhsbuf[iB], alpha=self.A[iB, iB])
                fsolve(x, rhs, res_other, dtau, dt, self.A[iB, iB], xinc, it, self.c[iB])
                fincrement(x, xinc, 1.0)
                if fstop(it, rhs, iB + 1):
                    break
                it += 1
            if it > max_iter:
                fstop(it, rhs, iB + 1)
        if self.explicit_first:
            self.has_last_end_rhs = True
            return
        x.copy_(x_last)
        for jB in range(self.n):
            x.add_(self.rhsbuf[jB], alpha=self.b[jB] * dt)


class BDF1Stepper:
    """Backward Euler in dual time (the k = 1 member of ODE.hpp:601-915): residual = (x_n - x)/dt + rhs(x)."""

    def __init__(self):
        self.rhs = None

    def step(self, x, frhs, fdt, fsolve, max_iter, fstop, fincrement, dt):
        if self.rhs is None:
            self.rhs = torch.zeros_like(x)
        x_last = x.clone()
        dtau = torch.zeros(x.shape[0], dtype=x.dtype, device=x.device)
        xinc = torch.zeros_like(x)
        for it in range(1, max_iter + 1):
            fdt(x, dtau, 1.0)
            frhs(self.rhs, x, dtau, it, 1.0)
            res = x_last * (1.0 / dt)
            res_other = res.clone()
            res.add_(x, alpha=-1.0 / dt)
            res.add_(self.rhs)
            fsolve(x, res, res_other, dtau, dt, 1.0, xinc, it, 1.0)
            fincrement(x, xinc, 1.0)
            if fstop(it, res, 1):
                return it
        return max_iter


def _lstsq(h, e):
    """Least-squares solve with rank report (HardEigen::EigenLeastSquareSolve semantics)."""
    y, _, rank, _ = np.linalg.lstsq(h, e, rcond=None)
    return y, rank


class GMRES:
    """Linear.hpp:11-133 GMRES_LeftPreconditioned on torch vectors."""

    def __init__(self, k_subspace, like):
        self.k = k_subspace
        self.V = [torch.zeros_like(like) for _ in range(k_subspace + 1)]
        self.tmp = torch.zeros_like(like)
        self.MLb = torch.zeros_like(like)

    def solve(self, FA, FML, fdot, b, x, n_restart, fstop):
        FML(b, self.MLb)
        scale = math.sqrt(fdot(self.MLb, self.MLb))
        h = np.zeros((self.k + 1, self.k))
        i_restart = 0
        for i_restart in range(n_restart + 1):
            FA(x, self.tmp)
            FML(self.tmp, self.V[0])
            self.V[0].add_(self.MLb, alpha=-1.0)
            beta = math.sqrt(fdot(self.V[0], self.V[0]))
            if fstop(i_restart, beta, scale):
                break
            if abs(beta) < VERY_SMALL or i_restart == n_restart:
                break
            self.V[0].mul_(-1.0 / beta)
            j = 0
            while j < self.k:
                FA(self.V[j], self.tmp)
                FML(self.tmp, self.V[j + 1])
                for i in range(j + 1):
                    h[i, j] = fdot(self.V[j + 1], self.V[i])
                for i in range(j + 1):
                    self.V[j + 1].add_(self.V[i], alpha=-h[i, j])
                h[j + 1, j] = math.sqrt(fdot(self.V[j + 1], self.V[j + 1]))
                if h[j + 1, j] < scale * 1e-32:
                    break
                self.V[j + 1].mul_(1.0 / h[j + 1, j])
                j += 1
            if j < 1:
                break
            e = np.zeros(j + 1)
            e[0] = beta
            y, rank = _lstsq(h[:j + 1, :j], e)
            for jj in range(j):
                x.add_(self.V[jj], alpha=float(y[jj]))
            if rank < h.shape[1]:
                break
        return i_restart < n_restart


@dataclass
class SolverConfig:
    """Field names follow EulerSolver.hpp (timeMarchControl, convergenceControl, linearSolverControl ...)."""
    odeCode: int = 0                 # 0 ESDIRK4, 101 SDIRK4, 103 backward Euler (steady)
    dtImplicit: float = 0.01
    nTimeStep: int = 100
    nTimeStepInternal: int = 20
    nTimeStepInternalMin: int = 5
    rhsThresholdInternal: float = 1e-10
    normOrd: int = 1
    useVolWiseResidual: bool = False
    CFL: float = 100.0
    useLocalDt: bool = True
    nCFLRampStart: int = 2 ** 31 - 1
    nCFLRampLength: int = 2 ** 31 - 1
    CFLRampEnd: float = 0.0
    nInternalRecStep: int = 1
    # implicitReconstructionControl (EulerSolver.hpp): recLinearScheme 0 = Jacobi sweeps, 1 = GMRES on the
    # linearised reconstruction (EulerSolver.hxx:270-339) with nGmresSpaceRec / nGmresIterRec, stopped at
    # recThreshold times the first sweep's residual; gmresRecScale 1 weighs the dot by the far-field state
    recLinearScheme: int = 0
    nGmresSpaceRec: int = 5
    nGmresIterRec: int = 1
    recThreshold: float = 1e-10
    gmresRecScale: int = 0
    jacobiCode: int = 1              # 1: Gauss-Seidel sweeps, 0: Jacobi, 2: the local LU (block ILU(0))
    sgsIter: int = 0
    gmresCode: int = 0               # 0: LU-SGS only, 1: GMRES preconditioned by SGS
    nGmresSpace: int = 30
    nGmresIter: int = 1
    gmresScale: int = 0
    linear_precision: str = "fp64"   # "fp32": FP32 preconditioner / GMRES inside the FP64 defect correction
    vr_precision: str = "fp64"       # coefficient precision of the VR sweeps
    # with vr_precision "fp32": the sweeps use FP32 coefficients only while the stage's relative residual is
    # above vrFP64Below and FP64 ones from then on, so that the stage converges to the FP64 fixed point
    # (0: FP32 throughout, whose fixed point differs by ~1e-7 relative)
    vrFP64Below: float = 0.0
    native_linear: bool = True       # one device call per linear solve (dndsb_eval_solve_linear) when the evaluator has it
    meanScale: tuple = ()            # GMRES dot weights (gmresScale), empty = ones
    # positivity-preserving increments (timeMarchControl.incrementPPRelax, uRecAlphaCompressPower,
    # ppEpsIsRelaxed); the floors scale with the far-field state, empty = plain u += alpha inc
    # limiterControl (EulerSolver.hxx:455-580, EulerSolver.hpp:670 useViscousLimited): WBAP_C after the VR
    # sweeps, the RHS with point values from the limited reconstruction and gradients from the limited
    # (useViscousLimited) or unlimited one
    useLimiter: bool = False
    useViscousLimited: bool = True
    smoothThreshold: float = 0.01
    WBAP_nStd: float = 10.0
    preserveLimited: bool = False
    farFieldStaticValue: tuple = ()
    incrementPPRelax: float = 0.9
    uRecAlphaCompressPower: float = 1.0
    ppEpsIsRelaxed: bool = False
    res_history: list = field(default_factory=list)


class ImplicitSolver:
    """The frhs / fdtau / fsolve / fincrement closures of EulerSolver::RunImplicitEuler."""

    def __init__(self, vr, ev, cfg: SolverConfig):
        self.vr, self.ev, self.cfg = vr, ev, cfg
        nc = vr.mesh.n_cell
        nv = ev.nVars
        self.uRec = vr.BuildURec(nv)
        self.uRecNew = vr.BuildURec(nv)
        dev = self.uRec.device
        # the evaluator's JDiag layout (scalar, per-variable for SA, or blocks with useScalarJacobian false)
        self.jd = ev.BuildJDiag() if hasattr(ev, "BuildJDiag") else torch.zeros((nc, nv) if nv == 6 else (nc,), dtype=torch.float64,
                                                                               device=dev)
        self.tmp = torch.zeros((nc, nv), dtype=torch.float64, device=dev)
        self.gmres = GMRES(cfg.nGmresSpace, self.tmp) if cfg.gmresCode else None
        self.resBase = None
        self.CFLNow = cfg.CFL
        self.n_rhs = 0
        self.vrPrec = cfg.vr_precision  # the sweeps' coefficient precision of the next pseudo-iteration
        self.n_sgs = 0
        self.gmresRec = None
        self.uRecLim = None
        if cfg.useLimiter:
            self.uRecLim = vr.BuildURec(nv)
        # EvaluateRHS reports non-physical states once per pseudo-iteration (fstop reads the residual
        # norm there anyway) instead of synchronising on every call
        self.deferred = hasattr(ev, "SetDeferredErrors")
        if self.deferred:
            ev.SetDeferredErrors(True)
        self.pp = None
        if cfg.farFieldStaticValue:
            far = [float(x) for x in cfg.farFieldStaticValue]
            self.farU = far
            gamma = float(ev.settings["gamma"])
            rho = far[0]
            self.pp = (rho, (gamma - 1) * (far[4] - 0.5 * (far[1] ** 2 + far[2] ** 2 + far[3] ** 2) / rho))
            self.alphaPP = torch.ones(nc, dtype=torch.float64, device=dev)
            self.incPP = torch.zeros((nc, nv), dtype=torch.float64, device=dev)
            self.nLimInc, self.alphaMinInc = 0, 1.0

    # EulerSolver.hxx:270-339, recLinearScheme 1: each of nInternalRecStep passes takes the sweep's residual
    # r = uRec - S(uRec) (DoReconstructionIter with recordInc), solves (I - dS/duRec) d = r by GMRES with the
    # linearised sweep (DoReconstructionIterDiff: the JVP of the sweep, boundary term included) and no
    # preconditioner, and sets uRec -= d; the passes stop once GMRES reaches recThreshold times the first residual
    def _rec_gmres(self, cx):
        cfg = self.cfg
        if self.gmresRec is None:
            self.gmresRec = GMRES(cfg.nGmresSpaceRec, self.uRec)
            self.recZeroU = torch.zeros_like(cx)
        nv = cx.shape[1]
        if cfg.gmresRecScale == 1 and self.pp is not None:
            far = self.farU
            ms = [far[0]] + [math.sqrt(far[0] * far[4])] * 3 + [far[4]] + [1.0] * (nv - 5)
        else:
            ms = [1.0] * nv
        s2 = torch.tensor([1.0 / (m + 1e-200) ** 2 for m in ms[:nv]], dtype=cx.dtype, device=cx.device)

        def fdot(a, b):
            return float(torch.sum(a * b * s2))

        def FA(x, Ax):
            Ax.copy_(x - self.vr.DoReconstructionIterJVP(x, self.recZeroU, self.uRec, cx))

        def FML(x, MLx):
            MLx.copy_(x)

        resB = None
        for _ in range(cfg.nInternalRecStep):
            self.vr.DoReconstructionIter(self.uRec, self.uRecNew, cx, putIntoNew=True, recordInc=True)
            d = self.uRecNew.clone()
            if resB is None:
                resB = float(d.norm())  # uRecNew1.norm2() of the first pass
            conv = self.gmresRec.solve(FA, FML, fdot, self.uRecNew, d, cfg.nGmresIterRec,
                                       lambda i, res, rb: res < resB * cfg.recThreshold)
            self.uRec.sub_(d)
            if conv:
                break

    # EulerSolver.hxx:147-672 (VR sweeps then EvaluateRHS)
    def frhs(self, crhs, cx, dtau, it, ct):
        if self.cfg.recLinearScheme == 1:
            self._rec_gmres(cx)
        for _ in range(self.cfg.nInternalRecStep if self.cfg.recLinearScheme == 0 else 0):
            self.vr.DoReconstructionIter(self.uRec, self.uRecNew, cx, putIntoNew=False, precision=self.vrPrec)
        if self.uRecLim is not None:
            si = self.vr.DoCalculateSmoothIndicator(cx, self.uRec)
            self.ev.DoLimiterWBAP_C(cx, self.uRec, si, self.uRecLim, self.cfg.smoothThreshold, self.cfg.WBAP_nStd, False)
            if self.cfg.preserveLimited:
                self.uRec.copy_(self.uRecLim)
            # EvaluateRHS(rhs, JSource, u, uRecUnlim, uRec, ...) with uRecUnlim = the limited reconstruction
            # (useViscousLimited, the default) or the unlimited one (EulerSolver.hxx:624-626)
            self.ev.EvaluateRHS(crhs, cx, self.uRecLim, uRecUnlim=self.uRecLim if self.cfg.useViscousLimited else self.uRec)
        else:
            self.ev.EvaluateRHS(crhs, cx, self.uRec)
        self.n_rhs += 1

    # EulerSolver.hxx:674-694
    def fdtau(self, cx, dtau, alphaDiag):
        self.ev.EvaluateDt(dtau, cx, self.CFLNow, 1e100, self.cfg.useLocalDt, want_min=False)
        dtau.mul_(1.0 / alphaDiag)

    # EulerSolver.hxx:696-738: EvaluateCellRHSAlpha, then AddFixedIncrement of alphaPP * inc (with a
    # far-field state); without one, u += alpha inc
    def fincrement(self, cx, cxInc, alpha):
        if self.pp is None:
            cx.add_(cxInc, alpha=alpha)
            return
        cfg, (refRho, refP) = self.cfg, self.pp
        self.nLimInc, self.alphaMinInc = self.ev.EvaluateCellRHSAlpha(cx, cxInc, self.alphaPP, refRho, refP, cfg.incrementPPRelax, 2,
                                                                     cfg.uRecAlphaCompressPower, cfg.ppEpsIsRelaxed, 0)
        torch.mul(cxInc, self.alphaPP[:, None], out=self.incPP)
        self.ev.AddFixedIncrement(cx, self.incPP, alpha, refRho, refP, cfg.ppEpsIsRelaxed)

    def _sgs_pair(self, alphaDiag, rhs, cx, xinc, zeroIn=False):
        """doPrecondition, EulerSolver.hxx:1605-1657: forward then backward sweep, or with jacobiCode 2 two solves with
        the local LU of the block Jacobian (factored once per linear solve)."""
        if self.cfg.jacobiCode == 2:
            for it in range(2):
                self.ev.LUSGSMatrixSolveJacobianLU(alphaDiag, rhs, cx, xinc, self.tmp, self.jd, zeroIn and it == 0, want_sum=False)
                xinc.copy_(self.tmp)
            self.n_sgs += 1
            return
        gs = self.cfg.jacobiCode == 1
        self.ev.UpdateSGS(alphaDiag, rhs, cx, xinc, self.tmp, self.jd, True, gs, False, want_sum=False)
        xinc.copy_(self.tmp)
        self.ev.UpdateSGS(alphaDiag, rhs, cx, xinc, self.tmp, self.jd, False, gs, False, want_sum=False)
        xinc.copy_(self.tmp)
        self.n_sgs += 1

    # EulerSolver.hxx:740-997 and solveLinear :1407-1579
    def fsolve(self, cx, cres, res_other, dtau, dt, alphaDiag, cxInc, it, ct):
        cfg = self.cfg
        if cfg.native_linear and hasattr(self.ev, "SolveLinear"):
            self.ev.SolveLinear(alphaDiag, dtau, dt, cx, cres, cxInc, gmresCode=cfg.gmresCode, jacobiCode=cfg.jacobiCode, sgsIter=cfg.sgsIter,
                                nGmresSpace=cfg.nGmresSpace, nGmresIter=cfg.nGmresIter, precision=cfg.linear_precision,
                                meanScale=cfg.meanScale or None)
            self.n_sgs += 1 + cfg.sgsIter
            return
        if cfg.linear_precision != "fp64":
            raise ValueError("an FP32 linear solve needs the device evaluator (native_linear)")
        self.ev.LUSGSMatrixInit(self.jd, dtau, dt, alphaDiag, cx)
        if self.cfg.jacobiCode == 2:
            self.ev.LUSGSMatrixToJacobianLU(alphaDiag, cx, self.jd)
        cxInc.zero_()
        if self.cfg.gmresCode in (0, 2):
            self._sgs_pair(alphaDiag, cres, cx, cxInc, zeroIn=True)
            for _ in range(self.cfg.sgsIter):
                self._sgs_pair(alphaDiag, cres, cx, cxInc)
            if self.cfg.gmresCode == 0:
                return
        x = torch.zeros_like(cxInc)

        def FA(v, Av):
            self.ev.LUSGSMatrixVec(alphaDiag, cx, v, self.jd, Av)

        def FML(v, MLv):
            MLv.zero_()
            for i in range(1 + self.cfg.sgsIter):
                self._sgs_pair(alphaDiag, v, cx, MLv, zeroIn=i == 0)

        nv = cres.shape[1]
        ms = [m if m > 0 else 1.0 for m in (list(self.cfg.meanScale) + [1.0] * nv)[:nv]]
        s2 = torch.tensor([1.0 / (m + 1e-200) ** 2 for m in ms], dtype=cres.dtype, device=cres.device)

        def fdot(a, b):
            return float(torch.sum(a * b * s2))

        if self.cfg.gmresCode == 2:
            x.copy_(cxInc)
        self.gmres.solve(FA, FML, fdot, cres, x, self.cfg.nGmresIter, lambda i, r, rb: False)
        cxInc.copy_(x)

    # EulerSolver_Init.hxx:490-733 functor_fstop: per-variable norm of the unsteady residual against
    # the running maximum of the step, density only; CFL ramp in log space
    def fstop(self, it, res, stage):
        cfg = self.cfg
        nrm = np.asarray(self.ev.EvaluateNorm(res, cfg.normOrd, cfg.useVolWiseResidual), dtype=np.float64)
        if self.deferred:
            self.ev.CheckErrors()
        if it == 1 or self.resBase is None:
            self.resBase = np.zeros_like(nrm)
        self.resBase = np.maximum(self.resBase, nrm)
        rel = nrm / (self.resBase + VERY_SMALL)
        stop = bool(rel[0] < cfg.rhsThresholdInternal) and it >= cfg.nTimeStepInternalMin
        if cfg.vr_precision == "fp32" and cfg.vrFP64Below > 0:
            # FP32 sweep coefficients far from convergence, FP64 ones below the threshold (latched for the stage)
            if it == 1:
                self.vrPrec = "fp32"
            if rel[0] < cfg.vrFP64Below:
                self.vrPrec = "fp64"
        cfg.res_history.append((stage, it, float(rel[0])))
        if cfg.nCFLRampStart <= it <= cfg.nCFLRampLength + cfg.nCFLRampStart:
            inter = (it - cfg.nCFLRampStart) / cfg.nCFLRampLength
            self.CFLNow = math.exp(math.log(cfg.CFL) + math.log(cfg.CFLRampEnd / cfg.CFL) * inter)
        if stop or it >= cfg.nTimeStepInternal:
            self.CFLNow = cfg.CFL
        return stop

    # restart (EulerSolver_PrintData.hxx:886-1073 PrintRestart / ReadRestart): the state u and the solver's
    # running reconstruction, as a raw binary dump (dndsr_b200.checkpoint)
    def save_state(self, path, u, **meta):
        from .checkpoint import save_state
        save_state(path, u, self.uRec, **meta)

    def restore_state(self, path, u):
        """Loads a dump into u and the running reconstruction; returns its metadata."""
        from .checkpoint import load_state
        a, b, meta = load_state(path, device=u.device)
        if tuple(a.shape) != tuple(u.shape) or tuple(b.shape) != tuple(self.uRec.shape):
            raise ValueError(f"restore_state: dump shapes {tuple(a.shape)}, {tuple(b.shape)} do not match the solver's")
        u.copy_(a)
        self.uRec.copy_(b)
        return meta

    def run(self, u, n_steps=None, dt=None):
        cfg = self.cfg
        ode = ESDIRK(1 if cfg.odeCode == 0 else 0) if cfg.odeCode in (0, 101) else BDF1Stepper()
        dt = cfg.dtImplicit if dt is None else dt
        for _ in range(cfg.nTimeStep if n_steps is None else n_steps):
            ode.step(u, self.frhs, self.fdtau, self.fsolve, cfg.nTimeStepInternal, self.fstop, self.fincrement, dt)
        return u
