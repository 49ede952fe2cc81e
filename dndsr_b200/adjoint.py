"""Steady discrete adjoint of the implicit residual path (no reference counterpart).

The implicit solver converges the coupled steady equations

    R_u(u, uRec)   = EvaluateRHS(u, uRec)           = 0
    R_rec(u, uRec) = S(uRec, u) - uRec              = 0

where S is one VR Jacobi sweep with its boundary term (the solver performs one sweep per
pseudo-iteration, EulerSolver.hxx:238-269).  ``SteadyAdjoint`` linearises them at a state
(u, uRec): ``op`` / ``op_T`` apply the Jacobian

    A = [[dR_u/du, dR_u/duRec], [dS/du, dS/duRec - I]]

and its transpose through the device JVP / VJP kernels, with the entropy-fix scale of the
last EvaluateDt held fixed.  For an objective J(u, uRec) with gradient g = (dJ/du, dJ/duRec),
the adjoint (psi, lam) solves A^T (psi, lam) = g; the derivative of J with respect to a
source s added to the residuals is then -<(psi, lam), s>, which the tangent solve A d = -s
reproduces as <g, d> (dual consistency).

Both systems are solved by right-preconditioned restarted GMRES on the device.  The u block
is preconditioned by the scalar-Jacobian LU-SGS pair (primal) or its transpose (adjoint),
the operator of LUSGSMatrixInit/UpdateSGS (EulerEvaluator.hxx:37-159, 550-693) at a pseudo
time step of CFL ``cfl`` (the transposed sweeps optionally on FP32 vectors, ``precision="fp32"``,
inside the FP64 Krylov iteration); the uRec block by a truncated Neumann series of the sweep,
-(I + M + ... + M^k), M = dS/duRec.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _dot(a, b):
    return float(sum(torch.sum(x * y) for x, y in zip(a, b)))


def _axpy(alpha, x, y):
    return tuple(yi + alpha * xi for xi, yi in zip(x, y))


def gmres(op, prec, b, restart=30, max_restarts=100, rtol=1e-10):
    """Right-preconditioned restarted GMRES (modified Gram-Schmidt, Givens rotations) for
    op(x) = b on tuples of device tensors; x = prec(z).  Returns x and the relative residual
    norm after every Arnoldi step."""
    bnorm = math.sqrt(_dot(b, b))
    x = tuple(torch.zeros_like(t) for t in b)
    hist = [1.0]
    if bnorm == 0.0:
        return x, hist
    for outer in range(max_restarts):
        r = b if outer == 0 else _axpy(-1.0, op(x), b)
        beta = math.sqrt(_dot(r, r))
        if outer > 0:
            hist.append(beta / bnorm)
        if beta <= rtol * bnorm:
            break
        V = [tuple(t / beta for t in r)]
        Z = []
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        k = 0
        for j in range(restart):
            z = prec(V[j])
            Z.append(z)
            w = op(z)
            for i in range(j + 1):
                H[i, j] = _dot(w, V[i])
                w = _axpy(-H[i, j], V[i], w)
            H[j + 1, j] = math.sqrt(_dot(w, w))
            V.append(tuple(t / H[j + 1, j] for t in w) if H[j + 1, j] > 0 else w)
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            d = math.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = H[j, j] / d, H[j + 1, j] / d
            H[j, j], H[j + 1, j] = d, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            k = j + 1
            hist.append(abs(g[j + 1]) / bnorm)
            if abs(g[j + 1]) <= rtol * bnorm:
                break
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        for i in range(k):
            x = _axpy(float(y[i]), Z[i], x)
        if hist[-1] <= rtol:
            r = _axpy(-1.0, op(x), b)
            hist.append(math.sqrt(_dot(r, r)) / bnorm)
            if hist[-1] <= rtol:
                break
    return x, hist


class SteadyAdjoint:
    """The coupled steady residual linearised at (u, uRec); see the module docstring."""

    def __init__(self, vr, ev, u, uRec, cfl=5.0, alphaDiag=1.0, n_neumann=4, dt=math.inf, precision="fp64"):
        self.vr, self.ev, self.u, self.uRec = vr, ev, u.contiguous(), uRec.contiguous()
        self.alphaDiag, self.n_neumann = alphaDiag, n_neumann
        # "fp32": the transposed LU-SGS preconditioner sweeps FP32 vectors (the operator stays FP64)
        self.pdt = torch.float32 if precision == "fp32" else torch.float64
        # dt < inf: the residual of one implicit Euler step, R_u - (u - u_n) / dt (its Jacobian gains -I / dt)
        self.idt = 0.0 if math.isinf(dt) else 1.0 / dt
        n = u.shape[0]
        self.dTau = torch.zeros(n, dtype=torch.float64, device=u.device)
        ev.EvaluateDt(self.dTau, self.u, cfl, 1e100, True)
        self.jd = ev.BuildJDiag()
        ev.LUSGSMatrixInit(self.jd, self.dTau, 1e100 if self.idt == 0.0 else dt, alphaDiag)

    # Jacobian and transpose of (R_u, R_rec)
    def op(self, x):
        du, dRec = x
        a = self.ev.EvaluateRHSJVP(du, dRec, self.u, self.uRec)
        if self.idt:
            a = a - self.idt * du
        b = self.vr.DoReconstructionIterJVP(dRec, du, self.uRec, self.u) - dRec
        return a, b

    def op_T(self, y):
        psi, lam = y
        gu, gRec = self.ev.EvaluateRHSVJP(psi, self.u, self.uRec)
        if self.idt:
            gu = gu - self.idt * psi
        vRec, vU = self.vr.DoReconstructionIterVJP(lam, self.uRec, self.u)
        return gu + vU, gRec + vRec - lam

    # preconditioners: u block -(LU-SGS pair) ~ (dR_u/du)^-1, uRec block -(I + M + ... + M^k) ~ (M - I)^-1
    def _sgs_pair(self, r, transposed):
        ev, a, jd = self.ev, self.alphaDiag, self.jd
        if transposed:
            rp = r.to(self.pdt).contiguous()
            z0 = torch.zeros_like(rp)
            z1, z2 = torch.empty_like(rp), torch.empty_like(rp)
            ev.UpdateSGST(a, rp, self.u, z0, z1, jd, True)
            ev.UpdateSGST(a, rp, self.u, z1, z2, jd, False)
            return z2.to(r.dtype)
        z0 = torch.zeros_like(r)
        z1, z2 = torch.empty_like(r), torch.empty_like(r)
        ev.UpdateSGS(a, r, self.u, z0, z1, jd, True, want_sum=False)
        ev.UpdateSGS(a, r, self.u, z1, z2, jd, False, want_sum=False)
        return z2

    def _neumann(self, r, transposed):
        acc, t = r.clone(), r
        zu = torch.zeros_like(self.u)
        for _ in range(self.n_neumann):
            if transposed:
                t, _ = self.vr.DoReconstructionIterVJP(t, self.uRec, self.u)
            else:
                t = self.vr.DoReconstructionIterJVP(t, zu, self.uRec, self.u)
            acc = acc + t
        return acc

    def prec(self, r):
        return -self._sgs_pair(r[0], False), -self._neumann(r[1], False)

    def prec_T(self, r):
        return -self._sgs_pair(r[0], True), -self._neumann(r[1], True)

    def solve_adjoint(self, gU, gRec, **kw):
        """(psi, lam) with A^T (psi, lam) = (gU, gRec), and the GMRES history."""
        x, hist = gmres(self.op_T, self.prec_T, (gU.contiguous(), gRec.contiguous()), **kw)
        return x[0], x[1], hist

    def shape_gradient(self, psi, lam, dJdX=None):
        """dJ/dX for the node coordinates X [nNode][3] at the converged state: the residuals R(u, uRec; X)
        stay zero, so dJ/dX = dJ/dX|_state - psi^T dR_u/dX - lam^T dS/dX (the time term of the implicit
        step and -uRec do not depend on X).  dJdX: the objective's own derivative (e.g.
        ``ev.PressureForceCoords``), or None for an objective of the state only."""
        g = self.ev.ResidualVJPCoords(psi.contiguous(), lam.contiguous(), self.u, self.uRec)
        return -g if dJdX is None else dJdX - g

    def solve_tangent(self, sU, sRec, **kw):
        """(du, dRec) with A (du, dRec) = -(sU, sRec): the state response to a residual source."""
        x, hist = gmres(self.op, self.prec, (-sU.contiguous(), -sRec.contiguous()), **kw)
        return x[0], x[1], hist
