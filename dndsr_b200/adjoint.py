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

Both systems are solved by right-preconditioned restarted (flexible) GMRES whose Arnoldi process runs on
the device through the native Krylov reductions (``gmres``).  The u block
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


def _krylov():
    from .solver import _C
    return _C()


def gmres(op, prec, b, restart=30, max_restarts=100, rtol=1e-10, check_every=5, info=None):
    """Right-preconditioned restarted flexible GMRES for op(x) = b on tuples of FP64 CUDA tensors; x = prec(z).

    The Arnoldi process runs on the device through the library's Krylov primitives (classical Gram-Schmidt
    with the deterministic one-launch reductions of the native linear solver, least squares by Givens
    rotations in a one-thread kernel), the preconditioned columns z_j are kept (so the preconditioner may vary,
    e.g. FP32 sweeps), and the host reads the least-squares residual only every ``check_every`` Arnoldi steps
    and at each restart.  Returns x and the relative residual norms (the least-squares estimate after every
    Arnoldi step, the true residual at every restart); ``info`` (a dict) receives the number of Arnoldi
    steps and of restarts."""
    if not 1 <= int(restart) <= 32:
        raise ValueError("gmres: restart must be 1..32 (the device Krylov reductions hold up to 33 columns)")
    C = _krylov()
    shapes = [t.shape for t in b]
    sizes = [t.numel() for t in b]
    n, k = sum(sizes), int(restart)
    dev = b[0].device
    f64 = dict(dtype=torch.float64, device=dev)
    ld = C.krylov_ld(n)
    V = torch.zeros((k + 1, ld), **f64)
    Z = torch.zeros((k, ld), **f64)
    H = torch.zeros(k * (k + 1), **f64)
    gsc = torch.zeros(8 + k, **f64)
    cs = torch.zeros(k + 1, **f64)
    ones = torch.ones(k + 1, **f64)
    work = torch.zeros(C.krylov_work_bytes(), dtype=torch.uint8, device=dev)
    res = torch.zeros(k, **f64)
    x = torch.zeros(ld, **f64)

    def split(vec):
        out, o = [], 0
        for shp, sz in zip(shapes, sizes):
            out.append(vec[o:o + sz].view(shp))
            o += sz
        return tuple(out)

    def put(dst, parts):
        for d, p in zip(split(dst), parts):
            d.copy_(p)

    bflat = torch.zeros(n, **f64)
    put(bflat, b)
    bnorm = float(torch.linalg.vector_norm(bflat))
    hist = [1.0]
    if bnorm == 0.0:
        return split(x[:n]), hist
    r = torch.empty(n, **f64)
    steps = 0
    for outer in range(max_restarts):
        if info is not None:
            info.update(arnoldi_steps=steps, restarts=outer)
        if outer == 0:
            r.copy_(bflat)
        else:
            put(r, op(split(x[:n])))
            torch.sub(bflat, r, out=r)
        C.krylov_start(r, V, gsc, cs, work, k)
        if outer > 0:
            beta = float(gsc[1])
            hist.append(beta / bnorm)
            if beta <= rtol * bnorm:
                break
        done, nread = False, 0
        for j in range(k):
            z = prec(split(V[j, :n] * cs[j]))
            put(Z[j, :n], z)
            put(V[j + 1, :n], op(z))
            C.krylov_arnoldi(n, j, k, V, H, cs, gsc, res[j:j + 1], work)
            steps += 1
            if (j + 1) % check_every == 0 or j == k - 1:
                est = res[nread:j + 1].cpu().numpy() / bnorm
                hist.extend(float(e) for e in est)
                nread = j + 1
                if est[-1] <= rtol:
                    done = True
                    break
        C.krylov_update(n, k, Z, gsc, ones, x)
        if info is not None:
            info.update(arnoldi_steps=steps, restarts=outer + 1)
        if done and outer == max_restarts - 1:
            put(r, op(split(x[:n])))
            hist.append(float(torch.linalg.vector_norm(bflat - r)) / bnorm)
    return tuple(t.clone() for t in split(x[:n])), hist


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
        """(psi, lam) with A^T (psi, lam) = (gU, gRec), and the GMRES history (keyword arguments: ``gmres``'s)."""
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
