"""torch.autograd bindings of the residual path.

``ResidualFunction`` is EvaluateRHS(u, uRec) with its hand-written VJP as the
backward; ``ReconstructionSweep`` is one VR Jacobi sweep (DoReconstructionIter,
putIntoNew) with the transposed sweep as the backward.  Composing them,

    uRec = uRec0
    for _ in range(k):
        uRec = ReconstructionSweep.apply(uRec, u, vr)
    rhs = ResidualFunction.apply(u, uRec, ev)

is the residual the implicit solver sees after k reconstruction sweeps, and
``torch.autograd.grad`` of any scalar of ``rhs`` runs the device VJP kernels in
reverse order.  The entropy-fix scale (deltaLambdaCell of the last EvaluateDt)
is held fixed, as between the reference's EvaluateDt and EvaluateRHS calls.
"""
from __future__ import annotations

import torch


class ResidualFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, uRec, ev):
        u, uRec = u.contiguous(), uRec.contiguous()
        rhs = torch.empty_like(u)
        ev.EvaluateRHS(rhs, u, uRec)
        ctx.save_for_backward(u, uRec)
        ctx.ev = ev
        return rhs

    @staticmethod
    def backward(ctx, w):
        u, uRec = ctx.saved_tensors
        du, duRec = ctx.ev.EvaluateRHSVJP(w.contiguous(), u, uRec)
        return du, duRec, None


class ReconstructionSweep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, uRec, u, vr):
        uRec, u = uRec.contiguous(), u.contiguous()
        new = torch.empty_like(uRec)
        vr.DoReconstructionIter(uRec, new, u, putIntoNew=True)
        ctx.save_for_backward(uRec, u)
        ctx.vr = vr
        return new

    @staticmethod
    def backward(ctx, cot):
        uRec, u = ctx.saved_tensors
        vRec, vU = ctx.vr.DoReconstructionIterVJP(cot.contiguous(), uRec, u)
        return vRec, vU, None


def residual(u, uRec0, vr, ev, n_sweeps=1):
    """EvaluateRHS after ``n_sweeps`` VR sweeps from ``uRec0``, differentiable in u and uRec0."""
    uRec = uRec0
    for _ in range(n_sweeps):
        uRec = ReconstructionSweep.apply(uRec, u, vr)
    return ResidualFunction.apply(u, uRec, ev)
