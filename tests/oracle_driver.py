"""Adapters that give the CPU oracle the evaluator interface the implicit driver uses.

Test infrastructure: lets tests run dndsr_b200.implicit on the oracle and on
the GPU library with identical orchestration and compare the trajectories.
"""
import numpy as np
import torch


class OracleVR:
    def __init__(self, o):
        self.o, self.mesh, self.R = o, o.mesh, o.R

    def BuildURec(self, nv):
        return torch.zeros((self.mesh.n_cell, self.R, nv), dtype=torch.float64)

    def BuildUDof(self, nv):
        return torch.zeros((self.mesh.n_cell, nv), dtype=torch.float64)

    def get(self, name):
        return self.o.get(name)

    def DoReconstructionIter(self, uRec, uRecNew, u, putIntoNew=False, recordInc=False, uRecIsZero=False, precision="fp64"):
        new = torch.tensor(self.o.vr_iter(uRec.numpy(), u.numpy(), recordInc, uRecIsZero))
        if putIntoNew:
            uRecNew.copy_(new)
        else:
            uRecNew.copy_(uRec)
            uRec.copy_(new)


class OracleEval:
    def __init__(self, o):
        self.o, self.nVars = o, o.nv
        self.vol = o.get("volume")

    def EvaluateRHS(self, rhs, u, uRec, uRecUnlim=None):
        if uRecUnlim is None:
            rhs.copy_(torch.tensor(self.o.eval_rhs(u.numpy(), uRec.numpy())))
        else:
            rhs.copy_(torch.tensor(self.o.eval_rhs_full(u.numpy(), uRecUnlim.numpy(), uRec.numpy())[0]))

    def EvaluateDt(self, dt, u, CFL, MaxDt=1e100, UseLocaldt=True, want_min=True):
        d, mn = self.o.eval_dt(u.numpy(), CFL, MaxDt, UseLocaldt)
        dt.copy_(torch.tensor(d))
        return mn

    blockJacobian = False

    def SetJacobianMode(self, useScalarJacobian=True, useRoeJacobian=False):
        self.o.set_jacobian_mode(useScalarJacobian, useRoeJacobian)
        self.blockJacobian = not useScalarJacobian

    def BuildJDiag(self):
        n, nv = self.vol.shape[0], self.nVars
        if self.blockJacobian:
            return torch.zeros((n, 2, nv, nv), dtype=torch.float64)
        return torch.zeros((n, nv) if nv == 6 else (n,), dtype=torch.float64)

    def LUSGSMatrixInit(self, jd, dTau, dt, alphaDiag, u=None):
        if self.blockJacobian:
            jd.copy_(torch.tensor(self.o.lusgs_init_block(dTau.numpy(), dt, alphaDiag, u.numpy())))
        else:
            jd.copy_(torch.tensor(self.o.lusgs_init(dTau.numpy(), dt, alphaDiag)))

    def LUSGSMatrixToJacobianLU(self, alphaDiag, u, jd):
        self.o.jacobian_lu(alphaDiag, u.numpy(), jd.numpy())

    def LUSGSMatrixSolveJacobianLU(self, alphaDiag, rhs, u, uInc, uIncNew, jd, uIncIsZero=False, want_sum=True):
        out, s = self.o.solve_jacobian_lu(alphaDiag, rhs.numpy(), u.numpy(), uInc.numpy(), jd.numpy(), uIncIsZero)
        uIncNew.copy_(torch.tensor(out))
        return s

    def UpdateSGS(self, alphaDiag, rhs, u, uInc, uIncNew, jd, forward, gsUpdate=True, uIncIsZero=False, want_sum=True):
        out, s = self.o.update_sgs(alphaDiag, rhs.numpy(), u.numpy(), uInc.numpy(), uIncNew.numpy(), jd.numpy(), forward, gsUpdate,
                                   uIncIsZero)
        uIncNew.copy_(torch.tensor(out))
        return s

    def LUSGSMatrixVec(self, alphaDiag, u, uInc, jd, Au):
        Au.copy_(torch.tensor(self.o.lusgs_matvec(alphaDiag, u.numpy(), uInc.numpy(), jd.numpy())))

    def EvaluateNorm(self, x, P=1, volWise=True):
        a = np.abs(x.numpy())
        w = self.vol[:, None] if volWise else 1.0
        if P == 1:
            return (a * w).sum(0)
        if P == 2:
            return np.sqrt((a * a * w).sum(0))
        return a.max(0)
