#!/usr/bin/env python
"""Throughput of the implicit residual path on one B200: Mcell*RHS/s in FP64.

Workload (the 3-D Navier-Stokes Taylor-Green configuration): periodic
[0, 2 pi]^3, 64^3 hexahedra (262,144 cells) with seeded +-5% node jitter,
Re = 1600 (mu = 1/1600, constant viscosity), Mach 0.1 Taylor-Green initial
field, VR degree 2 (intOrder 5: 9 Gauss points per face), HLLE+ convective
flux with the compact viscous flux.  One step = one RHS evaluation as the
reference's solver performs it per pseudo-iteration: one VR block-Jacobi
sweep followed by EvaluateRHS (Gauss-point reconstruction, Riemann and
viscous flux, per-cell gather).

Arms:
  default           the CUDA library through the C-ABI (value: device-resident
                    inputs; e2e: host buffers with the copies inside the timing)
  --impl reference  the reference's CPU algorithm (the oracle port, OpenMP on
                    all host cores; the reference itself cannot be built here)
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell*RHS/s FP64 (one VR sweep + EvaluateRHS per step)"
UNIT = "Mcell*RHS/s"
# algorithmic bytes per cell (compulsory FP64 traffic under the reference data model, basis recomputed):
#   RHS:  8*[(R+2)*nv + (2d+1+R) + (nf/2)*(gF*(2d+1)+1)] with d=3, nv=5, R=9, nf=6, gF=9 -> 2104 B
#   VR:   8*(nf*R^2 + nf*R) + 8*(2*R*nv + nv) -> 5080 B
B_RHS = 8 * ((9 + 2) * 5 + (2 * 3 + 1 + 9) + 3 * (9 * (2 * 3 + 1) + 1))
B_VR = 8 * (6 * 81 + 6 * 9) + 8 * (2 * 9 * 5 + 5)
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes per cell of one k_rhs_face_fast launch (the face kernel: 97% of EvaluateRHS; the per-cell
# gather adds ~4% more bytes), from the ncu capture of the same workload at 48^3 (dram__bytes_read.sum +
# dram__bytes_write.sum = 273.1 MB for 110,592 cells); traffic grows in proportion to cells and faces, so
# a 64^3 launch is scaled by the cell count
RHS_TRAFFIC_PER_CELL = 273.1e6 / 48 ** 3
RHS_FP64_PIPE_PCT = 30.5  # sm__pipe_fp64_cycles_active of the same capture
# algorithmic flops per cell (F_alg), counted by the op-counting build of the oracle on this workload
# (python -m oracle.falg: +, -, *, / and sqrt one each; profiles/falg_tgv_p2.md)
F_RHS = {2: 50310.0, 1: 30546.0}
F_VR = {2: 6300.0, 1: 1020.0}
# the reference's published TGV throughput for this path: 71.8 M cell-iterations/s on 10,240 CPU ranks
REF_PUBLISHED_MCIPS = 71.8


def workload_config(n, p):
    return {"workload": f"Taylor-Green vortex NS, periodic [0,2pi]^3, {n}^3 hex ({n ** 3} cells), +-5% jitter, Re=1600, "
                        f"VR degree {p} (intOrder 5), HLLE+ + compact viscous flux; step = VR Jacobi sweep + EvaluateRHS",
            "cells": n ** 3, "vr_degree": p, "riemann": "HLLEP", "gauss_points_per_face": 9,
            "l2": "working set (VR matrices 1.19 GB) exceeds the 126 MB L2; no flush needed"}


VR_SETTINGS = dict(intOrder=5, dirWeightScheme="HQM_OPT", geomWeightScheme="HQM_SD", geomWeightBias=1.0, geomWeightPower=0.5)
EULER_SETTINGS = dict(nVars=5, riemannSolverType="HLLEP", muGas=1.0 / 1600, muModel=0, prGas=0.71, gamma=1.4, Rgas=1.0)


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def fp64_peak_tflops(dev):
    """FP64 throughput of cuBLAS DGEMM (8192^3, best of 5 after a warm-up) on this GPU: the measured FP64 peak the
    FP64-pipe fraction of the RHS is quoted against (MEASURED_PEAKS.json carries no FP64 figure)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = a @ b
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b, out=c)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b, c
    torch.cuda.empty_cache()
    return best


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 2 + i and r[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_baseline_oracle(n_sample, p, seconds, threads=None):
    """Times the oracle port (OpenMP) on a bounded sample of the same workload: a smaller TGV mesh with the same settings."""
    import oracle
    from dndsr_b200 import mesh as M
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    m = M.tgv_mesh(n_sample)
    vr = dict(maxOrder=p, intOrder=5, jacobiRelax=1.0, SORInstead=0, scaleType=1, scaleMultiplier=1.0, dirWeightScheme=1,
              geomWeightScheme=1, geomWeightBias=1.0, geomWeightPower=0.5, bcWeight=1.0)
    es = dict(nVars=5, rsType=oracle.RS["HLLEP"], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=1.0 / 1600, prGas=0.71,
              TRef=273.15, CSutherland=110.4, muModel=0, ignoreVis=0)
    o = oracle.Oracle(m, vr, es)
    o.construct()
    u = o.init_field(3)
    uRec = np.zeros((m.n_cell, o.R, 5))
    o.eval_dt(u, 5.0)
    for _ in range(2):
        uRec = o.vr_iter(uRec, u)
        o.eval_rhs(u, uRec)
    steps, t0 = 0, time.perf_counter()
    while True:
        uRec = o.vr_iter(uRec, u)
        o.eval_rhs(u, uRec)
        steps += 1
        el = time.perf_counter() - t0
        if el > seconds:
            break
    cpu_baseline_oracle.per_operator = _cpu_per_operator(o, u, uRec, m.n_cell)
    return m.n_cell * steps / el / 1e6, steps, el, m.n_cell


def _cpu_per_operator(o, u, uRec, n_cell, reps=5, warm=2):
    """Median CPU times of the oracle's operators on the sample (after warm-up): the VR sweep (a1),
    EvaluateRHS (a9) and one forward + backward SGS sweep pair (a14)."""
    dTau, _ = o.eval_dt(u, 5.0)
    jd = o.lusgs_init(dTau, 1e100, 1.0)
    rhs = o.eval_rhs(u, uRec)
    z, t1, t2 = np.zeros_like(u), np.zeros_like(u), np.zeros_like(u)

    def sgs_pair():
        o.update_sgs(1.0, rhs, u, z, t1, jd, True)
        o.update_sgs(1.0, rhs, u, t1, t2, jd, False)

    ops = {"vr_sweep": lambda: o.vr_iter(uRec, u), "evaluate_rhs": lambda: o.eval_rhs(u, uRec), "sgs_pair": sgs_pair}
    out = {}
    for name, fn in ops.items():
        ts = []
        for i in range(warm + reps):
            t0 = time.perf_counter()
            fn()
            if i >= warm:
                ts.append(time.perf_counter() - t0)
        ms = float(np.median(ts)) * 1e3
        out[name] = {"ms": ms, "mcell_per_s": n_cell / ms / 1e3}
    return out


def _bump_c3(nx, ny, nz, p=1):
    """The transonic bump of the steady configuration: channel [-2,2]x[0,1]x[0,0.5], bump 0.05 exp(-25 x^2) on
    the floor, tetrahedra; BCFar inflow and outflow, BCWallInvis floor and ceiling, BCSym side planes; Mach 0.8;
    VR degree p; the Roe flux with the Lax-type eigenvalues of Roe_M2 (Gas.hpp:1082-1090)."""
    from dndsr_b200 import mesh as M
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction, euler_bc_dir_weights
    mesh = M.bump_channel_tet(nx, ny, nz)
    far = M.freestream(0.8)
    types = np.zeros(7, np.int32)
    vals = np.zeros((7, 5))
    for z, tp in M.BUMP_BC_TYPES.items():
        types[z], vals[z] = tp, far
    vr = VariationalReconstruction(mesh, dict(maxOrder=p, intOrder=2 if p == 1 else 5, dirWeightScheme="HQM_OPT", geomWeightScheme="HQM_SD",
                                              geomWeightBias=1.0)).construct(euler_bc_dir_weights(types))
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe_M2", muGas=0.0, ignoreVis=True))
    ev.SetBC(types, vals)
    return mesh, vr, ev, far


def run_steady(args):
    """Wall time to a 1e-10 residual drop, mixed vs FP64, on the steady transonic bump (BCFar in/out, BCWallInvis
    floor/ceiling, BCSym sides, Mach 0.8, VR degree 1, Roe_M2): BDF1 dual time at CFL 200, GMRES(30) preconditioned
    by one SGS pair, FP64 or FP32 linear solve inside the FP64 defect correction, each precision from the free
    stream after a two-iteration warm-up; on the configuration's ~2M-tet mesh and on a 250k-tet one.  With the Roe
    Jacobian (roe_jacobian): the same runs with the block Roe Jacobian and the local LU preconditioner."""
    import torch
    from dndsr_b200 import implicit as I

    # the scalar Jacobian: CFL 200, GMRES(30) preconditioned by one SGS pair, one VR sweep per iteration;
    # the Roe Jacobian (useRoeJacobian, block diagonal): CFL 1e4, GMRES(10) preconditioned by the local LU
    # (jacobiCode 2, block ILU(0)), four VR sweeps per iteration
    SCALAR = dict(CFL=200.0, gmresCode=1, nGmresSpace=30, jacobiCode=1, nInternalRecStep=1)
    ROE = dict(CFL=1e4, gmresCode=1, nGmresSpace=10, jacobiCode=2, nInternalRecStep=4)

    def solve(vr, ev, far, prec, iters, thr, lin=SCALAR):
        ev.SetJacobianMode(lin is SCALAR, lin is ROE)
        u = vr.BuildUDof(5)
        u[:] = torch.tensor(far, device="cuda")
        I.ImplicitSolver(vr, ev, I.SolverConfig(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=2, nTimeStepInternalMin=2,
                                                linear_precision=prec, **lin)).run(u)
        u[:] = torch.tensor(far, device="cuda")
        cfg = I.SolverConfig(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=iters, nTimeStepInternalMin=5, nGmresIter=1, sgsIter=0,
                             rhsThresholdInternal=thr, linear_precision=prec, **lin)
        solver = I.ImplicitSolver(vr, ev, cfg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver.run(u)
        torch.cuda.synchronize()
        return u, time.perf_counter() - t0, len(cfg.res_history), cfg.res_history[-1][2], solver

    def measure(dims, iters):
        nx, ny, nz = dims
        mesh, vr, ev, far = _bump_c3(nx, ny, nz)
        out = {}
        for prec in ("fp64", "fp32"):
            out[prec] = solve(vr, ev, far, prec, iters, 1e-10)
        a, b = out["fp64"], out["fp32"]
        # component times at the converged state (CUDA events, 5 calls each)
        comp = {}
        for prec in ("fp64", "fp32"):
            s = out[prec][4]
            u = out[prec][0]
            rhs = torch.zeros_like(u)
            dtau = torch.zeros(mesh.n_cell, dtype=torch.float64, device="cuda")
            xinc = torch.zeros_like(u)
            s.fdtau(u, dtau, 1.0)
            evs = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            evs[0].record()
            for _ in range(5):
                s.frhs(rhs, u, dtau, 1, 1.0)
            evs[1].record()
            for _ in range(5):
                s.fsolve(u, rhs, rhs, dtau, 1e100, 1.0, xinc, 1, 1.0)
            evs[2].record()
            torch.cuda.synchronize()
            comp[prec] = (evs[0].elapsed_time(evs[1]) / 5, evs[1].elapsed_time(evs[2]) / 5)
        res = {"cells": mesh.n_cell, "mesh": f"{nx}x{ny}x{nz}x6 tets",
               "converged_fp64": a[3] < 1e-10, "converged_mixed": b[3] < 1e-10,
               "iterations_fp64": a[2], "iterations_mixed": b[2], "fp64_s": a[1], "mixed_s": b[1], "mixed_over_fp64_time": b[1] / a[1],
               "fp64_ms_per_iter": 1e3 * a[1] / a[2], "mixed_ms_per_iter": 1e3 * b[1] / b[2],
               "final_drop_fp64": a[3], "final_drop_mixed": b[3],
               "state_rel_diff": float((a[0] - b[0]).abs().max() / a[0].abs().max()),
               "ms_vr_sweep_plus_rhs": comp["fp64"][0], "ms_linear_solve_fp64": comp["fp64"][1], "ms_linear_solve_fp32": comp["fp32"][1]}
        if args.steady_roe:
            roe = {}
            for prec in ("fp64", "fp32"):
                roe[prec] = solve(vr, ev, far, prec, iters, 1e-10, ROE)
            c, d = roe["fp64"], roe["fp32"]
            res["roe_jacobian"] = {
                "settings": "useRoeJacobian (block diagonal), CFL 1e4, GMRES(10) preconditioned by the local LU (jacobiCode 2, block "
                            "ILU(0) in colour order), nInternalRecStep 4",
                "converged_fp64": c[3] < 1e-10, "converged_mixed": d[3] < 1e-10, "iterations_fp64": c[2], "iterations_mixed": d[2],
                "fp64_s": c[1], "mixed_s": d[1], "mixed_over_fp64_time": d[1] / c[1], "fp64_ms_per_iter": 1e3 * c[1] / c[2],
                "mixed_ms_per_iter": 1e3 * d[1] / d[2], "final_drop_fp64": c[3], "final_drop_mixed": d[3],
                "fp64_over_scalar_fp64_time": c[1] / a[1], "mixed_over_scalar_fp64_time": d[1] / a[1],
                "state_rel_diff_vs_scalar": float((c[0] - a[0]).abs().max() / a[0].abs().max())}
            del roe, c, d
            ev.SetJacobianMode(True, False)
        del out, vr, ev
        torch.cuda.empty_cache()
        return res

    # the configuration's ~2M-tet mesh, then a 250k-tet one
    res = {"workload": "steady Euler over the bump, BCFar in/out, BCWallInvis floor/ceiling, BCSym sides, Mach 0.8, VR degree 1, "
                       "Roe_M2, BDF1 dual time CFL 200, GMRES(30) preconditioned by one SGS pair; each precision run from the free "
                       "stream to a 1e-10 density residual drop",
           **measure(args.steady_big_mesh, args.steady_big_iters)}
    res["small_mesh"] = measure(args.steady_mesh, args.steady_iters)
    return res


def run_linear_solve(args):
    """One native linear solve (dndsb_eval_solve_linear) on the steady bump at a perturbed free stream, CUDA events over
    5 calls after 2: the scalar Jacobian with GMRES(30) and one SGS pair, the Roe Jacobian with GMRES(10) and the local
    LU (block ILU(0)), each FP64 and FP32; 'build_factor_pair' is gmresCode 0 (the operator build, the ILU
    factorisation and one preconditioner application)."""
    import torch
    nx, ny, nz = args.linear_mesh
    mesh, vr, ev, far = _bump_c3(nx, ny, nz)
    u = vr.BuildUDof(5)
    u[:] = torch.tensor(far, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(1)
    u[:, 0] *= 1 + 0.01 * torch.rand(mesh.n_cell, device="cuda", dtype=torch.float64, generator=g)
    uRec = vr.BuildURec(5)
    dt = torch.zeros(mesh.n_cell, dtype=torch.float64, device="cuda")
    rhs = torch.zeros_like(u)
    out = {"workload": f"steady bump, {mesh.n_cell} tets, VR degree 1, Roe_M2, local pseudo time step at CFL 1e4, dt = 1e100",
           "cells": mesh.n_cell}
    for mode, cases in (("scalar", ((1, 30, 1, "gmres30_sgs"),)), ("roe", ((1, 10, 2, "gmres10_ilu"), (0, 1, 2, "build_factor_pair")))):
        ev.SetJacobianMode(mode == "scalar", mode == "roe")
        ev.EvaluateDt(dt, u, 1e4)
        ev.EvaluateRHS(rhs, u, uRec)
        for code, k, jac, name in cases:
            for prec in ("fp64", "fp32"):
                x = torch.zeros_like(u)
                for _ in range(2):
                    ev.SolveLinear(1.0, dt, 1e100, u, rhs, x, gmresCode=code, nGmresSpace=k, jacobiCode=jac, precision=prec)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(5):
                    ev.SolveLinear(1.0, dt, 1e100, u, rhs, x, gmresCode=code, nGmresSpace=k, jacobiCode=jac, precision=prec)
                b.record()
                torch.cuda.synchronize()
                out[f"{mode}_{name}_{prec}_ms"] = a.elapsed_time(b) / 5
    ev.SetJacobianMode(True, False)
    return out


def run_dual_time(args):
    """Wall time to a 1e-10 residual drop, mixed vs FP64, where the defect correction converges: one ESDIRK4
    step of the TGV workload (dt 0.02, local pseudo time step at CFL 50, GMRES(30) preconditioned by one SGS
    pair), every stage's pseudo-time iterations run until the density residual falls below 1e-10 of its
    maximum.  Each precision is warmed up once (workspace, CUDA graph) before its timed run."""
    import torch
    from dndsr_b200 import implicit as I
    from dndsr_b200 import mesh as M
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    n, p = args.n, args.p
    mesh = M.tgv_mesh(n)
    vr = VariationalReconstruction(mesh, dict(VR_SETTINGS, maxOrder=p)).construct()
    ev = EulerEvaluator(vr, EULER_SETTINGS)

    def measure(lin):
        out = {}
        for prec in ("fp64", "fp32"):
            for timed_run in (False, True):
                u = vr.BuildUDof(5)
                ev.InitializeUDOF(u, 3)
                cfg = I.SolverConfig(odeCode=0, dtImplicit=0.02, nTimeStep=1, nTimeStepInternal=300 if timed_run else 2,
                                     nTimeStepInternalMin=5 if timed_run else 2, CFL=50.0, nGmresIter=1, rhsThresholdInternal=1e-10,
                                     linear_precision=prec, **lin)
                solver = I.ImplicitSolver(vr, ev, cfg)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                solver.run(u)
                torch.cuda.synchronize()
                el = time.perf_counter() - t0
            final = {}
            for (stage, it, rel) in cfg.res_history:
                final[stage] = (it, rel)
            out[prec] = (u, el, len(cfg.res_history), max(r for (_, r) in final.values()), [it for (it, _) in final.values()])
        return out["fp64"], out["fp32"]

    a, b = measure(dict(gmresCode=1, nGmresSpace=30, sgsIter=0))
    res = {"workload": f"one ESDIRK4 step of the TGV workload ({n}^3 hex, VR degree {p}, HLLE+ viscous), dt 0.02, pseudo time step "
                       "CFL 50, GMRES(30) with one SGS pair; every stage iterated to a 1e-10 density residual drop",
           "fp64_s": a[1], "mixed_s": b[1], "mixed_over_fp64_time": b[1] / a[1],
           "inner_iterations_fp64": a[2], "inner_iterations_mixed": b[2], "iterations_per_stage_fp64": a[4],
           "worst_final_drop_fp64": a[3], "worst_final_drop_mixed": b[3],
           "state_rel_diff": float((a[0] - b[0]).abs().max() / a[0].abs().max())}
    # the same step with LU-SGS alone (two SGS pairs per linear solve, no GMRES): the pseudo-iteration count is set by
    # the reconstruction, not by the linear solve, so the cheaper solve reaches 1e-10 in about as many iterations
    c, d = measure(dict(gmresCode=0, sgsIter=1))
    res["lusgs_only"] = {"settings": "gmresCode 0, two SGS pairs per linear solve (sgsIter 1)", "fp64_s": c[1], "mixed_s": d[1],
                         "mixed_over_fp64_time": d[1] / c[1], "inner_iterations_fp64": c[2], "inner_iterations_mixed": d[2],
                         "worst_final_drop_fp64": c[3], "fp64_over_gmres30_fp64_time": c[1] / a[1],
                         "state_rel_diff_vs_gmres30": float((c[0] - a[0]).abs().max() / a[0].abs().max())}
    return res


def run_sa_plate(args):
    """The SA flat-plate workload at full size: Re_L 5e6, Mach 0.2, nuTilde_inf = 3 nu, stretched hexahedra
    (first cell 5e-6, growth 1.1), VR degree 1, Roe, 6 variables (NS_SA with the IDDES length scale and the
    analytic wall distance).  Reported: VR sweep + EvaluateRHS throughput (CUDA events) and BDF1 pseudo
    iterations (CFL 50, GMRES(30) with one SGS pair) with the FP64 and the FP32 linear solve, each after a
    two-iteration warm-up."""
    import torch
    from dndsr_b200 import implicit as I
    from dndsr_b200 import mesh as M
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    nx, ny, nz = args.sa_mesh
    mesh = M.flat_plate_hex(nx, ny, nz, y1=5e-6, growth=1.1)
    far5 = M.freestream(0.2)
    mu = np.linalg.norm(far5[1:4]) / far5[0] / 5e6
    far = np.concatenate([far5, [3.0 * far5[0]]])
    types, vals = np.zeros(6, np.int32), np.zeros((6, 6))
    w = np.ones((6, 4))
    for z, tp in M.PLATE_BC_TYPES.items():
        types[z], vals[z], w[z] = tp, far, (1, 0, 0, 0)
    vr = VariationalReconstruction(mesh, dict(maxOrder=1, intOrder=3, dirWeightScheme="HQM_OPT", geomWeightScheme="HQM_SD",
                                              geomWeightBias=1.0)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType="Roe", muGas=mu, muModel=0, prGas=0.72))
    ev.SetBC(types, vals)
    ev.SetWallDistance(M.plate_wall_distance(vr.get("cellPP").reshape(mesh.n_cell, -1, 3)))
    u = vr.BuildUDof(6)
    u[:] = torch.tensor(far, device="cuda")
    uRec, tmp, rhs = vr.BuildURec(6), vr.BuildURec(6), torch.zeros_like(u)
    dt = torch.zeros(mesh.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    vr.DoReconstructionIter(uRec, tmp, u, putIntoNew=False)
    ev.EvaluateRHS(rhs, u, uRec)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(5):
        vr.DoReconstructionIter(uRec, tmp, u, putIntoNew=False)
        ev.EvaluateRHS(rhs, u, uRec)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / 5
    out = {"workload": f"SA flat plate, {mesh.n_cell} hex ({nx}x{ny}x{nz}), Re_L 5e6, Mach 0.2, VR degree 1, Roe, 6 variables",
           "ms_vr_sweep_plus_rhs": ms, "mcell_rhs_per_s": mesh.n_cell / ms / 1e3}
    res = {}
    for prec in ("fp64", "fp32"):
        u[:] = torch.tensor(far, device="cuda")
        I.ImplicitSolver(vr, ev, I.SolverConfig(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=2, nTimeStepInternalMin=2,
                                                CFL=50.0, gmresCode=1, nGmresSpace=30, linear_precision=prec)).run(u)
        u[:] = torch.tensor(far, device="cuda")
        cfg = I.SolverConfig(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=args.sa_iters, nTimeStepInternalMin=args.sa_iters,
                             CFL=50.0, gmresCode=1, nGmresSpace=30, nGmresIter=1, sgsIter=0, rhsThresholdInternal=1e-9, linear_precision=prec)
        solver = I.ImplicitSolver(vr, ev, cfg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver.run(u)
        torch.cuda.synchronize()
        res[prec] = (u.clone(), time.perf_counter() - t0, len(cfg.res_history), cfg.res_history[-1][2])
    a64, a32 = res["fp64"], res["fp32"]
    out.update({"iterations": a64[2], "fp64_ms_per_iter": 1e3 * a64[1] / a64[2], "mixed_ms_per_iter": 1e3 * a32[1] / a32[2],
                "mixed_over_fp64_time": a32[1] / a64[1], "residual_drop_fp64": a64[3], "residual_drop_mixed": a32[3],
                "state_rel_diff": float((a64[0] - a32[0]).abs().max() / a64[0].abs().max())})
    del vr, ev, u, uRec, tmp, rhs, res, solver
    torch.cuda.empty_cache()
    out["adjoint"] = sa_adjoint(args)
    return out


def sa_adjoint(args):
    """The skin-friction adjoint with the SA terms (the x force of the wall flux, pressure and friction,
    EvaluateRHS.hxx:599-637) on a smaller plate (the same settings) after a bounded primal solve: CUDA-event
    times of EvaluateRHS and its VJP (SA convective/diffusion fluxes, eddy viscosity, source; forward-mode
    kernels), of the VR sweep and its VJP and of the objective gradient; then the adjoint of the coupled
    residual of one implicit step (dt = 5 of the median local steps) by the device GMRES(32) with the
    transposed LU-SGS pair (pseudo time step CFL 20) to a 1e-8 drop, bounded in restarts."""
    import torch
    from dndsr_b200 import implicit as I
    from dndsr_b200 import mesh as M
    from dndsr_b200.adjoint import SteadyAdjoint
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    nx, ny, nz = args.sa_adjoint_mesh
    mesh = M.flat_plate_hex(nx, ny, nz, y1=5e-6, growth=1.1)
    far5 = M.freestream(0.2)
    mu = np.linalg.norm(far5[1:4]) / far5[0] / 5e6
    far = np.concatenate([far5, [3.0 * far5[0]]])
    types, vals = np.zeros(6, np.int32), np.zeros((6, 6))
    w = np.ones((6, 4))
    for z, tp in M.PLATE_BC_TYPES.items():
        types[z], vals[z], w[z] = tp, far, (1, 0, 0, 0)
    vr = VariationalReconstruction(mesh, dict(maxOrder=1, intOrder=3, dirWeightScheme="HQM_OPT", geomWeightScheme="HQM_SD",
                                              geomWeightBias=1.0)).construct(w)
    ev = EulerEvaluator(vr, dict(nVars=6, riemannSolverType="Roe", muGas=mu, muModel=0, prGas=0.72))
    ev.SetBC(types, vals)
    ev.SetWallDistance(M.plate_wall_distance(vr.get("cellPP").reshape(mesh.n_cell, -1, 3)))
    u = vr.BuildUDof(6)
    u[:] = torch.tensor(far, device="cuda")
    cfg = I.SolverConfig(odeCode=1, dtImplicit=1e100, nTimeStep=1, nTimeStepInternal=args.sa_adjoint_primal_iters,
                         nTimeStepInternalMin=args.sa_adjoint_primal_iters, CFL=50.0, gmresCode=1, nGmresSpace=30, linear_precision="fp32")
    solver = I.ImplicitSolver(vr, ev, cfg)
    solver.run(u)
    uRec = solver.uRec
    d = np.zeros(6)
    d[1] = 1.0
    dTau = torch.zeros(mesh.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, u, 1.0)
    rhs, tmp = torch.zeros_like(u), torch.empty_like(uRec)
    W, C = torch.randn_like(u), torch.randn_like(uRec)

    def timed(fn, n=5):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    t_rhs = timed(lambda: ev.EvaluateRHS(rhs, u, uRec))
    t_vr = timed(lambda: vr.DoReconstructionIter(uRec, tmp, u, putIntoNew=True))
    t_vjp = timed(lambda: ev.EvaluateRHSVJP(W, u, uRec))
    t_vrvjp = timed(lambda: vr.DoReconstructionIterVJP(C, uRec, u))
    t_obj = timed(lambda: ev.WallFluxVJP(d, u, uRec))
    ev.EvaluateRHS(rhs, u, uRec, flags=0, JSource=torch.zeros_like(u))
    J = float(d @ ev.get("fluxWallSum"))
    gU, gR = ev.WallFluxVJP(d, u, uRec)
    out = {"workload": f"SA flat plate, {mesh.n_cell} hex ({nx}x{ny}x{nz}), {args.sa_adjoint_primal_iters} primal BDF1 iterations at "
                       "CFL 50 first; objective: x force of the wall flux (pressure and skin friction)",
           "J": J, "primal_residual_drop": cfg.res_history[-1][2], "ms_rhs": t_rhs, "ms_vr_sweep": t_vr, "ms_rhs_vjp": t_vjp,
           "ms_vr_sweep_vjp": t_vrvjp, "ms_objective_gradient": t_obj, "residual_vjp_over_primal": (t_vjp + t_vrvjp) / (t_rhs + t_vr)}
    # the implicit step's time step: 5 of the median local steps (the stretched wall cells take local steps
    # three orders of magnitude below the largest; with 5 of the largest the system is nearly the steady one,
    # as badly conditioned as the primal defect correction)
    dt = 5.0 * float(dTau.median())
    adj = SteadyAdjoint(vr, ev, u, uRec, cfl=20.0, dt=dt, precision="fp32")
    adj.solve_adjoint(gU, gR, restart=32, max_restarts=1, rtol=1e-10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    info = {}
    psi, lam, hist = adj.solve_adjoint(gU, gR, restart=32, max_restarts=args.sa_adjoint_restarts, rtol=1e-8, info=info)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    out.update({"adjoint_system": f"one implicit step, dt = 5 median local steps = {dt:.3e}", "gmres_iterations": info["arnoldi_steps"],
                "adjoint_drop": hist[-1], "adjoint_s": el, "adjoint_s_per_iteration": el / max(info["arnoldi_steps"], 1)})
    return out


def run_adjoint_cost(args):
    """Cost of the residual VJP against one primal RHS (inviscid bump, the derivative configuration):
    CUDA-event times of EvaluateRHS, EvaluateRHSVJP, one VR sweep and its VJP."""
    import torch
    from dndsr_b200 import mesh as M
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction, euler_bc_dir_weights
    nx, ny, nz = args.adjoint_mesh
    mesh = M.bump_channel_tet(nx, ny, nz, periodic_z=True)
    far = M.freestream(0.8)
    types = np.zeros(7, np.int32)
    vals = np.zeros((7, 5))
    for z in (1, 2, 3, 4):
        types[z], vals[z] = M.BUMP_BC_TYPES[z], far
    out = {}
    for p in (1, 2):
        vr = VariationalReconstruction(mesh, dict(maxOrder=p, intOrder=4, dirWeightScheme="HQM_OPT", geomWeightScheme="HQM_SD",
                                                  geomWeightBias=1.0)).construct(euler_bc_dir_weights(types))
        ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType="Roe", muGas=0.0, ignoreVis=True))
        ev.SetBC(types, vals)
        u = vr.BuildUDof(5)
        u[:] = torch.tensor(far, device="cuda")
        uRec, uNew = vr.BuildURec(5), vr.BuildURec(5)
        dt = torch.zeros(mesh.n_cell, dtype=torch.float64, device="cuda")
        for _ in range(3):
            vr.DoReconstructionIter(uRec, uNew, u, putIntoNew=False)
        ev.EvaluateDt(dt, u, 1.0)
        rhs = torch.zeros_like(u)
        w = torch.randn(u.shape, dtype=torch.float64, device="cuda")
        cot = torch.randn(uRec.shape, dtype=torch.float64, device="cuda")

        def timed(fn, n=10):
            fn()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(n):
                fn()
            b.record()
            torch.cuda.synchronize()
            return a.elapsed_time(b) / n

        t_rhs = timed(lambda: ev.EvaluateRHS(rhs, u, uRec))
        t_vjp = timed(lambda: ev.EvaluateRHSVJP(w, u, uRec))
        t_vr = timed(lambda: vr.DoReconstructionIter(uRec, uNew, u, putIntoNew=True))
        t_vrvjp = timed(lambda: vr.DoReconstructionIterVJP(cot, uRec, u))
        # node-coordinate VJPs (geometry, VR setup and face geometry recomputed per cell in dual numbers)
        t_xr = timed(lambda: ev.EvaluateRHSVJPCoords(w, u, uRec), n=3)
        t_xv = timed(lambda: vr.DoReconstructionIterVJPCoords(cot, uRec, u), n=3)
        t_xb = timed(lambda: ev.ResidualVJPCoords(w, cot, u, uRec), n=3)
        # the limiter step (every cell limited) and the positivity-preserving increment, against one residual
        si = vr.DoCalculateSmoothIndicator(u, uRec)
        uLim = torch.empty_like(uRec)
        t_si = timed(lambda: vr.DoCalculateSmoothIndicator(u, uRec))
        t_lim = timed(lambda: ev.DoLimiterWBAP_C(u, uRec, si, uLim, 0.01, 10.0, True))
        inc = torch.randn(u.shape, dtype=torch.float64, device="cuda") * 1e-2 * u.abs()
        alphaPP, uInc = torch.ones(mesh.n_cell, dtype=torch.float64, device="cuda"), u.clone()
        t_alpha = timed(lambda: ev.EvaluateCellRHSAlpha(u, inc, alphaPP, far[0], 1.0, 0.9))
        t_fix = timed(lambda: ev.AddFixedIncrement(uInc, inc, 1e-6, far[0], 1.0))
        limiter = {"ms_smooth_indicator": t_si, "ms_wbap_limiter_all_cells": t_lim, "ms_cell_rhs_alpha": t_alpha,
                   "ms_add_fixed_increment": t_fix, "limiter_over_residual": (t_si + t_lim) / (t_rhs + t_vr)}
        V = torch.randn((mesh.n_node, 3), dtype=torch.float64, device="cuda") * 1e-3
        a_r = float((ev.EvaluateRHSVJPCoords(w, u, uRec) * V).sum())
        b_r = float((w * ev.EvaluateRHSJVPCoords(V, u, uRec)).sum())
        a_v = float((vr.DoReconstructionIterVJPCoords(cot, uRec, u) * V).sum())
        b_v = float((cot * vr.DoReconstructionIterJVPCoords(V, uRec, u)).sum())
        out[f"p{p}"] = {"ms_rhs": t_rhs, "ms_rhs_vjp": t_vjp, "vjp_over_rhs": t_vjp / t_rhs, "ms_vr_sweep": t_vr, "ms_vr_sweep_vjp": t_vrvjp,
                        "residual_vjp_over_primal": (t_vjp + t_vrvjp) / (t_rhs + t_vr), "ms_rhs_vjp_coords": t_xr,
                        "ms_vr_sweep_vjp_coords": t_xv, "ms_residual_vjp_coords_one_pass": t_xb,
                        "coords_vjp_over_primal": t_xb / (t_rhs + t_vr),
                        "coords_dual_consistency_rhs": abs(a_r - b_r) / max(abs(a_r), 1e-300),
                        "coords_dual_consistency_sweep": abs(a_v - b_v) / max(abs(a_v), 1e-300), **limiter}
        if p == 1:
            out["adjoint_solve_p1"] = adjoint_solve(vr, ev, u, uRec, far, mesh, t_rhs + t_vr)
    out["tgv_viscous"] = tgv_vjp_cost(args)
    return {"workload": f"inviscid bump, {mesh.n_cell} tets, Roe, intOrder 4; VJP with respect to u and uRec (state) and to the node coordinates; "
                        f"tgv_viscous: the TGV workload ({args.n}^3, p={args.p}, HLLE+ and viscous flux)", **out}


def tgv_vjp_cost(args):
    """CUDA-event times of EvaluateRHS and of its VJP (inviscid and viscous parts) on the TGV workload."""
    import torch
    from dndsr_b200 import mesh as M
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    mesh = M.tgv_mesh(args.n)
    vr = VariationalReconstruction(mesh, dict(VR_SETTINGS, maxOrder=args.p)).construct()
    ev = EulerEvaluator(vr, EULER_SETTINGS)
    u, uRec, tmp = vr.BuildUDof(5), vr.BuildURec(5), vr.BuildURec(5)
    ev.InitializeUDOF(u, 3)
    vr.DoReconstructionIter(uRec, tmp, u, putIntoNew=False)
    dt = torch.zeros(mesh.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, 1.0)
    rhs = torch.zeros_like(u)
    w = torch.randn(u.shape, dtype=torch.float64, device="cuda")

    def timed(fn, n=5):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    t_rhs = timed(lambda: ev.EvaluateRHS(rhs, u, uRec))
    t_vjp = timed(lambda: ev.EvaluateRHSVJP(w, u, uRec))
    return {"ms_rhs": t_rhs, "ms_rhs_vjp": t_vjp, "vjp_over_rhs": t_vjp / t_rhs}


def adjoint_solve(vr, ev, u, uRec, far, mesh, ms_primal):
    """Adjoint of the pressure drag on the bump for the coupled (EvaluateRHS, VR sweep) residual of one
    implicit Euler step (dt = 5 local CFL-1 steps) at a smooth non-uniform state: GMRES(32) preconditioned
    by the transposed LU-SGS pair (FP64, then on FP32 vectors) and a 4-term Neumann series of the
    transposed sweep, to a 1e-10 drop."""
    import torch
    from dndsr_b200 import mesh as M
    from dndsr_b200.adjoint import SteadyAdjoint
    X = torch.tensor(mesh.cell_coords().mean(1), device="cuda")
    us = u.clone()
    us[:, 0] *= 1 + 0.05 * torch.sin(3 * X[:, 0]) * torch.cos(2 * X[:, 1])
    us[:, 2] += 0.02 * torch.sin(2 * X[:, 0])
    ur = uRec.clone()
    tmp = torch.empty_like(ur)
    for _ in range(3):
        vr.DoReconstructionIter(ur, tmp, us, putIntoNew=False)
    dTau = torch.zeros(mesh.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dTau, us, 1.0)
    J, gU, gR = ev.PressureForce(M.BUMP_ZONES["bump"], (1.0, 0.0, 0.0), us, ur, grad=True)
    out = {"objective": "pressure drag on the bump", "J": J}
    for prec in ("fp64", "fp32"):
        adj = SteadyAdjoint(vr, ev, us, ur, cfl=5.0, dt=5.0 * float(dTau.max()), precision=prec)
        adj.solve_adjoint(gU, gR, restart=32, max_restarts=1, rtol=1e-10)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = {}
        psi, lam, hist = adj.solve_adjoint(gU, gR, restart=32, max_restarts=40, rtol=1e-10, info=info)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        key = "" if prec == "fp64" else "_fp32_preconditioner"
        out.update({"gmres_iterations" + key: info["arnoldi_steps"], "final_drop" + key: hist[-1], "seconds" + key: el,
                    "solve_over_one_residual" + key: 1e3 * el / ms_primal})
    return out


def n_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count()


def run_reference(args, rank, world):
    """The reference's CPU algorithm (the oracle port, OpenMP on all host cores) on the same workload: the full
    n^3 mesh; each step is one VR sweep + EvaluateRHS, timed individually."""
    if rank != 0:
        return
    import oracle
    from dndsr_b200 import mesh as M
    cores = n_cores()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    m = M.tgv_mesh(args.n)
    vr = dict(maxOrder=args.p, intOrder=5, jacobiRelax=1.0, SORInstead=0, scaleType=1, scaleMultiplier=1.0, dirWeightScheme=1,
              geomWeightScheme=1, geomWeightBias=1.0, geomWeightPower=0.5, bcWeight=1.0)
    es = dict(nVars=5, rsType=oracle.RS["HLLEP"], rsFixScale=1.0, rsIncFScale=1.0, gamma=1.4, Rgas=1.0, muGas=1.0 / 1600, prGas=0.71,
              TRef=273.15, CSutherland=110.4, muModel=0, ignoreVis=0)
    o = oracle.Oracle(m, vr, es)
    o.construct()
    u = o.init_field(3)
    uRec = np.zeros((m.n_cell, o.R, 5))
    o.eval_dt(u, 5.0)
    per_step = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        uRec = o.vr_iter(uRec, u)
        o.eval_rhs(u, uRec)
        el = time.perf_counter() - t0
        if i >= args.warmup:
            per_step.append(el)
    ms = 1e3 * float(np.mean(per_step))
    value = m.n_cell / (ms * 1e-3) / 1e6
    sample = f"oracle port (OpenMP, {cores} threads): VR sweep + EvaluateRHS on the full {args.n}^3 workload, {args.steps} timed steps"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": workload_config(args.n, args.p),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    from dndsr_b200 import mesh as M
    from dndsr_b200.solver import EulerEvaluator, VariationalReconstruction
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    n, p = args.n, args.p
    mesh = M.tgv_mesh(n, seed=0x1234 + rank)
    vr = VariationalReconstruction(mesh, dict(VR_SETTINGS, maxOrder=p)).construct()
    ev = EulerEvaluator(vr, EULER_SETTINGS)
    nc = mesh.n_cell
    u = vr.BuildUDof(5)
    ev.InitializeUDOF(u, 3)
    uRec, uRecNew = vr.BuildURec(5), vr.BuildURec(5)
    rhs = torch.zeros_like(u)
    dt = torch.zeros(nc, dtype=torch.float64, device=dev)
    for _ in range(5):  # converge the reconstruction a little so the RHS sees realistic gradients
        vr.DoReconstructionIter(uRec, uRecNew, u, putIntoNew=False)
    ev.EvaluateDt(dt, u, 5.0)  # spectral radii for the HLLE+ fix (deltaLambdaCell)

    def step(a, b):
        vr.DoReconstructionIter(a, b, u, putIntoNew=True)
        ev.EvaluateRHS(rhs, u, b)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    bufs = [uRec, uRecNew]
    for i in range(args.warmup):
        step(bufs[i % 2], bufs[(i + 1) % 2])
    K = args.steps
    ev_vr = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    ev_rhs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local_rank) as clk:
        start.record()
        for i in range(K):
            a, b = bufs[i % 2], bufs[(i + 1) % 2]
            ev_vr[i][0].record()
            vr.DoReconstructionIter(a, b, u, putIntoNew=True)
            ev_vr[i][1].record()
            ev_rhs[i][0].record()
            ev.EvaluateRHS(rhs, u, b)
            ev_rhs[i][1].record()
        stop.record()
        barrier()
    ms = start.elapsed_time(stop)
    t_vr = float(np.mean([s.elapsed_time(e) for s, e in ev_vr]))
    t_rhs = float(np.mean([s.elapsed_time(e) for s, e in ev_rhs]))
    # end to end through the public API with host buffers: every step copies its inputs u, uRec from
    # pinned host memory and its results rhs, uRecNew back.  The copies of neighbouring steps overlap
    # the computation (copy-in, compute and copy-out streams, two buffer sets), as a caller streaming
    # batches through the library would run it.
    u_h = u.cpu().pin_memory()
    rec_h = bufs[0].cpu().pin_memory()
    nb = 2
    u_d = [torch.empty_like(u) for _ in range(nb)]
    rec_d = [torch.empty_like(uRec) for _ in range(nb)]
    recn_d = [torch.empty_like(uRec) for _ in range(nb)]
    rhs_d = [torch.empty_like(rhs) for _ in range(nb)]
    rhs_h = [torch.empty_like(rhs, device="cpu").pin_memory() for _ in range(nb)]
    recn_h = [torch.empty_like(rec_h).pin_memory() for _ in range(nb)]
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(nb)]
    ev_comp = [torch.cuda.Event() for _ in range(nb)]
    ev_out = [torch.cuda.Event() for _ in range(nb)]

    def copy_in(k):
        b = k % nb
        with torch.cuda.stream(s_in):
            s_in.wait_event(ev_comp[b])  # buffer b's previous step has finished reading its inputs
            u_d[b].copy_(u_h, non_blocking=True)
            rec_d[b].copy_(rec_h, non_blocking=True)
            ev_in[b].record(s_in)

    def compute_and_copy_out(k):
        b = k % nb
        with torch.cuda.stream(s_comp):
            s_comp.wait_event(ev_in[b])
            s_comp.wait_event(ev_out[b])  # buffer b's previous results have been copied out
            vr.DoReconstructionIter(rec_d[b], recn_d[b], u_d[b], putIntoNew=True)
            ev.EvaluateRHS(rhs_d[b], u_d[b], recn_d[b])
            ev_comp[b].record(s_comp)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_comp[b])
            rhs_h[b].copy_(rhs_d[b], non_blocking=True)
            recn_h[b].copy_(recn_d[b], non_blocking=True)
            ev_out[b].record(s_out)

    def e2e_run(n_steps, s2=None, e2=None):
        if s2 is not None:
            s2.record(s_in)
        copy_in(0)
        for k in range(n_steps):
            if k + 1 < n_steps:
                copy_in(k + 1)
            compute_and_copy_out(k)
        if e2 is not None:
            e2.record(s_out)

    e2e_run(max(1, args.warmup))
    barrier()
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_run(K, s2, e2)
    barrier()
    ms_e2e = s2.elapsed_time(e2)
    h2d = u_h.numel() * 8 + rec_h.numel() * 8
    d2h = rhs_h[0].numel() * 8 + recn_h[0].numel() * 8
    if dist:
        t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e = float(t[0]), float(t[1])
    if rank != 0:
        return
    value = world * nc * K / (ms * 1e-3) / 1e6
    e2e = world * nc * K / (ms_e2e * 1e-3) / 1e6
    hbm, src = peaks()
    dom_name, dom_t, dom_b = ("vr_jacobi_sweep", t_vr, B_VR) if t_vr >= t_rhs else ("evaluate_rhs", t_rhs, B_RHS)
    achieved = dom_b * nc / (dom_t * 1e-3) / 1e9
    p64 = fp64_peak_tflops(dev)
    f_dom = (F_VR if dom_name == "vr_jacobi_sweep" else F_RHS).get(p)
    fp64 = None
    if f_dom:
        ach_tf = f_dom * nc / (dom_t * 1e-3) / 1e12
        fp64 = {"falg_per_cell": f_dom, "falg_source": "op-counting build of the oracle (python -m oracle.falg)",
                "achieved_tflops": ach_tf, "peak_tflops": p64, "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                "frac": ach_tf / p64}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": value / REF_PUBLISHED_MCIPS, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(n, p), parallelism=f"replicas{world}" if world > 1 else "single GPU"),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": 3 * K,
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback 6650 GB/s",
                         "traffic": RHS_TRAFFIC_PER_CELL * nc if dom_name == "evaluate_rhs" else None,
                         "traffic_source": "constant copied from the ncu capture of k_rhs_face_fast at 48^3 (profiles/), scaled by cells",
                         "fp64_pipe_pct": RHS_FP64_PIPE_PCT if dom_name == "evaluate_rhs" else None,
                         "fp64_pipe_pct_source": "constant copied from the same 48^3 ncu capture",
                         "algorithmic_bytes_per_cell": dom_b,
                         "fp64": fp64},
            "kernels_ms": {"vr_jacobi_sweep": t_vr, "evaluate_rhs": t_rhs,
                           "vr_GBps": B_VR * nc / (t_vr * 1e-3) / 1e9, "rhs_GBps": B_RHS * nc / (t_rhs * 1e-3) / 1e9},
            "clocks": clk.summary()}
    if world == 1 and not args.no_steady:
        blocks = set(args.blocks.split(","))
        if "time_to_1e-10" in blocks:
            line["time_to_1e-10"] = run_dual_time(args)
        if "steady" in blocks:
            line["steady"] = run_steady(args)
        if "linear_solve" in blocks:
            line["linear_solve"] = run_linear_solve(args)
        if "adjoint_cost" in blocks:
            line["adjoint_cost"] = run_adjoint_cost(args)
        if not args.no_sa and "sa_plate" in blocks:
            line["sa_plate"] = run_sa_plate(args)
    if world == 1 and not args.no_cpu_baseline:
        v, steps, el, cells = cpu_baseline_oracle(args.sample_n, p, args.sample_seconds, n_cores())
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": n_cores(), "kind": "port",
                                "sample": f"oracle port, OpenMP: {steps} steps of VR sweep + EvaluateRHS on TGV {args.sample_n}^3 "
                                          f"({cells} cells, same settings) in {el:.1f} s",
                                "per_operator": {"sample": f"TGV {args.sample_n}^3, median of 5 after 2 warm-ups",
                                                 **cpu_baseline_oracle.per_operator}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--p", type=int, default=2)
    ap.add_argument("--sample-n", type=int, default=32)
    ap.add_argument("--sample-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-steady", action="store_true")
    ap.add_argument("--sa-adjoint-mesh", type=int, nargs=3, default=(120, 80, 8))
    ap.add_argument("--sa-adjoint-primal-iters", type=int, default=300)
    ap.add_argument("--sa-adjoint-restarts", type=int, default=25)
    ap.add_argument("--steady-mesh", type=int, nargs=3, default=(80, 40, 13))
    ap.add_argument("--steady-iters", type=int, default=3000)
    ap.add_argument("--steady-big-mesh", type=int, nargs=3, default=(160, 80, 26))
    ap.add_argument("--steady-big-iters", type=int, default=4000)
    ap.add_argument("--no-steady-roe", dest="steady_roe", action="store_false", help="skip the Roe-Jacobian steady runs")
    ap.add_argument("--linear-mesh", type=int, nargs=3, default=(160, 80, 26))
    ap.add_argument("--adjoint-mesh", type=int, nargs=3, default=(80, 40, 13))
    ap.add_argument("--no-sa", action="store_true")
    # the extra measurement blocks after the headline, comma separated (a subset for profiling runs)
    ap.add_argument("--blocks", default="time_to_1e-10,steady,linear_solve,adjoint_cost,sa_plate")
    ap.add_argument("--sa-mesh", type=int, nargs=3, default=(300, 100, 100))
    ap.add_argument("--sa-iters", type=int, default=30)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
