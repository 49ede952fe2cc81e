"""CPU oracle for the DNDSR implicit residual path -- test infrastructure only.

``oracle/oracle.cpp`` restates the reference's algorithms on the CPU; this
module binds it with ctypes.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg use it, as the checker (or the timed CPU
baseline); the GPU library in ``dndsr_b200/`` never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_CNT_PATH = os.path.join(_HERE, "liboracle_opcount.so")
_lib = None
_cnt = None


def build():
    """Compile oracle/oracle.cpp into oracle/liboracle.so (g++ + OpenMP)."""
    root = os.path.dirname(_HERE)
    subprocess.check_call(["make", "-s", "-f", os.path.join("oracle", "Makefile")], cwd=root)


def _load(path):
    src = os.path.join(_HERE, "oracle.cpp")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        build()
    L = ctypes.CDLL(path)
    _declare(L)
    return L


def lib():
    global _lib
    if _lib is None:
        _lib = _load(_LIB_PATH)
    return _lib


def opcount_lib():
    """The op-counting build (oracle/opcount.hpp): same entry points, every floating-point operation counted."""
    global _cnt
    if _cnt is None:
        _cnt = _load(_CNT_PATH)
        _cnt.orc_opcount_reset.argtypes = []
        _cnt.orc_opcount_get.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
    return _cnt


class VRSettings(ctypes.Structure):
    """Mirror of ``OrcVRSettings`` (field names follow CFV/VRSettings.hpp)."""
    _fields_ = [
        ("maxOrder", ctypes.c_int), ("intOrder", ctypes.c_int),
        ("jacobiRelax", ctypes.c_double), ("SORInstead", ctypes.c_int),
        ("anisotropicLengths", ctypes.c_int), ("scaleType", ctypes.c_int),
        ("scaleMultiplier", ctypes.c_double), ("dirWeightScheme", ctypes.c_int),
        ("manualDirWeights", ctypes.c_double * 4), ("geomWeightScheme", ctypes.c_int),
        ("geomWeightBias", ctypes.c_double), ("geomWeightPower", ctypes.c_double),
        ("geomWeightPower1", ctypes.c_double), ("geomWeightPower2", ctypes.c_double),
        ("bcWeight", ctypes.c_double),
    ]


class EulerSettings(ctypes.Structure):
    """Mirror of ``OrcEulerSettings`` (Euler/EulerEvaluatorSettings.hpp names)."""
    _fields_ = [
        ("nVars", ctypes.c_int), ("rsType", ctypes.c_int),
        ("rsFixScale", ctypes.c_double), ("rsIncFScale", ctypes.c_double),
        ("gamma", ctypes.c_double), ("Rgas", ctypes.c_double), ("muGas", ctypes.c_double),
        ("prGas", ctypes.c_double), ("TRef", ctypes.c_double), ("CSutherland", ctypes.c_double),
        ("muModel", ctypes.c_int), ("ignoreVis", ctypes.c_int), ("rsMeanValueEig", ctypes.c_int),
    ]


_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_long)
_I = ctypes.POINTER(ctypes.c_int)
_V = ctypes.c_void_p


_I64 = ctypes.POINTER(ctypes.c_int64)


def _optional_decls():
    # entry points that the op-counting build leaves out (limiter, positivity, the reference unit-case surfaces of
    # the limiter functions, eigenvectors, compression ratio, local LU and quadrature): name -> argtypes, or
    # (argtypes, restype)
    return {
        "orc_wbap_l2_biway": [ctypes.c_long, _D, _D, ctypes.c_double, _D],
        "orc_wbap_l2_multiway": [ctypes.c_long, ctypes.c_int, _D, ctypes.c_double, _D],
        "orc_pp_compression_ratio": ([_D, _D, ctypes.c_double, ctypes.POINTER(ctypes.c_int)], ctypes.c_double),
        "orc_euler_eigen": [_D, ctypes.c_double, _D, _D],
        "orc_block_ilu0": ([ctypes.c_int64, ctypes.c_int, ctypes.c_int, _I64, _D, _D, _D], ctypes.c_int),
        "orc_block_ilu0_solve": [ctypes.c_int64, ctypes.c_int, ctypes.c_int, _I64, _D, _D, _D, _D],
        "orc_quad_npoints": ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "orc_quad_point": [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D],
        "orc_shape": [ctypes.c_int, _D, _D, _D],
        "orc_smooth_indicator": [_V, _D, _D, _D],
        "orc_limiter_wbap_c": [_V, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double],
        "orc_cell_rhs_alpha": [ctypes.c_long, ctypes.c_int, ctypes.c_double, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_long), _D],
        "orc_cell_rhs_alpha_expansion": [ctypes.c_long, ctypes.c_int, ctypes.c_double, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double],
        "orc_add_fixed_increment": [ctypes.c_long, ctypes.c_int, ctypes.c_double, _D, _D, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, _D],
    }


def _declare(L):
    for name, decl in _optional_decls().items():  # absent from the op-counting build
        if hasattr(L, name):
            fn = getattr(L, name)
            if isinstance(decl, tuple):
                fn.argtypes, fn.restype = decl
            else:
                fn.argtypes = decl
    L.orc_create.restype = _V
    L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, _D, ctypes.c_long, ctypes.c_int, _L, _D,
                             ctypes.c_long, ctypes.c_int, _L, _D, _L, _I, _D, ctypes.c_int, _L,
                             ctypes.POINTER(VRSettings), ctypes.POINTER(EulerSettings)]
    L.orc_destroy.argtypes = [_V]
    L.orc_construct.restype = ctypes.c_int
    L.orc_construct.argtypes = [_V, _D, ctypes.c_int]
    L.orc_sizes.argtypes = [_V, _L]
    L.orc_get.restype = ctypes.c_long
    L.orc_get.argtypes = [_V, ctypes.c_char_p, _D]
    L.orc_set_delta_lambda.argtypes = [_V, _D]
    L.orc_set_bc.argtypes = [_V, ctypes.c_int, _I, _D, ctypes.c_int]
    L.orc_set_wall_dist.argtypes = [_V, _D]
    L.orc_init_field.argtypes = [_V, ctypes.c_int, ctypes.c_double, _D]
    L.orc_vr_iter.argtypes = [_V, _D, _D, _D, ctypes.c_int, ctypes.c_int]
    L.orc_eval_dt.argtypes = [_V, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int, _D, _D]
    L.orc_eval_rhs.argtypes = [_V, _D, _D, _D, _D]
    L.orc_eval_rhs_full.argtypes = [_V, _D, _D, _D, _D, _D, _D, _D]
    L.orc_lusgs_init.argtypes = [_V, _D, ctypes.c_double, ctypes.c_double, _D]
    L.orc_set_jacobian_mode.argtypes = [_V, ctypes.c_int]
    L.orc_vr_iter_sor.argtypes = [_V, _D, _D]
    L.orc_jacobian_lu.argtypes = [_V, ctypes.c_double, _D, _D]
    L.orc_jacobian_lu.restype = ctypes.c_int
    L.orc_solve_jacobian_lu.argtypes = [_V, ctypes.c_double, _D, _D, _D, _D, _D, ctypes.c_int, _D]
    L.orc_roe_fdiff.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]
    L.orc_lusgs_init_block.argtypes = [_V, _D, ctypes.c_double, ctypes.c_double, _D, _D]
    L.orc_lusgs_init_block.restype = ctypes.c_int
    L.orc_update_sgs.argtypes = [_V, ctypes.c_double, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]
    L.orc_update_lusgs.argtypes = [_V, ctypes.c_double, _D, _D, _D, _D, _D, ctypes.c_int]
    L.orc_lusgs_matvec.argtypes = [_V, ctypes.c_double, _D, _D, _D, _D]
    L.orc_lusgs_matvec_t.argtypes = [_V, ctypes.c_double, _D, _D, _D, _D]
    L.orc_update_sgs_t.argtypes = [_V, ctypes.c_double, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int]
    L.orc_pressure_force.argtypes = [_V, ctypes.c_int, _D, _D, _D, _D, _D]
    L.orc_pressure_force.restype = ctypes.c_double
    L.orc_riemann.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, _D, _D]
    L.orc_viscous_flux.argtypes = [_D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, _D]
    L.orc_cell_point_values.argtypes = [_V, _D, _D, _D]
    L.orc_cell_quad_weights.argtypes = [_V, _D]


def _p(a, t=_D):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# Riemann solver codes: Euler/Gas.hpp:61-96
RS = dict(Roe=1, HLLC=2, HLLEP=3, HLLEP_V1=21, Roe_M1=11, Roe_M2=12, Roe_M3=13, Roe_M4=14,
          Roe_M5=15, Roe_M6=16, Roe_M7=17, Roe_M8=18)


def riemann(rs, UL, UR, n, gamma=1.4, ULm=None, URm=None, dLambda=0.0, fixScale=0.0, incFScale=0.0):
    """One call of the reference's InviscidFlux_IdealGas_Dispatcher (Gas.hpp:1434)."""
    UL, UR, n = _f64(UL), _f64(UR), _f64(n)
    ULm = UL if ULm is None else _f64(ULm)
    URm = UR if URm is None else _f64(URm)
    F = np.zeros(5)
    lam = np.zeros(3)
    code = RS[rs] if isinstance(rs, str) else int(rs)
    lib().orc_riemann(code, _p(UL), _p(UR), _p(ULm), _p(URm), _p(n), gamma, dLambda, fixScale, incFScale, _p(F), _p(lam))
    return F, lam


def euler_eigen(U, gamma=1.4):
    """(R, L): the right and left eigenvectors of the Euler flux Jacobian at the conservative state U (x direction)."""
    R, L = np.zeros((5, 5)), np.zeros((5, 5))
    lib().orc_euler_eigen(_p(_f64(U)), float(gamma), _p(R), _p(L))
    return R, L


def pp_compression_ratio(u, inc, newRhoE=0.0):
    """Gas.hpp IdealGasGetCompressionRatioPressure (scheme 0): the largest alpha in [0, 1) keeping rhoE(u + alpha inc)
    above newRhoE; returns (alpha, bad)."""
    bad = ctypes.c_int(0)
    a = lib().orc_pp_compression_ratio(_p(_f64(u)), _p(_f64(inc)), float(newRhoE), ctypes.byref(bad))
    return a, bool(bad.value)


def wbap_l2_biway(u1, u2, n=1.0):
    """Limiters.hpp FWBAP_L2_Biway entry by entry (the limiter function of the oracle's WBAP_C)."""
    u1, u2 = _f64(u1), _f64(u2)
    out = np.zeros_like(u1)
    lib().orc_wbap_l2_biway(u1.size, _p(u1), _p(u2), float(n), _p(out))
    return out


def wbap_l2_multiway(others, n1=1.0):
    """Limiters.hpp FWBAP_L2_Multiway entry by entry; others [nOther][...] with the cell's own values first."""
    o = _f64(others)
    out = np.zeros(o.shape[1:])
    lib().orc_wbap_l2_multiway(int(np.prod(o.shape[1:])), o.shape[0], _p(o), float(n1), _p(out))
    return out


QUAD_ELEM = dict(line=0, tri=1, quad=2, tet=3, hex=4)


def quad_rule(elem, order):
    """The oracle's quadrature rule (QuadratureHub.hpp:39-380) for an element kind of QUAD_ELEM and an integration
    order on the reference element: points [n][3] and weights [n]."""
    e = QUAD_ELEM[elem]
    n = lib().orc_quad_npoints(e, order)
    pts, w = np.zeros((n, 3)), np.zeros(n)
    for i in range(n):
        lib().orc_quad_point(e, order, i, _p(pts[i]), _p(w[i:i + 1]))
    return pts, w


def shape(elem, p):
    """The oracle's shape functions (Geom/Elements/*.hpp) of an element kind of QUAD_ELEM at a parametric point:
    N [nNode], dN [3][nNode]."""
    nn = dict(line=2, tri=3, quad=4, tet=4, hex=8)[elem]
    N, dN = np.zeros(8), np.zeros((3, 8))
    lib().orc_shape(QUAD_ELEM[elem], _p(_f64(np.asarray(p, float).reshape(3))), _p(N), _p(dN))
    return N[:nn], dN[:, :nn]


def block_ilu0(nbr, off, diag):
    """Block ILU(0) in natural order on a general neighbour table (JacobianLocalLU::InPlaceDecompose with
    iluCode 0, Solver/Direct.hpp:312-405).  nbr [n][K] (-1: none), off [n][K][bs][bs] the blocks A_(i, nbr[i][k]),
    diag [n][bs][bs].  Returns (factors [n][K][bs][bs]: L for lower neighbours, U for upper; dinv [n][bs][bs])."""
    nbr = np.ascontiguousarray(nbr, dtype=np.int64)
    n, K = nbr.shape
    bs = np.asarray(diag).shape[-1]
    f = _f64(off).reshape(n, K, bs, bs).copy()
    d = _f64(diag).reshape(n, bs, bs)
    dinv = np.zeros_like(d)
    if lib().orc_block_ilu0(n, bs, K, _p(nbr, ctypes.POINTER(ctypes.c_int64)), _p(f), _p(d), _p(dinv)) != 0:
        raise ValueError("block_ilu0: singular pivot or block size above 8")
    return f, dinv


def block_ilu0_solve(nbr, factors, dinv, b):
    """x = (L U)^-1 b with the factors of block_ilu0 (JacobianLocalLU::Solve, Solver/Direct.hpp:487-540)."""
    nbr = np.ascontiguousarray(nbr, dtype=np.int64)
    n, K = nbr.shape
    bs = np.asarray(dinv).shape[-1]
    b = _f64(b).reshape(n, bs)
    x = np.zeros_like(b)
    lib().orc_block_ilu0_solve(n, bs, K, _p(nbr, ctypes.POINTER(ctypes.c_int64)), _p(_f64(factors)), _p(_f64(dinv)), _p(b), _p(x))
    return x


def roe_fdiff_matrix(U, UOther, n, lam, gamma=1.4):
    """The matrix of RoeFluxIncFDiff (Gas.hpp:1149-1243) at the Roe average of (U, UOther) with the eigenvalues
    lam = (l0, l123, l4): column i is the dissipation of the unit jump e_i."""
    U, UOther, n = _f64(U), _f64(UOther), _f64(n)
    nv = len(U)
    M = np.zeros((nv, nv))
    for i in range(nv):
        e = np.zeros(nv)
        e[i] = 1.0
        col = np.zeros(nv)
        lib().orc_roe_fdiff(nv, gamma, _p(U), _p(UOther), _p(n), _p(e), float(lam[0]), float(lam[1]), float(lam[2]), _p(col))
        M[:, i] = col
    return M


def cell_rhs_alpha(u, res, refRho, refP, gamma=1.4, relax=0.9, compress=2, compressPower=1.0, ppEpsIsRelaxed=False, flag=0):
    """EvaluateCellRHSAlpha (EulerEvaluator.hxx:1938-2062): (alpha per cell, nLim, alphaMin, assertion_failed)."""
    u, res = _f64(u), _f64(res)
    alpha = np.zeros(u.shape[0])
    n = ctypes.c_long()
    amin = np.zeros(1)
    bad = lib().orc_cell_rhs_alpha(u.shape[0], u.shape[1], gamma, _p(u), _p(res), _p(alpha), refRho, refP, relax, int(compress),
                                   compressPower, int(ppEpsIsRelaxed), int(flag), ctypes.byref(n), _p(amin))
    return alpha, int(n.value), float(amin[0]), bool(bad)


def cell_rhs_alpha_expansion(u, res, alpha, refRho, refP, alphaMin, gamma=1.4):
    """EvaluateCellRHSAlphaExpansion (EulerEvaluator.hxx:2064-2140) on a copy of alpha."""
    u, res = _f64(u), _f64(res)
    a = _f64(alpha).copy()
    lib().orc_cell_rhs_alpha_expansion(u.shape[0], u.shape[1], gamma, _p(u), _p(res), _p(a), refRho, refP, alphaMin)
    return a


def add_fixed_increment(u, inc, alpha, refRho, refP, gamma=1.4, ppEpsIsRelaxed=False):
    """AddFixedIncrement (EulerEvaluator.hpp:1795-1857) on a copy of u: (u_new, alpha_fix_min, assertion_failed)."""
    un, inc = _f64(u).copy(), _f64(inc)
    amin = np.zeros(1)
    bad = lib().orc_add_fixed_increment(un.shape[0], un.shape[1], gamma, _p(un), _p(inc), float(alpha), refRho, refP,
                                        int(ppEpsIsRelaxed), _p(amin))
    return un, float(amin[0]), bool(bad)


def viscous_flux(U, gradU, n, gamma, mu, k, Cp, adiabatic=False):
    U, gradU, n = _f64(U), _f64(gradU), _f64(n)
    F = np.zeros(5)
    lib().orc_viscous_flux(_p(U), _p(gradU), _p(n), gamma, mu, k, Cp, int(adiabatic), _p(F))
    return F


class Oracle:
    """One mesh + VR + evaluator instance of the CPU restatement."""

    def __init__(self, mesh, vr: dict, euler: dict, opcount=False):
        """opcount: run on the op-counting build (oracle/opcount.hpp), single-threaded; see op_counts()."""
        self.mesh = mesh
        L = opcount_lib() if opcount else lib()
        self.L = L
        a = mesh.arrays()
        self._keep = a
        vs = VRSettings()
        for k, v in vr.items():
            if k == "manualDirWeights":
                for i, x in enumerate(v):
                    vs.manualDirWeights[i] = x
            else:
                setattr(vs, k, v)
        es = EulerSettings()
        for k, v in euler.items():
            setattr(es, k, v)
        self.vs, self.es = vs, es
        ctype = {1: 1, 2: 2, 3: 3, 4: 4}[mesh.cell_type]
        nf = mesh.cell2face.shape[1]
        self.nf = nf
        self.h = L.orc_create(mesh.dim, ctype, mesh.face_type, mesh.n_node, _p(a["coords"]), mesh.n_cell,
                              a["cell2node"].shape[1], _p(a["cell2node"], _L), _p(a["cell_shift"]), mesh.n_face,
                              a["face2node"].shape[1], _p(a["face2node"], _L), _p(a["face_shift"]), _p(a["face2cell"], _L),
                              _p(a["face_zone"], _I), _p(a["face_pshift"]), nf, _p(a["cell2face"], _L),
                              ctypes.byref(vs), ctypes.byref(es))
        self.nv = es.nVars

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def op_counts(self, reset=False):
        """Operations counted by the op-counting build since the last reset:
        dict(add, mul, div, sqrt, fn) (fn: exp / pow / log / trigonometric calls)."""
        out = np.zeros(5, dtype=np.uint64)
        self.L.orc_opcount_get(out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        if reset:
            self.L.orc_opcount_reset()
        return dict(zip(("add", "mul", "div", "sqrt", "fn"), [int(x) for x in out]))

    def construct(self, bc_dir_weight=None):
        if bc_dir_weight is None:
            bad = self.L.orc_construct(self.h, None, 0)
        else:
            w = _f64(bc_dir_weight)
            bad = self.L.orc_construct(self.h, _p(w), w.shape[0])
        out = np.zeros(4, dtype=np.int64)
        self.L.orc_sizes(self.h, _p(out, _L))
        self.NDOF, self.R, self.nGf, self.nGc = [int(x) for x in out]
        return bad

    def get(self, name):
        n = self.L.orc_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        self.L.orc_get(self.h, name.encode(), _p(out))
        return out

    def set_bc(self, types, values):
        """Boundary table per face zone (index = zone id, zone 0 interior): EulerBC.hpp type codes
        and the far-field / inflow state (or wall temperature) of each zone."""
        t = np.ascontiguousarray(types, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(len(t), self.nv)
        self._bc = (t, v)
        self.L.orc_set_bc(self.h, len(t), t.ctypes.data_as(_I), _p(v), self.nv)

    def set_wall_distance(self, d):
        """Wall distance at every cell Gauss point, [nCell][nGc] (the SA model's dWall)."""
        d = np.ascontiguousarray(d, dtype=np.float64)
        self._dwall = d
        self.L.orc_set_wall_dist(self.h, _p(d))

    def init_field(self, kind, chi=5.0):
        u = np.zeros((self.mesh.n_cell, self.nv))
        self.L.orc_init_field(self.h, kind, chi, _p(u))
        return u

    def vr_iter(self, uRec, u, recordInc=False, uRecIsZero=False):
        uRec, u = _f64(uRec), _f64(u)
        out = np.zeros_like(uRec)
        self.L.orc_vr_iter(self.h, _p(uRec), _p(out), _p(u), int(recordInc), int(uRecIsZero))
        return out

    def vr_iter_sor(self, uRec, u):
        """One SOR sweep (SORInstead) from uRec, in natural cell order; returns the new uRec."""
        out = np.array(uRec, dtype=np.float64, copy=True, order="C")
        self.L.orc_vr_iter_sor(self.h, _p(out), _p(_f64(u)))
        return out

    def eval_dt(self, u, CFL, MaxDt=1e100, useLocalDt=True):
        u = _f64(u)
        dt = np.zeros(self.mesh.n_cell)
        mn = np.zeros(1)
        self.L.orc_eval_dt(self.h, _p(u), CFL, MaxDt, int(useLocalDt), _p(dt), _p(mn))
        return dt, float(mn[0])

    def set_delta_lambda(self, dl):
        dl = _f64(dl)
        self.L.orc_set_delta_lambda(self.h, _p(dl))

    def eval_rhs(self, u, uRec, want_face_flux=False):
        u, uRec = _f64(u), _f64(uRec)
        rhs = np.zeros_like(u)
        ff = np.zeros((self.mesh.n_face, self.nv)) if want_face_flux else None
        self.L.orc_eval_rhs(self.h, _p(u), _p(uRec), _p(rhs), _p(ff) if ff is not None else None)
        return (rhs, ff) if want_face_flux else rhs

    def eval_rhs_full(self, u, uRecUnlim, uRec, alpha=None):
        """EvaluateRHS(rhs, JSource, u, uRecUnlim, uRec, uRecBeta, cellRHSAlpha, ...): face values from uRec,
        gradients from uRecUnlim, SA source scaled by alpha.  Returns (rhs, JSource [nCell][nv], fluxWallSum [nv])."""
        u, uU, uR = _f64(u), _f64(uRecUnlim), _f64(uRec)
        rhs = np.zeros_like(u)
        js = np.zeros_like(u)
        fw = np.zeros(self.nv)
        a = _f64(alpha) if alpha is not None else None
        self.L.orc_eval_rhs_full(self.h, _p(u), _p(uU), _p(uR), _p(a) if a is not None else None, _p(rhs), _p(js), _p(fw))
        return rhs, js, fw

    def lusgs_init(self, dTau, dt, alphaDiag):
        dTau = _f64(dTau)
        jd = np.zeros(self.mesh.n_cell * (self.nv if self.nv >= 6 else 1))
        self.L.orc_lusgs_init(self.h, _p(dTau), dt, alphaDiag, _p(jd))
        return jd if self.nv < 6 else jd.reshape(self.mesh.n_cell, self.nv)

    def set_jacobian_mode(self, useScalarJacobian=True, useRoeJacobian=False):
        """EulerEvaluatorSettings useScalarJacobian / useRoeJacobian (EulerEvaluatorSettings.hpp:53-54, exclusive).
        Block modes take the jdiag of lusgs_init_block in every LU-SGS operator; useRoeJacobian also makes
        eval_rhs record the face eigenvalues lambdaFace0 / 123 / 4."""
        if useScalarJacobian and useRoeJacobian:
            raise ValueError("useScalarJacobian and useRoeJacobian are mutually exclusive")
        self.L.orc_set_jacobian_mode(self.h, 2 if useRoeJacobian else (0 if useScalarJacobian else 1))

    def lusgs_init_block(self, dTau, dt, alphaDiag, u):
        """LUSGSMatrixInit in block mode: [nCell][2][nv][nv], the block and its inverse."""
        dTau, u = _f64(dTau), _f64(u)
        jd = np.zeros((self.mesh.n_cell, 2, self.nv, self.nv))
        if self.L.orc_lusgs_init_block(self.h, _p(dTau), dt, alphaDiag, _p(u), _p(jd)) != 0:
            raise FloatingPointError("singular diagonal block")
        return jd

    def jacobian_lu(self, alphaDiag, u, jdiag):
        """LUSGSMatrixToJacobianLU + InPlaceDecompose (iluCode 0, natural ordering), kept inside the oracle."""
        if self.L.orc_jacobian_lu(self.h, alphaDiag, _p(_f64(u)), _p(_f64(jdiag))) != 0:
            raise FloatingPointError("singular pivot block")

    def solve_jacobian_lu(self, alphaDiag, rhs, u, uInc, jdiag, uIncIsZero=False):
        """LUSGSMatrixSolveJacobianLU: returns (uIncNew, sumInc)."""
        rhs, u, uInc, jdiag = _f64(rhs), _f64(u), _f64(uInc), _f64(jdiag)
        out = np.zeros_like(rhs)
        s = np.zeros(self.nv)
        self.L.orc_solve_jacobian_lu(self.h, alphaDiag, _p(rhs), _p(u), _p(uInc), _p(out), _p(jdiag), int(uIncIsZero), _p(s))
        return out, s

    def update_sgs(self, alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward, gsUpdate=True, uIncIsZero=False):
        rhs, u, uInc, jdiag = _f64(rhs), _f64(u), _f64(uInc), _f64(jdiag)
        out = np.array(uIncNew, dtype=np.float64, copy=True, order="C")
        s = np.zeros(self.nv)
        self.L.orc_update_sgs(self.h, alphaDiag, _p(rhs), _p(u), _p(uInc), _p(out), _p(jdiag), int(forward), int(gsUpdate),
                             int(uIncIsZero), _p(s))
        return out, s

    def update_lusgs(self, alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward, inplace=False):
        """UpdateLUSGSForward / UpdateLUSGSBackward (EulerEvaluator.hxx:376-529) on a copy of uIncNew.
        inplace: uInc is the same array as uIncNew (the copy), as the reference's callers pass it."""
        rhs, u, jdiag = _f64(rhs), _f64(u), _f64(jdiag)
        out = np.array(uIncNew, dtype=np.float64, copy=True, order="C")
        src = out if inplace else _f64(uInc)
        self.L.orc_update_lusgs(self.h, alphaDiag, _p(rhs), _p(u), _p(src), _p(out), _p(jdiag), int(forward))
        return out

    def lusgs_matvec(self, alphaDiag, u, uInc, jdiag):
        u, uInc, jdiag = _f64(u), _f64(uInc), _f64(jdiag)
        out = np.zeros_like(uInc)
        self.L.orc_lusgs_matvec(self.h, alphaDiag, _p(u), _p(uInc), _p(jdiag), _p(out))
        return out

    def lusgs_matvec_t(self, alphaDiag, u, y, jdiag):
        """Transpose of lusgs_matvec applied to y."""
        u, y, jdiag = _f64(u), _f64(y), _f64(jdiag)
        out = np.zeros_like(y)
        self.L.orc_lusgs_matvec_t(self.h, alphaDiag, _p(u), _p(y), _p(jdiag), _p(out))
        return out

    def update_sgs_t(self, alphaDiag, b, u, y, yNew, jdiag, forward, gsUpdate=True):
        """One Gauss-Seidel sweep on the transposed LU-SGS system, natural cell order."""
        b, u, y, jdiag = _f64(b), _f64(u), _f64(y), _f64(jdiag)
        out = np.array(yNew, dtype=np.float64, copy=True, order="C")
        self.L.orc_update_sgs_t(self.h, alphaDiag, _p(b), _p(u), _p(y), _p(out), _p(jdiag), int(forward), int(gsUpdate))
        return out

    def pressure_force(self, zone, direction, u, uRec, grad=False):
        """Pressure force along direction on boundary zone; with grad, also (dJ/du, dJ/duRec)."""
        u, uRec = _f64(u), _f64(uRec)
        d = _f64(np.asarray(direction, dtype=np.float64))
        gU = np.zeros_like(u) if grad else None
        gR = np.zeros_like(uRec) if grad else None
        J = self.L.orc_pressure_force(self.h, int(zone), _p(d), _p(u), _p(uRec), _p(gU) if grad else None, _p(gR) if grad else None)
        return (J, gU, gR) if grad else J

    def smooth_indicator(self, u, uRec):
        """DoCalculateSmoothIndicator (procedure 0, density and energy), one value per cell."""
        u, uRec = _f64(u), _f64(uRec)
        si = np.zeros(self.mesh.n_cell)
        self.L.orc_smooth_indicator(self.h, _p(u), _p(uRec), _p(si))
        return si

    def limiter_wbap_c(self, u, uRec, si, smoothThreshold=0.01, WBAP_nStd=10.0, ifAll=False, gamma=1.4):
        """DoLimiterWBAP_C (WBAP-L2 biway and multiway, characteristic variables): the limited uRec."""
        u, uRec, si = _f64(u), _f64(uRec), _f64(si)
        out = np.zeros_like(uRec)
        bad = self.L.orc_limiter_wbap_c(self.h, _p(u), _p(uRec), _p(si), _p(out), smoothThreshold, WBAP_nStd, int(ifAll), gamma)
        assert bad == 0, "singular derivative basis at a face centre"
        return out

    def cell_point_values(self, u, uRec):
        u, uRec = _f64(u), _f64(uRec)
        out = np.zeros((self.mesh.n_cell, self.nGc, self.nv))
        self.L.orc_cell_point_values(self.h, _p(u), _p(uRec), _p(out))
        return out

    def cell_quad_weights(self):
        w = np.zeros(self.nGc)
        self.L.orc_cell_quad_weights(self.h, _p(w))
        return w
