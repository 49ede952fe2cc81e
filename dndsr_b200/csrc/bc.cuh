// Boundary ghost states (EulerEvaluator_EvaluateDt.hxx:1743-2468 generateBoundaryValue,
// linMode 0, no rotating frame, anchors or CL driver, zero grid velocity) and the
// positivity fallback of reconstructed boundary values (EulerEvaluator.hpp:1541-1625).
#pragma once
#include "solver.cuh"

namespace dndsb
{
// Gas.hpp IdealGasThermalConservative2Primitive / Primitive2Conservative (3 velocity components)
template <int NV, typename T>
DNDSB_HD void bc_cons2prim(const T *U, T *P, real gamma)
{
    P[0] = U[0];
    for (int d = 0; d < 3; d++)
        P[1 + d] = U[1 + d] / U[0];
    T vsqr = P[1] * P[1] + P[2] * P[2] + P[3] * P[3];
    P[4] = (gamma - 1) * (U[4] - 0.5 * U[0] * vsqr);
    for (int j = 5; j < NV; j++)
        P[j] = U[j] / U[0];
}

template <int NV, typename T>
DNDSB_HD void bc_prim2cons(const T *P, T *U, real gamma)
{
    U[0] = P[0];
    for (int d = 0; d < 3; d++)
        U[1 + d] = P[1 + d] * P[0];
    T vsqr = P[1] * P[1] + P[2] * P[2] + P[3] * P[3];
    U[4] = P[4] / (gamma - 1) + 0.5 * P[0] * vsqr;
    for (int j = 5; j < NV; j++)
        U[j] = P[j] * P[0];
}

// ghost state UR of the boundary zone for the inner state UL and outward unit normal n;
// false for a zone without a supported boundary type
// n: real, or dual numbers of the same kind as T for derivatives with respect to the face geometry
template <int NV, typename T, typename TN>
DNDSB_HD bool bc_value(const BoundaryD &b, int zone, const T *UL, const TN *n, T *UR)
{
    if (zone < 0 || zone >= b.nZone)
        return false;
    const int type = b.type[zone];
    const real *far = b.val + zone * 8;
    const real g = b.gamma;
    switch (type)
    {
    case BC_FAR:
    case BC_OUTP:
    {
        // generateBV_FarField: supersonic out / subsonic out (far pressure) / subsonic in
        // (inner pressure) / supersonic in, switched on the normal velocity
        T un = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) / UL[0];
        T vsqr = (UL[1] * UL[1] + UL[2] * UL[2] + UL[3] * UL[3]) / (UL[0] * UL[0]);
        T p, asqr, H;
        gas_thermal(UL[4], UL[0], vsqr, g, p, asqr, H);
        T a = sqrt(asqr);
        if (un - a > 0)
        {
            for (int v = 0; v < NV; v++)
                UR[v] = UL[v];
        }
        else if (un > 0)
        {
            real fp[NV];
            T lp[NV];
            bc_cons2prim<NV>(far, fp, g);
            bc_cons2prim<NV>(UL, lp, g);
            lp[4] = fp[4];
            bc_prim2cons<NV>(lp, UR, g);
        }
        else if (un + a > 0)
        {
            real fp0[NV];
            T fp[NV], lp[NV];
            bc_cons2prim<NV>(far, fp0, g);
            for (int v = 0; v < NV; v++)
                fp[v] = fp0[v];
            bc_cons2prim<NV>(UL, lp, g);
            fp[4] = lp[4];
            bc_prim2cons<NV>(fp, UR, g);
        }
        else
        {
            for (int v = 0; v < NV; v++)
                UR[v] = far[v];
        }
        return true;
    }
    case BC_WALL_INVIS:
    case BC_SYM:
    {
        // generateBV_InviscidWall: momentum mirrored about the face
        for (int v = 0; v < NV; v++)
            UR[v] = UL[v];
        T mn = UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2];
        for (int d = 0; d < 3; d++)
            UR[1 + d] -= 2 * mn * n[d];
        return true;
    }
    case BC_WALL:
    case BC_WALL_ISOTHERMAL:
    {
        // generateBV_ViscousWall: momentum (and the SA variable) reversed; isothermal density
        for (int v = 0; v < NV; v++)
            UR[v] = UL[v];
        for (int d = 0; d < 3; d++)
            UR[1 + d] = -UR[1 + d];
        if (type == BC_WALL_ISOTHERMAL)
        {
            T P[NV];
            bc_cons2prim<NV>(UR, P, g);
            P[0] = P[4] / far[0] / b.Rgas;
            bc_prim2cons<NV>(P, UR, g);
        }
        for (int j = 5; j < NV; j++)
            UR[j] = -UR[j];
        return true;
    }
    case BC_OUT:
        for (int v = 0; v < NV; v++)
            UR[v] = UL[v];
        return true;
    case BC_IN:
        for (int v = 0; v < NV; v++)
            UR[v] = far[v];
        return true;
    }
    return false;
}

// the ghost state at a Gauss point with fixUL (USE_FIX_ZERO_SA_NUT_AT_WALL,
// EulerEvaluator_EvaluateDt.hxx:2291-2296): on wall types the SA variable of both the inner
// state (modified in place) and the ghost is set to zero
template <int NV, typename T, typename TN>
DNDSB_HD bool bc_value_fix(const BoundaryD &b, int zone, T *UL, const TN *n, T *UR)
{
    bool ok = bc_value<NV>(b, zone, UL, n, UR);
    if (ok && NV > 5 && (b.type[zone] == BC_WALL || b.type[zone] == BC_WALL_ISOTHERMAL))
        for (int j = 5; j < NV; j++)
            UL[j] = UR[j] = T(0.0);
    return ok;
}

// CompressRecPart: the cell mean replaces a reconstructed value with rho < 0 or e < 0
template <int NV, typename T>
DNDSB_HD void compress_rec(const T *um, const T *U, T *out)
{
    for (int v = 0; v < NV; v++)
        out[v] = U[v];
    if (out[0] < 0)
        for (int v = 0; v < NV; v++)
            out[v] = um[v];
    T eK = (out[1] * out[1] + out[2] * out[2] + out[3] * out[3]) * 0.5 / (kVerySmall + out[0]);
    if (out[4] - eK < 0)
        for (int v = 0; v < NV; v++)
            out[v] = um[v];
}
} // namespace dndsb
