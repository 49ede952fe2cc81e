// Block-diagonal and Roe-linearised LU-SGS operators (EulerEvaluatorSettings useScalarJacobian = false,
// useRoeJacobian): the block branch of LUSGSMatrixInit (EulerEvaluator.hxx:37-159), the Roe form of the
// flux increment (EulerEvaluator.hpp:1100-1180 fluxJacobian0_Right_Times_du(_AsMatrix) with useRoeTerm,
// Gas.hpp:1149-1243 GetRoeAverage / RoeFluxIncFDiff), the linearised ghost states (generateBoundaryValue
// with linMode 1, EulerEvaluator_EvaluateDt.hxx:1743-1835, 2199-2270) and the block inverse
// (JacobianDiagBlock::GetInvert, EulerJacobian.hpp:150-180).
//
// Modes (EvalD::jacMode): 0 scalar diagonal (useScalarJacobian), 1 block diagonal without the Roe term
// (equal to the scalar operator, stored as blocks), 2 block diagonal with the Roe term.  A block jdiag is
// [nCell][2][NV][NV]: the row-major block and its inverse.
#pragma once
#include "solver.cuh"
#include "bc.cuh"

namespace dndsb
{
namespace roej
{
// A(U; n) dU of the inviscid flux (Gas.hpp:462-513 IdealGasUIncrement + GasInviscidFluxFacialIncrement)
template <int NV>
DNDSB_HD void flux_inc(const real *U, const real *n, const real *dU, real gamma, real *dF)
{
    real ir = 1.0 / U[0];
    real v[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
    real p, a2, H;
    gas_thermal(U[4], U[0], dot3(v, v), gamma, p, a2, H);
    real dv[3];
    for (int d = 0; d < 3; d++)
        dv[d] = (dU[1 + d] - U[1 + d] * ir * dU[0]) * ir;
    real dp = (gamma - 1) * (dU[4] - 0.5 * (dU[1] * v[0] + dU[2] * v[1] + dU[3] * v[2] + U[1] * dv[0] + U[2] * dv[1] + U[3] * dv[2]));
    real vn = dot3(v, n), dvn = dot3(dv, n);
    dF[0] = dU[1] * n[0] + dU[2] * n[1] + dU[3] * n[2];
    for (int d = 0; d < 3; d++)
        dF[1 + d] = dU[1 + d] * vn + U[1 + d] * dvn + n[d] * dp;
    dF[4] = (dU[4] + dp) * vn + (U[4] + p) * dvn;
    for (int j = 5; j < NV; j++)
        dF[j] = dU[j] * vn + U[j] * dvn;
}

// dF += RoeFluxIncFDiff(dU; n, r, l0, l123, l4): the Roe dissipation of the jump dU, passive scalars with l123
template <int NV>
DNDSB_HD void roe_fdiff_add(const real *dU, const real *n, const RoeAvg &r, real gamma, real l0, real l123, real l4, real *dF)
{
    RoeWavesT<real> w;
    roe_waves(dU, n, r, gamma, w);
    real d[5];
    roe_dissipation(w, n, r, l0, l123, l4, d);
    for (int i = 0; i < 5; i++)
        dF[i] += d[i];
    for (int j = 5; j < NV; j++)
        dF[j] += dU[j] * l123;
}

// the eigenvalues of face f seen from the cell on side `side` (lambda0 and lambda4 swap with the normal)
struct FaceLam
{
    real l0, l123, l4, vis, main;
};
DNDSB_HD FaceLam face_lam(const EvalD &ev, int64_t f, int side)
{
    FaceLam L;
    L.l0 = side ? ev.lambdaFace4[f] : ev.lambdaFace0[f];
    L.l4 = side ? ev.lambdaFace0[f] : ev.lambdaFace4[f];
    L.l123 = ev.lambdaFace123[f];
    L.vis = ev.lambdaFaceVis[f];
    L.main = ev.lambdaFace[f];
    return L;
}

// the flux increment of neighbour state Uo seen from cell state Uc through n (outward from the cell):
// roe: A(Uo) dU - RoeDiff(dU; Roe(Uo, Uc)) - lambdaVis dU (fluxJacobian0_Right_Times_du, incFsign -1);
// otherwise the scalar form A(Uo) dU - lambdaFace dU
template <int NV>
DNDSB_HD void nbr_inc(bool roe, const real *Uo, const real *Uc, const real *n, const real *dU, const FaceLam &L, real gamma, real *dF)
{
    flux_inc<NV>(Uo, n, dU, gamma, dF);
    if (roe)
    {
        RoeAvg r;
        roe_average(Uo, Uc, gamma, r);
        roe_fdiff_add<NV>(dU, n, r, gamma, -L.l0, -L.l123, -L.l4, dF);
        for (int j = 0; j < NV; j++)
            dF[j] -= L.vis * dU[j];
    }
    else
        for (int j = 0; j < NV; j++)
            dF[j] -= L.main * dU[j];
}

// generateBoundaryValue(e_i, ..., linMode = 1) as a matrix: zero for far-field, outflow and inflow types;
// the momentum mirrored for slip walls and symmetry; reversed for no-slip walls.  Column-major.
template <int NV>
DNDSB_HD void bc_linear(int type, const real *n, real *J)
{
    for (int i = 0; i < NV * NV; i++)
        J[i] = 0;
    if (type == BC_WALL_INVIS || type == BC_SYM)
    {
        for (int i = 0; i < NV; i++)
            J[i * NV + i] = 1;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                J[(1 + b) * NV + 1 + a] -= 2 * n[a] * n[b];
    }
    else if (type == BC_WALL || type == BC_WALL_ISOTHERMAL)
        for (int i = 0; i < NV; i++)
            J[i * NV + i] = (i >= 1 && i <= 3) ? -1 : 1;
}

// the diagonal block of cell c (row-major B), LUSGSMatrixInit's block branch:
// roe: sum over faces of w (RoeDiff(.; Roe(u_c, u_j), +l) + lambdaVis I) (omitF, incFsign +1), boundary faces
//      also w (A(u_g) - RoeDiff(.; Roe(u_g, u_c)) - lambdaVis I) dGhost/du_c with the ghost u_g of u_c;
//      then 1/dTau + 1/dt on the diagonal;
// otherwise the scalar diagonal 1/dTau + 1/dt + sum_f w lambdaFace;
// both: + alphaDiag JSource (the SA source Jacobian diagonal).  w = (alphaDiag / 2) A_f / V_c.
template <int NV>
DNDSB_HD void cell_block(const MeshD &m, const GeomD &g, const BoundaryD &bnd, const EvalD &ev, bool roe, const real *dTau, real dt,
                         real alphaDiag, const real *u, int64_t c, real *B)
{
    const real gamma = ev.s.gamma;
    for (int i = 0; i < NV * NV; i++)
        B[i] = 0;
    const real *uc = u + c * NV;
    real fp = 1.0 / dTau[c] + 1.0 / dt;
    const real iv = 1.0 / g.vol[c];
    for (int k = 0; k < m.nf; k++)
    {
        int pk = m.cell2face[c * m.nf + k];
        int64_t f = pk >> 1;
        int side = pk & 1;
        fp += (0.5 * alphaDiag) * g.faceArea[f] * ev.lambdaFace[f] * iv;
        if (!roe)
            continue;
        real sg = side ? -1.0 : 1.0;
        real n[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
        int o = m.cellNbr[c * m.nf + k];
        bool isBnd = o < 0;
        real uj[NV];
        int zone = m.faceZone[f];
        if (isBnd)
        {
            if (!bc_value<NV>(bnd, zone, uc, n, uj))
                for (int v = 0; v < NV; v++)
                    uj[v] = uc[v];
        }
        else
            for (int v = 0; v < NV; v++)
                uj[v] = u[(int64_t)o * NV + v];
        FaceLam L = face_lam(ev, f, side);
        real w = (0.5 * alphaDiag) * g.faceArea[f] * iv;
        RoeAvg r;
        roe_average(uc, uj, gamma, r);
        real JBC[NV * NV];
        int bt = (isBnd && zone >= 0 && zone < bnd.nZone) ? bnd.type[zone] : 0;
        if (isBnd)
            bc_linear<NV>(bt, n, JBC);
        for (int i = 0; i < NV; i++)
        {
            real e[NV], col[NV];
            for (int v = 0; v < NV; v++)
                e[v] = v == i ? 1.0 : 0.0, col[v] = 0;
            roe_fdiff_add<NV>(e, n, r, gamma, L.l0, L.l123, L.l4, col);
            for (int v = 0; v < NV; v++)
                B[v * NV + i] += w * (col[v] + (v == i ? L.vis : 0.0));
        }
        if (isBnd)
        {
            // columns of (A(u_g) - RoeDiff - lambdaVis I) JBC: apply to the columns of JBC
            for (int i = 0; i < NV; i++)
            {
                real dcol[NV], col[NV];
                bool zero = true;
                for (int v = 0; v < NV; v++)
                    dcol[v] = JBC[i * NV + v], zero = zero && dcol[v] == 0;
                if (zero)
                    continue;
                nbr_inc<NV>(true, uj, uc, n, dcol, L, gamma, col);
                for (int v = 0; v < NV; v++)
                    B[v * NV + i] += w * col[v];
            }
        }
    }
    for (int i = 0; i < NV; i++)
    {
        if (roe)
            B[i * NV + i] += 1.0 / dTau[c] + 1.0 / dt;
        else
            B[i * NV + i] = fp;
        if (NV >= 6 && ev.jSource)
            B[i * NV + i] += alphaDiag * ev.jSource[c * NV + i];
    }
}

// inverse of a row-major block: rows scaled by the inverse diagonal, Gauss-Jordan with partial pivoting,
// columns scaled back (the reference pivots fully; both are exact up to rounding for these blocks).
// False for a zero diagonal entry or a zero pivot.
template <int NV>
DNDSB_HD bool block_inv(const real *A, real *Ai)
{
    real M[NV * NV], X[NV * NV], D[NV];
    for (int i = 0; i < NV; i++)
    {
        real a = A[i * NV + i];
        if (a == 0)
            return false;
        D[i] = 1.0 / a;
    }
    for (int i = 0; i < NV; i++)
        for (int j = 0; j < NV; j++)
            M[i * NV + j] = D[i] * A[i * NV + j], X[i * NV + j] = i == j ? 1.0 : 0.0;
    for (int k = 0; k < NV; k++)
    {
        int pr = k;
        real best = fabs(M[k * NV + k]);
        for (int i = k + 1; i < NV; i++)
            if (fabs(M[i * NV + k]) > best)
                best = fabs(M[i * NV + k]), pr = i;
        if (!(best > 0))
            return false;
        if (pr != k)
            for (int j = 0; j < NV; j++)
            {
                real t = M[k * NV + j];
                M[k * NV + j] = M[pr * NV + j], M[pr * NV + j] = t;
                t = X[k * NV + j];
                X[k * NV + j] = X[pr * NV + j], X[pr * NV + j] = t;
            }
        real ip = 1.0 / M[k * NV + k];
        for (int j = 0; j < NV; j++)
            M[k * NV + j] *= ip, X[k * NV + j] *= ip;
        for (int i = 0; i < NV; i++)
        {
            if (i == k)
                continue;
            real fct = M[i * NV + k];
            for (int j = 0; j < NV; j++)
                M[i * NV + j] -= fct * M[k * NV + j], X[i * NV + j] -= fct * X[k * NV + j];
        }
    }
    for (int i = 0; i < NV; i++)
        for (int j = 0; j < NV; j++)
            Ai[i * NV + j] = X[i * NV + j] * D[j];
    return true;
}

// y = M x for a row-major NV x NV block
template <int NV, typename T, typename TX>
DNDSB_HD void block_mul(const T *M, const TX *x, TX *y)
{
    for (int r = 0; r < NV; r++)
    {
        TX acc = 0;
        for (int l = 0; l < NV; l++)
            acc += (TX)M[r * NV + l] * x[l];
        y[r] = acc;
    }
}
} // namespace roej
} // namespace dndsb
