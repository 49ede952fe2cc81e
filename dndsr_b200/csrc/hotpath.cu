// Hot-path kernels: VR block-Jacobi sweep, right-hand side (face flux +
// per-cell gather, no atomics), local time step, LU-SGS diagonal, multicolour
// SGS sweeps and the LU-SGS matrix-vector product.
#include "solver.cuh"
#include "basis_eval.cuh"
#include "sa.cuh"

namespace dndsb
{
namespace
{
DNDSB_D bool finite5(const real *v, int n)
{
    bool ok = true;
    for (int i = 0; i < n; i++)
        ok = ok && isfinite(v[i]);
    return ok;
}

// ---------------------------------------------------------------------------
// VR iteration: VariationalReconstruction_Reconstruction.hxx:485-615
// (Jacobi branch).  uRecNew_i = (1 - w) uRec_i + w sum_k (A^-1B_k uRec_k + A^-1b_k (u_k - u_i))
// recordInc: uRecNew_i = uRec_i - sum_k (...) (the preconditioned residual)
// ---------------------------------------------------------------------------
template <int R, int NV, typename TC>
DNDSB_GLOBAL void k_vr_jacobi(int64_t nCell, int nf, const int32_t *__restrict__ nbr, const TC *__restrict__ AAInvB,
                              const TC *__restrict__ AInvb, const real *__restrict__ uRec, real *__restrict__ uRecNew,
                              const real *__restrict__ u, real relax, int recordInc, int uRecIsZero)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        real acc[R * NV];
        const real *in = uRec + c * R * NV;
        for (int i = 0; i < R * NV; i++)
            acc[i] = recordInc ? (uRecIsZero ? 0.0 : in[i]) : in[i] * (1 - relax);
        real ui[NV];
        for (int v = 0; v < NV; v++)
            ui[v] = u[c * NV + v];
        real sgn = recordInc ? -1.0 : relax;
        for (int k = 0; k < nf; k++)
        {
            int o = nbr[c * nf + k];
            if (o < 0)
                continue;
            const TC *M = AAInvB + ((c * (nf + 1) + 1 + k) * R) * R;
            const TC *b = AInvb + (c * nf + k) * R;
            const real *uo = uRec + (int64_t)o * R * NV;
            real du[NV];
            for (int v = 0; v < NV; v++)
                du[v] = u[(int64_t)o * NV + v] - ui[v];
            for (int i = 0; i < R; i++)
            {
                real t[NV];
                real bi = (real)b[i];
                for (int v = 0; v < NV; v++)
                    t[v] = bi * du[v];
                if (!(recordInc && uRecIsZero))
                    for (int j = 0; j < R; j++)
                    {
                        real mij = (real)M[i * R + j];
                        for (int v = 0; v < NV; v++)
                            t[v] += mij * uo[j * NV + v];
                    }
                for (int v = 0; v < NV; v++)
                    acc[i * NV + v] += sgn * t[v];
            }
        }
        real *out = uRecNew + c * R * NV;
        for (int i = 0; i < R * NV; i++)
            out[i] = acc[i];
    }
}

DNDSB_GLOBAL void k_fill_from(int64_t n, const real *src, real *out)
{
    DNDSB_KERNEL_LOOP(i, n)
    {
        out[i] = *src;
    }
}

DNDSB_GLOBAL void k_swap(int64_t n, real *a, real *b)
{
    DNDSB_KERNEL_LOOP(i, n)
    {
        real t = a[i];
        a[i] = b[i], b[i] = t;
    }
}

// ---------------------------------------------------------------------------
// RHS face kernel: EulerEvaluator_EvaluateRHS.hxx:171-562 with the flux of
// EulerEvaluator_EvaluateDt.hxx:1084-1511 (interior and periodic faces).
// Writes the integrated face flux -(F_inv - F_vis).n dA; the per-cell
// gather below divides by the volume.
// ---------------------------------------------------------------------------
template <int DIM, int P, int NV>
// uRecG: the reconstruction the gradients come from (the reference's uRecUnlim, EvaluateRHS.hxx:264-327;
// the same array as uRec when there is no limiter); point values come from uRec
// lam (may be nullptr): [3][nFace] face integrals of the Riemann eigenvalues l0, l123, l4 divided by the area
// (EvaluateRHS.hxx:527-545, recorded for useRoeJacobian)
DNDSB_GLOBAL void k_rhs_face(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ u, const real *__restrict__ uRec,
                             const real *__restrict__ uRecG, const real *__restrict__ dLamCell, real *__restrict__ faceFlux, int *err,
                             real *__restrict__ lam)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        int c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        real fluxEs[NV];
        for (int v = 0; v < NV; v++)
            fluxEs[v] = 0;
        if (c1 < 0)
        {
            for (int v = 0; v < NV; v++)
                faceFlux[f * NV + v] = 0;
            continue;
        }
        const real *ULm = u + (int64_t)c0 * NV, *URm = u + (int64_t)c1 * NV;
        const real *r0 = uRec + (int64_t)c0 * R * NV, *r1 = uRec + (int64_t)c1 * R * NV;
        const real *q0 = uRecG + (int64_t)c0 * R * NV, *q1 = uRecG + (int64_t)c1 * R * NV;
        real dLambda = dmax(dLamCell[c0], dLamCell[c1]);
        real minVol = dmin(g.vol[c0], g.vol[c1]);
        real db[3];
        for (int d = 0; d < 3; d++)
            db[d] = g.cellBary[c1 * 3 + d] - m.facePShift[f * 3 + d] - g.cellBary[c0 * 3 + d];
        real areaInv2 = 2.0 / g.faceArea[f];
        bool bad = false;
        real lamEs[3] = {0, 0, 0};
        for (int q = 0; q < g.nGf; q++)
        {
            const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
            real p0[3], p1[3];
            for (int d = 0; d < 3; d++)
            {
                p0[d] = g.facePP[(f * g.nGf + q) * 3 + d];
                p1[d] = p0[d] + m.facePShift[f * 3 + d];
            }
            real T0[(DIM + 1) * NDOF], T1[(DIM + 1) * NDOF];
            cell_basis<DIM, NDOF>(&g.cellCent[c0 * 3], &g.cellScale[c0 * 3], &vr.baseMoment[(int64_t)c0 * NDOF], vr.s.anisotropicLengths, p0,
                                  DIM + 1, T0);
            cell_basis<DIM, NDOF>(&g.cellCent[c1 * 3], &g.cellScale[c1 * 3], &vr.baseMoment[(int64_t)c1 * NDOF], vr.s.anisotropicLengths, p1,
                                  DIM + 1, T1);
            real UL[NV], UR[NV], GL[3 * NV], GR[3 * NV];
            for (int v = 0; v < NV; v++)
            {
                real a = ULm[v], b = URm[v];
                real ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
                for (int j = 0; j < R; j++)
                {
                    real x0 = r0[j * NV + v], x1 = r1[j * NV + v];
                    real y0 = q0[j * NV + v], y1 = q1[j * NV + v];
                    a += T0[1 + j] * x0;
                    b += T1[1 + j] * x1;
                    for (int d = 0; d < DIM; d++)
                        ga[d] += T0[(1 + d) * NDOF + 1 + j] * y0, gb[d] += T1[(1 + d) * NDOF + 1 + j] * y1;
                }
                UL[v] = a, UR[v] = b;
                for (int d = 0; d < 3; d++)
                    GL[d * NV + v] = ga[d], GR[d * NV + v] = gb[d];
            }
            real distBaryPerp = fabs(dot3(db, n));
            real distGRP = minVol * areaInv2;
            distGRP = dmax(dmin(distBaryPerp, distGRP * 2), distGRP * 0.25);
            real UM[NV], GM[3 * NV], GP[3 * NV], Fv[NV];
            for (int v = 0; v < NV; v++)
                UM[v] = 0.5 * (UL[v] + UR[v]);
            for (int v = 0; v < NV; v++)
                Fv[v] = 0;
            if (!s.ignoreVis)
            {
                real iD = 1.0 / distGRP;
                for (int d = 0; d < 3; d++)
                    for (int v = 0; v < NV; v++)
                        GM[d * NV + v] = (GR[d * NV + v] + GL[d * NV + v]) * 0.5 + iD * (n[d] * (UR[v] - UL[v]));
                grad_cons2prim<NV>(UM, GM, GP, gamma);
                point_viscous_flux<NV>(s, UM, GP, n, false, Fv);
            }
            real F[NV], l0, l1, l4;
            bad |= !riemann_flux(s.rsType, UL, UR, ULm, URm, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4,
                                 s.rsMeanValueEig ? &g.faceMeanNorm[f * 3] : nullptr);
            if (NV == 6)
                F[NV - 1] = sa_convective_flux(UL, UR, n, l1);
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            for (int v = 0; v < NV; v++)
                fluxEs[v] -= (F[v] - Fv[v]) * JW;
            lamEs[0] += l0 * JW, lamEs[1] += l1 * JW, lamEs[2] += l4 * JW;
        }
        if (bad || !finite5(fluxEs, NV))
            atomicOr(err, bad ? (int)DE_NONPHYSICAL : (int)DE_NONFINITE);
        for (int v = 0; v < NV; v++)
            faceFlux[f * NV + v] = fluxEs[v];
        if (lam)
            for (int i = 0; i < 3; i++)
                lam[i * m.nFace + f] = lamEs[i] / g.faceArea[f];
    }
}

// per-cell gather of the face fluxes (deterministic, replaces the reference's face scatter)
template <int NV>
DNDSB_GLOBAL void k_rhs_gather(int64_t nCell, int nf, const int32_t *__restrict__ c2f, const real *__restrict__ vol,
                               const real *__restrict__ faceFlux, real *__restrict__ rhs)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        real acc[NV];
        for (int v = 0; v < NV; v++)
            acc[v] = 0;
        real iv = 1.0 / vol[c];
        for (int k = 0; k < nf; k++)
        {
            int fp = c2f[c * nf + k];
            int64_t f = fp >> 1;
            real sg = (fp & 1) ? -1.0 : 1.0;
            for (int v = 0; v < NV; v++)
                acc[v] += sg * faceFlux[f * NV + v];
        }
        for (int v = 0; v < NV; v++)
            rhs[c * NV + v] = acc[v] * iv;
    }
}

// ---------------------------------------------------------------------------
// Local time step: EulerEvaluator_EvaluateDt.hxx:875-1039
// ---------------------------------------------------------------------------
template <int NV>
DNDSB_GLOBAL void k_dt_face(MeshD m, GeomD g, EulerSettingsD s, const real *__restrict__ u, real *lamFace, real *lamFaceC,
                            real *lamFaceVis, real *lamConv, real *dLamFace)
{
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        int c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        const real *n = &g.faceMeanNorm[f * 3];
        const real *UL = u + (int64_t)c0 * NV;
        real uM[NV];
        for (int v = 0; v < NV; v++)
            uM[v] = UL[v];
        real vL[3] = {UL[1] / UL[0], UL[2] / UL[0], UL[3] / UL[0]}, vR[3];
        real pL, a2L, HL, pR, a2R, HR;
        gas_thermal(UL[4], UL[0], dot3(vL, vL), gamma, pL, a2L, HL);
        vR[0] = vL[0], vR[1] = vL[1], vR[2] = vL[2], pR = pL, a2R = a2L;
        real volR = g.vol[c0];
        if (c1 >= 0)
        {
            const real *UR = u + (int64_t)c1 * NV;
            for (int v = 0; v < NV; v++)
                uM[v] = (uM[v] + UR[v]) * 0.5;
            for (int d = 0; d < 3; d++)
                vR[d] = UR[1 + d] / UR[0];
            gas_thermal(UR[4], UR[0], dot3(vR, vR), gamma, pR, a2R, HR);
            volR = g.vol[c1];
        }
        real vnL = dot3(vL, n), vnR = dot3(vR, n);
        real vnM = 0.5 * (vnL + vnR);
        real pM = (pL + pR) * 0.5;
        real aL = sqrt(a2L), aR = sqrt(a2R);
        real lamC = dmax(aL + fabs(vnL), aR + fabs(vnR));
        real T = pM / ((gamma - 1) / gamma * cp * uM[0]);
        real mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, uM[0], T);
        if (NV == 6)
            mu += sa_mu_tur(uM, s.muGas, mu);
        real lamVis = mu / uM[0] * dmax(4. / 3., gamma / s.prGas);
        real area = g.faceArea[f];
        real vis = lamVis * area * (1. / g.vol[c0] + 1. / volR);
        lamFace[f] = lamC + vis;
        lamFaceC[f] = fabs(vnM) + vis;
        lamFaceVis[f] = vis;
        lamConv[f] = lamC;
        real dvn = vnR - vnL;
        dLamFace[f] = dmax(dmax(fabs(dvn + aR - aL), fabs(dvn - aR + aL)), fabs(aL - aR));
    }
}

DNDSB_GLOBAL void k_dt_cell(MeshD m, GeomD g, const real *__restrict__ lamFace, const real *__restrict__ dLamFace, real CFL, real MaxDt,
                            real *dt, real *dLamCell)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real lc = 0, dl = 0;
        for (int k = 0; k < m.nf; k++)
        {
            int64_t f = m.cell2face[c * m.nf + k] >> 1;
            lc += lamFace[f] * g.faceArea[f];
            dl = dmax(dl, dLamFace[f]);
        }
        dt[c] = dmin(CFL * g.vol[c] * g.smoothRatio[c] / (lc + 1e-100), MaxDt);
        dLamCell[c] = dl;
    }
}

// ---------------------------------------------------------------------------
// LU-SGS (EulerEvaluator.hxx:37-159 init, :550-693 UpdateSGS, :175-274 MatrixVec)
// scalar Jacobian, inviscid flux-increment Jacobian EulerEvaluator.hpp:1100-1158
// ---------------------------------------------------------------------------
// nd = 1: one diagonal per cell; nd = nv (SA model): fp plus alphaDiag JSource per variable
DNDSB_GLOBAL void k_lusgs_init(MeshD m, GeomD g, const real *__restrict__ lamFace, const real *__restrict__ dTau, real dt, real alphaDiag,
                               const real *__restrict__ jSource, int nd, real *jdiag)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real fp = 1.0 / dTau[c] + 1.0 / dt;
        real iv = 1.0 / g.vol[c];
        for (int k = 0; k < m.nf; k++)
        {
            int64_t f = m.cell2face[c * m.nf + k] >> 1;
            fp += (0.5 * alphaDiag) * g.faceArea[f] * lamFace[f] * iv;
        }
        for (int v = 0; v < nd; v++)
            jdiag[c * nd + v] = fp + (nd > 1 ? alphaDiag * jSource[c * nd + v] : 0.0);
    }
}

template <int NV>
DNDSB_D void flux_jac_du(const real *U, const real *n, const real *dU, real lam, real gamma, real *dF)
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
    for (int j = 0; j < NV; j++)
        dF[j] -= lam * dU[j];
}

template <int NV>
DNDSB_GLOBAL void k_sgs_color(MeshD m, GeomD g, real gamma, const real *__restrict__ lamFace, const int32_t *__restrict__ cellColor,
                              int64_t cBeg, int64_t cEnd, int color, real alphaDiag, const real *__restrict__ rhs, const real *__restrict__ u,
                              const real *__restrict__ uInc, real *uIncNew, const real *__restrict__ jdiag, int forward, int gsUpdate,
                              int uIncIsZero, real *absInc)
{
    DNDSB_KERNEL_LOOP(ii, cEnd - cBeg)
    {
        int64_t c = m.colorCells[cBeg + ii];
        real buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = rhs[c * NV + v];
        real cf = 0.5 * alphaDiag / g.vol[c];
        for (int k = 0; k < m.nf; k++)
        {
            int o = m.cellNbr[c * m.nf + k];
            if (o < 0 || o == c)
                continue;
            int oc = cellColor[o];
            bool useNew = gsUpdate && (forward ? oc < color : oc > color);
            if (uIncIsZero && !useNew)
                continue;
            int fp = m.cell2face[c * m.nf + k];
            int64_t f = fp >> 1;
            real sg = (fp & 1) ? -1.0 : 1.0;
            real n[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
            const real *dU = useNew ? uIncNew + (int64_t)o * NV : uInc + (int64_t)o * NV;
            real dF[NV];
            flux_jac_du<NV>(u + (int64_t)o * NV, n, dU, lamFace[f], gamma, dF);
            real w = cf * g.faceArea[f];
            for (int v = 0; v < NV; v++)
                buf[v] -= w * dF[v];
        }
        for (int v = 0; v < NV; v++)
        {
            real id = 1.0 / jdiag[NV == 6 ? c * NV + v : c];
            real nv = buf[v] * id;
            absInc[c * NV + v] = fabs(nv - uIncNew[c * NV + v]);
            uIncNew[c * NV + v] = nv;
        }
    }
}

// UpdateLUSGSForward / UpdateLUSGSBackward (EulerEvaluator.hxx:376-529): forward
//   uIncNew_c = D_c^-1 (rhs_c - sum_{o < c} (alpha/2)(A_f/V_c) dF(u_o; uInc_o)),
// backward uIncNew_c += D_c^-1 (- sum_{o > c} of the same).  "Lower" and "upper" are cell indices,
// as in the reference.  cells == nullptr: every cell of [cBeg, cEnd) in one launch (uInc distinct from
// uIncNew, so the cells are independent); otherwise the cells of one colour (in-place sweep).
template <int NV>
DNDSB_GLOBAL void k_lusgs_sweep(MeshD m, GeomD g, real gamma, const real *__restrict__ lamFace, const int32_t *__restrict__ cells,
                                int64_t cBeg, int64_t cEnd, real alphaDiag, const real *__restrict__ rhs, const real *__restrict__ u,
                                const real *uInc, real *uIncNew, const real *__restrict__ jdiag, int forward)
{
    DNDSB_KERNEL_LOOP(ii, cEnd - cBeg)
    {
        int64_t c = cells ? (int64_t)cells[cBeg + ii] : cBeg + ii;
        real buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = forward ? rhs[c * NV + v] : 0.0;
        real cf = 0.5 * alphaDiag / g.vol[c];
        for (int k = 0; k < m.nf; k++)
        {
            int o = m.cellNbr[c * m.nf + k];
            if (o < 0 || !(forward ? o < c : o > c))
                continue;
            int fp = m.cell2face[c * m.nf + k];
            int64_t f = fp >> 1;
            real sg = (fp & 1) ? -1.0 : 1.0;
            real n[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
            real dF[NV];
            flux_jac_du<NV>(u + (int64_t)o * NV, n, uInc + (int64_t)o * NV, lamFace[f], gamma, dF);
            real w = cf * g.faceArea[f];
            for (int v = 0; v < NV; v++)
                buf[v] -= w * dF[v];
        }
        for (int v = 0; v < NV; v++)
        {
            real x = buf[v] / jdiag[NV == 6 ? c * NV + v : c];
            uIncNew[c * NV + v] = forward ? x : uIncNew[c * NV + v] + x;
        }
    }
}

template <int NV>
DNDSB_GLOBAL void k_matvec(MeshD m, GeomD g, real gamma, const real *__restrict__ lamFace, real alphaDiag, const real *__restrict__ u,
                           const real *__restrict__ uInc, const real *__restrict__ jdiag, real *AuInc)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = 0;
        real cf = 0.5 * alphaDiag / g.vol[c];
        for (int k = 0; k < m.nf; k++)
        {
            int o = m.cellNbr[c * m.nf + k];
            if (o < 0)
                continue;
            int fp = m.cell2face[c * m.nf + k];
            int64_t f = fp >> 1;
            real sg = (fp & 1) ? -1.0 : 1.0;
            real n[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
            real dF[NV];
            flux_jac_du<NV>(u + (int64_t)o * NV, n, uInc + (int64_t)o * NV, lamFace[f], gamma, dF);
            real w = cf * g.faceArea[f];
            for (int v = 0; v < NV; v++)
                buf[v] -= w * dF[v];
        }
        for (int v = 0; v < NV; v++)
            AuInc[c * NV + v] = jdiag[NV == 6 ? c * NV + v : c] * uInc[c * NV + v] - buf[v];
    }
}

// EulerEvaluator.hxx:1039-1143: 2 = isentropic vortex (SpecialFields.hpp:42-77) at t = 0, 3 = Taylor-Green (M0 = 0.1)
template <int NV>
DNDSB_GLOBAL void k_init_field(MeshD m, GeomD g, real gamma, int kind, real chi, real *u)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real um[NV];
        for (int v = 0; v < NV; v++)
            um[v] = 0;
        for (int q = 0; q < g.nGc; q++)
        {
            const real *x = &g.cellPP[(c * g.nGc + q) * 3];
            real rho, ux, uy, p;
            if (kind == 2)
            {
                real px = x[0] - floor(x[0] / 10) * 10, py = x[1] - floor(x[1] / 10) * 10;
                real r2 = sqr(px - 5) + sqr(py - 5);
                real dT = -(gamma - 1) / (8 * gamma * sqr(kPi)) * sqr(chi) * exp(1 - r2);
                real e = chi / 2 / kPi * exp((1 - r2) / 2);
                ux = 1 - e * (py - 5), uy = 1 + e * (px - 5);
                real T = dT + 1;
                rho = pow(T, 1 / (gamma - 1));
                p = T * rho;
            }
            else
            {
                const real M0 = 0.1;
                ux = sin(x[0]) * cos(x[1]) * cos(x[2]);
                uy = -cos(x[0]) * sin(x[1]) * cos(x[2]);
                p = 1. / (gamma * sqr(M0)) + 1. / 16 * ((cos(2 * x[0]) + cos(2 * x[1])) * (2 + cos(2 * x[2])));
                rho = gamma * sqr(M0) * p;
            }
            real JW = g.cellJDet[c * g.nGc + q] * g.cellQw[q];
            um[0] += rho * JW, um[1] += rho * ux * JW, um[2] += rho * uy * JW;
            um[4] += (0.5 * (ux * ux + uy * uy) * rho + p / (gamma - 1)) * JW;
        }
        for (int v = 0; v < NV; v++)
            u[c * NV + v] = um[v] / g.vol[c];
    }
}

// EvaluateRHS.hxx:665-801 for the SA model: the source at the cell Gauss points (state and
// conservative gradient from the reconstruction), integrated and divided by the volume, added to
// rhs; the mode-1 diagonal Jacobian gives JSource.  The NS source is zero.
template <int DIM, int P>
// values from uRec, gradients from uRecG (uRecUnlim); the integral times cellRHSAlpha / V (EvaluateRHS.hxx:790;
// alpha == nullptr: 1), for the source and its Jacobian diagonal alike
DNDSB_GLOBAL void k_sa_source(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ u, const real *__restrict__ uRec,
                              const real *__restrict__ uRecG, const real *__restrict__ alpha, const real *__restrict__ dWall, real *rhs,
                              real *jSource)
{
    constexpr int NV = 6, NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real S = 0, J = 0;
        real hMax = g.hMax[c];
        for (int q = 0; q < g.nGc; q++)
        {
            real T[(DIM + 1) * NDOF];
            cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], &vr.baseMoment[c * NDOF], vr.s.anisotropicLengths,
                                  &g.cellPP[(c * g.nGc + q) * 3], DIM + 1, T);
            real U[NV], G[3 * NV];
            for (int v = 0; v < NV; v++)
            {
                real a = u[c * NV + v];
                real ga[3] = {0, 0, 0};
                for (int j = 0; j < R; j++)
                {
                    real x = uRec[(c * R + j) * NV + v], y = uRecG[(c * R + j) * NV + v];
                    a += T[1 + j] * x;
                    for (int d = 0; d < DIM; d++)
                        ga[d] += T[(1 + d) * NDOF + 1 + j] * y;
                }
                U[v] = a;
                for (int d = 0; d < 3; d++)
                    G[d * NV + v] = ga[d];
            }
            real pM, a2M, HM;
            gas_thermal(U[4], U[0], (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / (U[0] * U[0]), gamma, pM, a2M, HM);
            real Tm = pM / ((gamma - 1) / gamma * cp * U[0]);
            real mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, U[0], Tm);
            real d = dmin(dWall[c * g.nGc + q], pow(kVeryLarge, 1. / 6.));
            real lLES = dmin(hMax * kVeryLarge, dmax(d, hMax));
            real JW = g.cellJDet[c * g.nGc + q] * g.cellQw[q];
            S += sa_source(U, G, s.muGas, mu, d, lLES, hMax, 0) * JW;
            J += sa_source(U, G, s.muGas, mu, d, lLES, hMax, 1) * JW;
        }
        real sc = (alpha ? alpha[c] : 1.0) / g.vol[c];
        rhs[c * NV + 5] += S * sc;
        for (int v = 0; v < NV; v++)
            jSource[c * NV + v] = v == 5 ? J * sc : 0.0;
    }
}

int check(cudaStream_t st, int *errWord, bool syncErr)
{
    if (last_error() != cudaSuccess)
        return ST_CUDA;
    if (!syncErr)
        return ST_OK;
    int e = 0;
    d2h(&e, errWord, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    if (e & DE_NONPHYSICAL)
        return ST_NONPHYSICAL;
    if (e & DE_NONFINITE)
        return ST_NONFINITE;
    return ST_OK;
}
} // namespace

int vr_iter(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *uRec, real *uRecNew, const real *u, int recordInc,
            int uRecIsZero, int useFP32, cudaStream_t st)
{
    // interior faces (tuned kernel when one is instantiated), then the boundary faces
    if (vr_iter_fast(m, vr, nv, uRec, uRecNew, u, recordInc, uRecIsZero, useFP32, st) == ST_OK)
        return vr_iter_bc(m, g, vr, nv, uRec, uRecNew, u, recordInc, uRecIsZero, useFP32, st);
    real relax = vr.s.jacobiRelax;
#define DNDSB_VRJ(RR, NVV)                                                                                                             \
    do                                                                                                                                 \
    {                                                                                                                                  \
        if (useFP32)                                                                                                                   \
            DNDSB_LAUNCH((k_vr_jacobi<RR, NVV, float>), m.nCell, 128, st, m.nCell, m.nf, m.cellNbr, vr.AAInvB32, vr.AInvb32, uRec, uRecNew, \
                         u, relax, recordInc, uRecIsZero);                                                                             \
        else                                                                                                                           \
            DNDSB_LAUNCH((k_vr_jacobi<RR, NVV, real>), m.nCell, 128, st, m.nCell, m.nf, m.cellNbr, vr.AAInvB, vr.AInvb, uRec, uRecNew, u, \
                         relax, recordInc, uRecIsZero);                                                                                \
    } while (0)
#define DNDSB_VRJ_NV(RR)          \
    do                            \
    {                             \
        if (nv == 5)              \
            DNDSB_VRJ(RR, 5);     \
        else if (nv == 6)         \
            DNDSB_VRJ(RR, 6);     \
        else if (nv == 1)         \
            DNDSB_VRJ(RR, 1);     \
        else                      \
            return ST_UNSUPPORTED; \
    } while (0)
    switch (vr.R)
    {
    case 2:
        DNDSB_VRJ_NV(2);
        break;
    case 3:
        DNDSB_VRJ_NV(3);
        break;
    case 5:
        DNDSB_VRJ_NV(5);
        break;
    case 9:
        DNDSB_VRJ_NV(9);
        break;
    case 19:
        DNDSB_VRJ_NV(19);
        break;
    default:
        return ST_UNSUPPORTED;
    }
#undef DNDSB_VRJ_NV
#undef DNDSB_VRJ
    if (last_error() != cudaSuccess)
        return ST_CUDA;
    return vr_iter_bc(m, g, vr, nv, uRec, uRecNew, u, recordInc, uRecIsZero, useFP32, st);
}

int vr_swap(int64_t n, real *a, real *b, cudaStream_t st)
{
    DNDSB_LAUNCH(k_swap, n, 256, st, n, a, b);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

// wall-flux integral of EvaluateRHS.hxx:599-607: minus the face fluxes of the BCWall / BCWallIsothermal faces
// (and of BCWallInvis faces when muGas < 1e-99), summed over the boundary-face list in a fixed order (one
// block: thread partial sums over a fixed stride, then a fixed tree)
template <int NV>
DNDSB_GLOBAL void k_wall_flux_sum(MeshD m, BoundaryD bnd, real muGas, const real *__restrict__ ff, real *out)
{
    __shared__ real sp[256][NV];
    real acc[NV];
    for (int v = 0; v < NV; v++)
        acc[v] = 0;
    for (int64_t ii = threadIdx.x; ii < m.nBndFace; ii += blockDim.x)
    {
        int64_t f = m.bndFace[ii];
        int zone = m.faceZone[f];
        int t = zone >= 0 && zone < bnd.nZone ? bnd.type[zone] : 0;
        if (t == BC_WALL || t == BC_WALL_ISOTHERMAL || (t == BC_WALL_INVIS && muGas < 1e-99))
            for (int v = 0; v < NV; v++)
                acc[v] -= ff[f * NV + v];
    }
    for (int v = 0; v < NV; v++)
        sp[threadIdx.x][v] = acc[v];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if ((int)threadIdx.x < w)
            for (int v = 0; v < NV; v++)
                sp[threadIdx.x][v] += sp[threadIdx.x + w][v];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < NV; v++)
            out[v] = sp[0][v];
}

int eval_rhs(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *u, const real *uRec, real *rhs, real *faceFlux,
             cudaStream_t st)
{
    return eval_rhs_ex(m, g, vr, ev, u, uRec, uRec, nullptr, 0, rhs, faceFlux, nullptr, st);
}

int eval_rhs_ex(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *u, const real *uRecG, const real *uRec,
                const real *alpha, unsigned flags, real *rhs, real *faceFlux, real *jSourceOut, cudaStream_t st)
{
    real *ff = faceFlux ? faceFlux : ev.faceFlux;
    int nv = ev.s.nVars;
    if (nv != 5 && nv != 6)
        return ST_UNSUPPORTED;
    // a per-call RHS_Ignore_Viscosity on top of the settings; in deferred mode the kernels OR into the
    // evaluator's deferred error word, which only dndsb_eval_check_errors reads and clears
    EvalD evc = ev;
    if (flags & RHSF_IGNORE_VISCOSITY)
        evc.s.ignoreVis = 1;
    if (ev.deferErr)
        evc.errWord = ev.errDeferred;
    else
        dev_zero(ev.errWord, sizeof(int), st);
    const EulerSettingsD &s = evc.s;
    real *lamOut = ev.jacMode == 2 ? ev.lambdaFace0 : nullptr; // [3][nFace]: lambdaFace0, 123, 4
    int frc = uRecG == uRec ? rhs_face_fast(m, g, vr, evc, u, uRec, ff, st) : (int)ST_UNSUPPORTED;
    if (frc == ST_CUDA)
        return ST_CUDA;
    if (frc != ST_OK)
    {
#define DNDSB_RF(D, PP, NVV) \
    DNDSB_LAUNCH((k_rhs_face<D, PP, NVV>), m.nFace, 128, st, m, g, vr, s, u, uRec, uRecG, ev.deltaLambdaCell, ff, evc.errWord, lamOut)
#define DNDSB_RF_P(D, NVV)        \
    do                            \
    {                             \
        if (vr.P == 1)            \
            DNDSB_RF(D, 1, NVV);  \
        else if (vr.P == 2)       \
            DNDSB_RF(D, 2, NVV);  \
        else                      \
            DNDSB_RF(D, 3, NVV);  \
    } while (0)
        if (m.dim == 2)
        {
            if (nv == 5)
                DNDSB_RF_P(2, 5);
            else
                DNDSB_RF_P(2, 6);
        }
        else
        {
            if (nv == 5)
                DNDSB_RF_P(3, 5);
            else
                DNDSB_RF_P(3, 6);
        }
#undef DNDSB_RF_P
#undef DNDSB_RF
    }
    int brc = rhs_bc(m, g, vr, evc, u, uRec, uRecG, ff, st);
    if (brc != ST_OK)
        return brc;
    if (nv == 5)
        DNDSB_LAUNCH(k_rhs_gather<5>, m.nCell, 256, st, m.nCell, m.nf, m.cell2face, g.vol, ff, rhs);
    else
    {
        DNDSB_LAUNCH(k_rhs_gather<6>, m.nCell, 256, st, m.nCell, m.nf, m.cell2face, g.vol, ff, rhs);
        // SA source (EvaluateRHS.hxx:665-801) and its Jacobian diagonal JSource
        if (!ev.dWall)
            return ST_BADARG;
#define DNDSB_SAS(D, PP) DNDSB_LAUNCH((k_sa_source<D, PP>), m.nCell, 64, st, m, g, vr, s, u, uRec, uRecG, alpha, ev.dWall, rhs, ev.jSource)
        if (m.dim == 2)
        {
            if (vr.P == 1)
                DNDSB_SAS(2, 1);
            else if (vr.P == 2)
                DNDSB_SAS(2, 2);
            else
                DNDSB_SAS(2, 3);
        }
        else
        {
            if (vr.P == 1)
                DNDSB_SAS(3, 1);
            else if (vr.P == 2)
                DNDSB_SAS(3, 2);
            else
                DNDSB_SAS(3, 3);
        }
#undef DNDSB_SAS
    }
    if (jSourceOut)
    {
        if (nv == 6)
            d2d(jSourceOut, ev.jSource, sizeof(real) * m.nCell * 6, st);
        else
            dev_zero(jSourceOut, sizeof(real) * m.nCell * nv, st);
    }
    if (!(flags & RHSF_DONT_UPDATE_INTEGRATION) && m.nBndFace > 0 && ev.fluxWall)
    {
        if (nv == 5)
            k_wall_flux_sum<5><<<1, 256, 0, st>>>(m, vr.bnd, s.muGas, ff, ev.fluxWall);
        else
            k_wall_flux_sum<6><<<1, 256, 0, st>>>(m, vr.bnd, s.muGas, ff, ev.fluxWall);
    }
    return check(st, evc.errWord, !ev.deferErr);
}

int eval_dt(const MeshD &m, const GeomD &g, EvalD &ev, const real *u, real CFL, real MaxDt, int useLocalDt, real *dt, real *dtMin,
            cudaStream_t st)
{
    if (ev.s.nVars == 5)
        DNDSB_LAUNCH(k_dt_face<5>, m.nFace, 256, st, m, g, ev.s, u, ev.lambdaFace, ev.lambdaFaceC, ev.lambdaFaceVis, ev.lambdaConv,
                     ev.deltaLambdaFace);
    else if (ev.s.nVars == 6)
        DNDSB_LAUNCH(k_dt_face<6>, m.nFace, 256, st, m, g, ev.s, u, ev.lambdaFace, ev.lambdaFaceC, ev.lambdaFaceVis, ev.lambdaConv,
                     ev.deltaLambdaFace);
    else
        return ST_UNSUPPORTED;
    DNDSB_LAUNCH(k_dt_cell, m.nCell, 256, st, m, g, ev.lambdaFace, ev.deltaLambdaFace, CFL, MaxDt, dt, ev.deltaLambdaCell);
    if (ev.lambdaFace0) // lambdaFace0 = lambdaFace123 = lambdaFace4 = the convective speed (EvaluateDt.hxx:995-996)
        for (real *l : {ev.lambdaFace0, ev.lambdaFace123, ev.lambdaFace4})
            d2d(l, ev.lambdaConv, sizeof(real) * m.nFace, st);
    if (useLocalDt && !dtMin) // nothing to reduce and nothing to report: no host synchronisation
        return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
    real *res = reduce_cols(1, m.nCell, 1, dt, nullptr, 0, ev.redBuf, st);
    real mn = 0;
    d2h(&mn, res, sizeof(real), st);
    if (dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    if (dtMin)
        *dtMin = mn;
    if (!useLocalDt) // every cell takes the global minimum
        DNDSB_LAUNCH(k_fill_from, m.nCell, 256, st, m.nCell, res, dt);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int lusgs_init(const MeshD &m, const GeomD &g, EvalD &ev, const real *dTau, real dt, real alphaDiag, real *jdiag, cudaStream_t st)
{
    int nd = ev.s.nVars == 6 ? 6 : 1;
    if (nd > 1 && !ev.jSource)
        return ST_BADARG;
    DNDSB_LAUNCH(k_lusgs_init, m.nCell, 256, st, m, g, ev.lambdaFace, dTau, dt, alphaDiag, ev.jSource, nd, jdiag);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int update_sgs(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc,
               real *uIncNew, const real *jdiag, int forward, int gsUpdate, int uIncIsZero, real *sumIncHost, cudaStream_t st)
{
    int nv = ev.s.nVars;
    real *absInc = ev.faceFlux; // [nCell][nv] fits in the [nFace][nv] scratch
    for (int ci = 0; ci < m.nColor; ci++)
    {
        int col = forward ? ci : m.nColor - 1 - ci;
        int64_t b = m.colorStart[col], e = m.colorStart[col + 1];
        if (nv == 5)
            DNDSB_LAUNCH(k_sgs_color<5>, e - b, 128, st, m, g, ev.s.gamma, ev.lambdaFace, m.cellColor, b, e, col, alphaDiag, rhs, u,
                         uInc, uIncNew, jdiag, forward, gsUpdate, uIncIsZero, absInc);
        else if (nv == 6)
            DNDSB_LAUNCH(k_sgs_color<6>, e - b, 128, st, m, g, ev.s.gamma, ev.lambdaFace, m.cellColor, b, e, col, alphaDiag, rhs, u,
                         uInc, uIncNew, jdiag, forward, gsUpdate, uIncIsZero, absInc);
        else
            return ST_UNSUPPORTED;
    }
    if (sumIncHost)
    {
        real *res = reduce_cols(0, m.nCell, nv, absInc, nullptr, 0, ev.redBuf, st);
        d2h(sumIncHost, res, sizeof(real) * nv, st);
        if (dev_sync(st) != cudaSuccess)
            return ST_CUDA;
    }
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int update_lusgs(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc,
                 real *uIncNew, const real *jdiag, int forward, cudaStream_t st)
{
    int nv = ev.s.nVars;
    if (nv != 5 && nv != 6)
        return ST_UNSUPPORTED;
    auto launch = [&](const int32_t *cells, int64_t b, int64_t e)
    {
        if (nv == 5)
            DNDSB_LAUNCH(k_lusgs_sweep<5>, e - b, 128, st, m, g, ev.s.gamma, ev.lambdaFace, cells, b, e, alphaDiag, rhs, u, uInc, uIncNew,
                         jdiag, forward);
        else
            DNDSB_LAUNCH(k_lusgs_sweep<6>, e - b, 128, st, m, g, ev.s.gamma, ev.lambdaFace, cells, b, e, alphaDiag, rhs, u, uInc, uIncNew,
                         jdiag, forward);
    };
    if (uInc != uIncNew)
        launch(nullptr, 0, m.nCell);
    else // in place: colour by colour, so a cell reads the new values of the neighbours swept before it
        for (int ci = 0; ci < m.nColor; ci++)
        {
            int col = forward ? ci : m.nColor - 1 - ci;
            launch(m.colorCells, m.colorStart[col], m.colorStart[col + 1]);
        }
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int lusgs_matvec(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *uInc, const real *jdiag,
                 real *AuInc, cudaStream_t st)
{
    if (ev.s.nVars == 5)
        DNDSB_LAUNCH(k_matvec<5>, m.nCell, 256, st, m, g, ev.s.gamma, ev.lambdaFace, alphaDiag, u, uInc, jdiag, AuInc);
    else if (ev.s.nVars == 6)
        DNDSB_LAUNCH(k_matvec<6>, m.nCell, 256, st, m, g, ev.s.gamma, ev.lambdaFace, alphaDiag, u, uInc, jdiag, AuInc);
    else
        return ST_UNSUPPORTED;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int init_field(const MeshD &m, const GeomD &g, const EvalD &ev, int kind, real chi, real *u, cudaStream_t st)
{
    if (ev.s.nVars != 5)
        return ST_UNSUPPORTED;
    DNDSB_LAUNCH(k_init_field<5>, m.nCell, 128, st, m, g, ev.s.gamma, kind, chi, u);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

// op 0: sum of |x|^powP * w over rows; op 2: max of |x|
int reduce_norm(int64_t n, int ncol, const real *x, const real *w, int op, int powP, real *redBuf, real *outHost, cudaStream_t st)
{
    real *res = reduce_cols(op, n, ncol, x, w, op == 0 ? powP : 1, redBuf, st);
    d2h(outHost, res, sizeof(real) * ncol, st);
    return dev_sync(st) == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
