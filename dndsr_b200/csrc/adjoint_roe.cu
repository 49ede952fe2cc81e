// Reverse-mode derivative of the interior-face Roe-family fluxes (Roe and Roe_M1..M8) and of HLLE+.
//
// RoeFlux_IdealGas_HartenYee (Gas.hpp:1038-1126) with the Roe averages r of the two cell means
// (Gas.hpp:229-259) is
//   F(U_L, U_R; r) = (F_phys(U_L) + F_phys(U_R)) / 2 - D(r, n) (U_R - U_L) / 2,
// where the dissipation D(r, n) = |A_Roe| (Gas.hpp:1098-1124, eigenvalues fixed by
// Roe_EntropyFixer, Gas.hpp:878-1007) depends on the means and the normal only.  Its
// cotangents therefore split:
//   * point states: Fbar^T dF/dU_L = (A(U_L)^T Fbar + D^T Fbar) / 2, dF/dU_R likewise with -D,
//     A = the physical-flux Jacobian (transposed by flux_jac_du_t), D^T Fbar from D applied to
//     the five unit jumps in real arithmetic;
//   * cell means: only D depends on them.  For plain Roe a hand-written reverse sweep of the
//     eigenvalues, wave strengths and dissipation gives, per Gauss point, D^T Fbar and the
//     cotangents of the Roe-average fields, and one Dual<10> evaluation of the averages per face
//     carries those to the means; the other schemes take the eigenvalues and D (U_R - U_L) in
//     Dual<10> per Gauss point.
// HLLEPFlux_IdealGas (Gas.hpp:601-714) mixes the point states into its wave-speed bounds, so it is
// reversed as a whole (hllep_rev), with the same per-face Dual<10> Roe averages for the means.
// This replaces two 10-wide forward passes through the whole flux.  Boundary faces keep the
// generic derivative kernel (ghost states).
#include "solver.cuh"
#include "basis_eval.cuh"
#include "flux_t.cuh"
#include "roe_rev.cuh"

namespace dndsb
{
namespace
{
constexpr int NV = 5;
constexpr int kHLLEP = 100; // flux mode of HLLE+ (Roe schemes use their eigScheme 0..8)
using D10 = Dual<10>;
using D1 = Dual<1>;
using roe_rev::RoeBar;
using roe_rev::roebar_zero;
using roe_rev::roe0_diss_rev;
using roe_rev::hllep_rev;

template <typename T>
DNDSB_D void roe_eigen(int es, const RoeAvgT<T> &r, const real *n, real dLambda, real fixScale, real incFScale, T &l0, T &l123, T &l4)
{
    T vRoe0 = dot3v(r.v, n);
    l0 = fabs(vRoe0 - r.a), l123 = fabs(vRoe0), l4 = fabs(vRoe0 + r.a);
    T vLm0 = dot3v(r.vL, n), vRm0 = dot3v(r.vR, n);
    if (es == 2)
    {
        l0 = l123 = l4 = dmax(T(fabs(vLm0) + r.aL), T(fabs(vRm0) + r.aR));
        return;
    }
    T VAve = sqrt(r.vsqr);
    roe_entropy_fix(es, r.aL, r.aR, r.a, vLm0, vRm0, vRoe0, VAve, dLambda, fixScale, incFScale, l0, l123, l4);
}

// incF = D(r, n) incU with the eigenvalues l0, l123, l4 (the Rusanov-like scheme 2 uses l0 I)
template <typename T>
DNDSB_D void roe_diss(int es, const T *incU, const real *n, const RoeAvgT<T> &r, real gamma, const T &l0, const T &l123, const T &l4, T *incF)
{
    if (es == 2)
    {
        for (int i = 0; i < 5; i++)
            incF[i] = l0 * incU[i];
        return;
    }
    RoeWavesT<T> w;
    roe_waves(incU, n, r, gamma, w);
    roe_dissipation(w, n, r, l0, l123, l4, incF);
}

template <int DIM, int P>
DNDSB_GLOBAL void k_rhs_vjp_face_roe(MeshD m, GeomD g, VRD vr, EulerSettingsD s, int es, const real *__restrict__ w, const real *__restrict__ u,
                                     const real *__restrict__ uRec, const real *__restrict__ dLamCell, real *__restrict__ faceAdj, int *err)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1, W = (R + 1) * NV;
    const real gamma = s.gamma;
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        int64_t c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        if (c1 < 0)
            continue;
        real *o0 = faceAdj + (f * 2) * W, *o1 = faceAdj + (f * 2 + 1) * W;
        real gbar[NV];
        for (int v = 0; v < NV; v++)
            gbar[v] = w[c0 * NV + v] / g.vol[c0] - w[c1 * NV + v] / g.vol[c1];
        const real *ULm = u + c0 * NV, *URm = u + c1 * NV;
        real dLambda = dmax(dLamCell[c0], dLamCell[c1]);
        RoeAvg r;
        roe_average(ULm, URm, gamma, r);
        RoeAvgT<D10> rD;
        {
            D10 a[NV], b[NV];
            for (int v = 0; v < NV; v++)
                a[v] = D10::var(ULm[v], v), b[v] = D10::var(URm[v], NV + v);
            roe_average(a, b, gamma, rD);
        }
        real acc0[W], acc1[W], mbar[2 * NV];
        for (int i = 0; i < W; i++)
            acc0[i] = 0, acc1[i] = 0;
        for (int i = 0; i < 2 * NV; i++)
            mbar[i] = 0;
        bool bad = !(r.asqr > 0);
        RoeBar rbar;
        roebar_zero(rbar);
        for (int q = 0; q < g.nGf; q++)
        {
            const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
            real p0[3], p1[3];
            for (int d = 0; d < 3; d++)
            {
                p0[d] = g.facePP[(f * g.nGf + q) * 3 + d];
                p1[d] = p0[d] + m.facePShift[f * 3 + d];
            }
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            real Fbar[NV];
            for (int v = 0; v < NV; v++)
                Fbar[v] = -JW * gbar[v];
            real T0[NDOF], T1[NDOF];
            cell_basis<DIM, NDOF>(&g.cellCent[c0 * 3], &g.cellScale[c0 * 3], &vr.baseMoment[c0 * NDOF], vr.s.anisotropicLengths, p0, 1, T0);
            cell_basis<DIM, NDOF>(&g.cellCent[c1 * 3], &g.cellScale[c1 * 3], &vr.baseMoment[c1 * NDOF], vr.s.anisotropicLengths, p1, 1, T1);
            real UL[NV], UR[NV], incU[NV];
            for (int v = 0; v < NV; v++)
            {
                real a = ULm[v], b = URm[v];
                for (int j = 0; j < R; j++)
                    a += T0[1 + j] * uRec[(c0 * R + j) * NV + v], b += T1[1 + j] * uRec[(c1 * R + j) * NV + v];
                UL[v] = a, UR[v] = b, incU[v] = b - a;
            }
            bad |= !(UL[0] > 0 && UR[0] > 0);
            if (es == kHLLEP)
            {
                real ULbar[NV], URbar[NV];
                hllep_rev(UL, UR, n, r, gamma, dLambda, s.rsFixScale, Fbar, ULbar, URbar, rbar);
                for (int v = 0; v < NV; v++)
                {
                    acc0[v] += ULbar[v];
                    acc1[v] += URbar[v];
                    for (int j = 0; j < R; j++)
                    {
                        acc0[NV + j * NV + v] += T0[1 + j] * ULbar[v];
                        acc1[NV + j * NV + v] += T1[1 + j] * URbar[v];
                    }
                }
                continue;
            }
            if (es == 0)
            {
                // plain Roe: one reverse sweep gives D^T incFb and the Roe-average cotangents
                real incFb[NV], incUb[NV], AtL[NV], AtR[NV];
                for (int v = 0; v < NV; v++)
                    incFb[v] = -0.5 * Fbar[v];
                roe0_diss_rev(incU, n, r, gamma, dLambda, s.rsFixScale, s.rsIncFScale, incFb, incUb, rbar);
                flux_jac_du_t<NV>(UL, n, Fbar, 0.0, gamma, AtL);
                flux_jac_du_t<NV>(UR, n, Fbar, 0.0, gamma, AtR);
                for (int v = 0; v < NV; v++)
                {
                    real ULbar = 0.5 * AtL[v] - incUb[v], URbar = 0.5 * AtR[v] + incUb[v];
                    acc0[v] += ULbar;
                    acc1[v] += URbar;
                    for (int j = 0; j < R; j++)
                    {
                        acc0[NV + j * NV + v] += T0[1 + j] * ULbar;
                        acc1[NV + j * NV + v] += T1[1 + j] * URbar;
                    }
                }
                continue;
            }
            // point states
            real l0, l123, l4;
            roe_eigen(es, r, n, dLambda, s.rsFixScale, s.rsIncFScale, l0, l123, l4);
            real DtF[NV];
            for (int i = 0; i < NV; i++)
            {
                real e[NV] = {0, 0, 0, 0, 0}, col[NV];
                e[i] = 1;
                roe_diss(es, e, n, r, gamma, l0, l123, l4, col);
                real a = 0;
                for (int k = 0; k < NV; k++)
                    a += Fbar[k] * col[k];
                DtF[i] = a;
            }
            real AtL[NV], AtR[NV];
            flux_jac_du_t<NV>(UL, n, Fbar, 0.0, gamma, AtL);
            flux_jac_du_t<NV>(UR, n, Fbar, 0.0, gamma, AtR);
            // cell means, through D(r, n) (U_R - U_L)
            {
                D10 L0, L123, L4, inc[NV], incF[NV];
                roe_eigen(es, rD, n, dLambda, s.rsFixScale, s.rsIncFScale, L0, L123, L4);
                for (int v = 0; v < NV; v++)
                    inc[v] = D10(incU[v]);
                roe_diss(es, inc, n, rD, gamma, L0, L123, L4, incF);
                for (int i = 0; i < 2 * NV; i++)
                {
                    real a = 0;
                    for (int k = 0; k < NV; k++)
                        a += Fbar[k] * incF[k].d[i];
                    mbar[i] -= 0.5 * a;
                }
            }
            for (int v = 0; v < NV; v++)
            {
                real ULbar = 0.5 * (AtL[v] + DtF[v]), URbar = 0.5 * (AtR[v] - DtF[v]);
                acc0[v] += ULbar;
                acc1[v] += URbar;
                for (int j = 0; j < R; j++)
                {
                    acc0[NV + j * NV + v] += T0[1 + j] * ULbar;
                    acc1[NV + j * NV + v] += T1[1 + j] * URbar;
                }
            }
        }
        if (es == 0 || es == kHLLEP)
        {
            // Roe-average cotangents -> cell means through the per-face Dual<10> averages
            for (int i = 0; i < 2 * NV; i++)
            {
                real a = rbar.aL * rD.aL.d[i] + rbar.aR * rD.aR.d[i] + rbar.vsqr * rD.vsqr.d[i] + rbar.H * rD.H.d[i] + rbar.asqr * rD.asqr.d[i] +
                         rbar.a * rD.a.d[i];
                for (int d = 0; d < 3; d++)
                    a += rbar.v[d] * rD.v[d].d[i] + rbar.vL[d] * rD.vL[d].d[i] + rbar.vR[d] * rD.vR[d].d[i];
                mbar[i] = a;
            }
        }
        for (int v = 0; v < NV; v++)
            acc0[v] += mbar[v], acc1[v] += mbar[NV + v];
        for (int i = 0; i < W; i++)
            o0[i] = acc0[i], o1[i] = acc1[i];
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}

} // namespace

// the reverse-mode flux of a Riemann-solver code: the Roe eigScheme 0..8, kHLLEP, or -1 (forward mode)
int roe_scheme_of(int rsType)
{
    if (rsType == RS_HLLEP)
        return kHLLEP;
    return rsType == RS_Roe ? 0 : (rsType >= RS_Roe_M1 && rsType <= RS_Roe_M8) ? rsType - 10 : -1;
}

int rhs_vjp_roe_interior(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *w, const real *u, const real *uRec,
                         real *faceAdj, cudaStream_t st, bool *viscDone)
{
    int es = roe_scheme_of(ev.s.rsType);
    if (es < 0 || ev.s.nVars != NV)
        return ST_UNSUPPORTED;
    *viscDone = false;
    // plain Roe and HLLE+ with the viscous flux: the Gauss-point-parallel kernel of adjoint_fast.cu (the
    // inviscid flux alone is as fast or faster in the thread-per-face kernel below: 1.06 against 1.88 ms for
    // plain Roe on 249,600 tets at degree 1, 3.7 ms either way for HLLE+ on the 64^3 TGV at degree 2)
    if ((es == 0 || es == kHLLEP) && !ev.s.ignoreVis)
    {
        int rc = rhs_vjp_interior_fast(m, g, vr, ev, es == kHLLEP, w, u, uRec, faceAdj, st);
        if (rc != ST_UNSUPPORTED)
        {
            *viscDone = !ev.s.ignoreVis;
            return rc;
        }
    }
#define DNDSB_ROE(DD, PP) DNDSB_LAUNCH((k_rhs_vjp_face_roe<DD, PP>), m.nFace, 64, st, m, g, vr, ev.s, es, w, u, uRec, ev.deltaLambdaCell, faceAdj, ev.errWord)
    if (m.dim == 2)
    {
        if (vr.P == 1)
            DNDSB_ROE(2, 1);
        else if (vr.P == 2)
            DNDSB_ROE(2, 2);
        else
            DNDSB_ROE(2, 3);
    }
    else if (vr.P == 1)
        DNDSB_ROE(3, 1);
    else if (vr.P == 2)
        DNDSB_ROE(3, 2);
    else
        DNDSB_ROE(3, 3);
#undef DNDSB_ROE
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
