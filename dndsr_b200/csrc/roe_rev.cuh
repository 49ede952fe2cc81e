// Hand-reversed inviscid face fluxes at one Gauss point (5 variables): the plain Roe dissipation with its
// Harten-Yee entropy fix and HLLE+, with the cotangents of the Roe-average fields.  Shared by the interior-face
// VJP kernels (adjoint_roe.cu, fast.cu).
#pragma once
#include "solver.cuh"
#include "flux_t.cuh"

namespace dndsb
{
namespace roe_rev
{
// cotangents of the Roe-average fields the plain Roe flux uses
struct RoeBar
{
    real v[3], vL[3], vR[3], aL, aR, vsqr, H, asqr, a;
};

DNDSB_D void roebar_zero(RoeBar &b)
{
    for (int d = 0; d < 3; d++)
        b.v[d] = b.vL[d] = b.vR[d] = 0;
    b.aL = b.aR = b.vsqr = b.H = b.asqr = b.a = 0;
}

// reverse of one Harten-Yee limiter application of Roe_EntropyFixer scheme 0 (Gas.hpp:878-930):
//   th = max(max(0, lam - lamL), lamR - lam) sHY,  out = v < th ? (v^2 / th + th) / 2 : v
DNDSB_D void flim_rev(real v, real lam, real lamL, real lamR, real sHY, real ob, real &vb, real &lamb, real &lamLb, real &lamRb)
{
    real d1 = lam - lamL, d2 = lamR - lam;
    real m1 = 0.0 > d1 ? 0.0 : d1;
    bool pick2 = !(m1 > d2);
    real th = (pick2 ? d2 : m1) * sHY;
    real thb = 0;
    if (v < th)
    {
        vb = ob * v / th;
        thb = ob * 0.5 * (1.0 - v * v / (th * th));
    }
    else
        vb = ob;
    real Mb = thb * sHY;
    lamb = 0, lamLb = 0, lamRb = 0;
    if (pick2)
        lamRb += Mb, lamb -= Mb;
    else if (!(0.0 > d1))
        lamb += Mb, lamLb -= Mb;
}

// Plain Roe (scheme 0): incF = D(r, n) incU.  Given incFb, adds the cotangents of incU (incUb, set)
// and of the Roe-average fields (rb, accumulated), recomputing the forward intermediates of
// roe_eigen / roe_waves / roe_dissipation statement by statement
// (l123bIn: an extra cotangent of the fixed eigenvalue l123, which the SA convective flux also uses; l123Out,
// when given, receives l123)
DNDSB_D void roe0_diss_rev(const real *incU, const real *n, const RoeAvg &r, real gamma, real dLambda, real fixScale, real incFScale,
                           const real *incFb, real *incUb, RoeBar &rb, real l123bIn = 0, real *l123Out = nullptr)
{
    // forward: eigenvalues
    const real sHY = 0.05 * fixScale;
    (void)dLambda;
    real vN = dot3(r.v, n), vLm0 = dot3(r.vL, n), vRm0 = dot3(r.vR, n);
    real in0 = fabs(vN - r.a), in123 = fabs(vN) * incFScale, in4 = fabs(vN + r.a);
    auto flim = [&](real v, real lam, real lamL, real lamR)
    {
        real th = dmax(dmax(0.0, lam - lamL), lamR - lam) * sHY;
        return v < th ? (v * v / th + th) * 0.5 : v;
    };
    real l0 = flim(in0, vN - r.a, vLm0 - r.aL, vRm0 - r.aR);
    real l123 = flim(in123, vN, vLm0, vRm0);
    real l4 = flim(in4, vN + r.a, vLm0 + r.aL, vRm0 + r.aR);
    if (l123Out)
        *l123Out = l123;
    // forward: waves
    real incU123N = incU[1] * n[0] + incU[2] * n[1] + incU[3] * n[2];
    real a23[3] = {incU[1] - incU[0] * r.v[0], incU[2] - incU[0] * r.v[1], incU[3] - incU[0] * r.v[2]};
    real a23n = dot3(a23, n);
    real a23T[3];
    for (int d = 0; d < 3; d++)
        a23T[d] = a23[d] - n[d] * a23n;
    real incU4b = incU[4] - dot3(a23T, r.v);
    real X = incU[0] * (r.H - vN * vN) + vN * incU123N - incU4b;
    real wa1 = (gamma - 1) / r.asqr * X;
    real num = incU[0] * (vN + r.a) - incU123N - r.a * wa1;
    real wa0 = num / (2 * r.a);
    real wa4 = incU[0] - (wa0 + wa1);
    // forward: dissipation products
    real A0 = wa0 * l0, A1 = wa1 * l123, A4 = wa4 * l4;
    real t[3] = {a23T[0] * l123, a23T[1] * l123, a23T[2] * l123};
    // reverse: dissipation
    const real *Fb = incFb;
    real A0b = Fb[0] + (r.H - vN * r.a) * Fb[4], A1b = Fb[0] + 0.5 * r.vsqr * Fb[4], A4b = Fb[0] + (r.H + vN * r.a) * Fb[4];
    real tb[3];
    real vNb = r.a * (A4 - A0) * Fb[4];
    rb.H += (A0 + A4) * Fb[4];
    rb.a += vN * (A4 - A0) * Fb[4];
    rb.vsqr += 0.5 * A1 * Fb[4];
    for (int d = 0; d < 3; d++)
    {
        A0b += (r.v[d] - r.a * n[d]) * Fb[1 + d];
        A1b += r.v[d] * Fb[1 + d];
        A4b += (r.v[d] + r.a * n[d]) * Fb[1 + d];
        tb[d] = r.v[d] * Fb[4] + Fb[1 + d];
        rb.a += n[d] * (A4 - A0) * Fb[1 + d];
        rb.v[d] += t[d] * Fb[4] + (A0 + A4 + A1) * Fb[1 + d];
    }
    real l0b = wa0 * A0b, l123b = wa1 * A1b + l123bIn, l4b = wa4 * A4b;
    real wa0b = l0 * A0b, wa1b = l123 * A1b, wa4b = l4 * A4b;
    real a23Tb[3];
    for (int d = 0; d < 3; d++)
    {
        a23Tb[d] = l123 * tb[d];
        l123b += a23T[d] * tb[d];
    }
    // reverse: waves
    for (int i = 0; i < 5; i++)
        incUb[i] = 0;
    incUb[0] += wa4b;
    wa0b -= wa4b;
    wa1b -= wa4b;
    real numb = wa0b / (2 * r.a);
    rb.a += -wa0 / r.a * wa0b;
    incUb[0] += (vN + r.a) * numb;
    vNb += incU[0] * numb;
    rb.a += (incU[0] - wa1) * numb;
    real incU123Nb = -numb;
    wa1b -= r.a * numb;
    real Xb = (gamma - 1) / r.asqr * wa1b;
    rb.asqr += -wa1 / r.asqr * wa1b;
    incUb[0] += (r.H - vN * vN) * Xb;
    rb.H += incU[0] * Xb;
    vNb += (-2 * vN * incU[0] + incU123N) * Xb;
    incU123Nb += vN * Xb;
    real incU4bb = -Xb;
    incUb[4] += incU4bb;
    real a23nb = 0, a23b[3];
    for (int d = 0; d < 3; d++)
    {
        a23Tb[d] += -r.v[d] * incU4bb;
        rb.v[d] += -a23T[d] * incU4bb;
        a23b[d] = a23Tb[d];
        a23nb -= n[d] * a23Tb[d];
    }
    for (int d = 0; d < 3; d++)
    {
        a23b[d] += n[d] * a23nb;
        incUb[1 + d] += a23b[d] + n[d] * incU123Nb;
        incUb[0] += -r.v[d] * a23b[d];
        rb.v[d] += -incU[0] * a23b[d];
    }
    // reverse: eigenvalues (the three limiter applications and the |.| of their inputs; at a kink
    // |x| takes the slope of x >= 0, as the forward-mode dual numbers do)
    real vLm0b = 0, vRm0b = 0, vb, lb, lLb, lRb;
    flim_rev(in0, vN - r.a, vLm0 - r.aL, vRm0 - r.aR, sHY, l0b, vb, lb, lLb, lRb);
    {
        real sg = vN - r.a >= 0 ? 1.0 : -1.0;
        vNb += sg * vb + lb;
        rb.a += -sg * vb - lb;
        vLm0b += lLb, rb.aL -= lLb, vRm0b += lRb, rb.aR -= lRb;
    }
    flim_rev(in123, vN, vLm0, vRm0, sHY, l123b, vb, lb, lLb, lRb);
    {
        real sg = vN >= 0 ? 1.0 : -1.0;
        vNb += incFScale * sg * vb + lb;
        vLm0b += lLb, vRm0b += lRb;
    }
    flim_rev(in4, vN + r.a, vLm0 + r.aL, vRm0 + r.aR, sHY, l4b, vb, lb, lLb, lRb);
    {
        real sg = vN + r.a >= 0 ? 1.0 : -1.0;
        vNb += sg * vb + lb;
        rb.a += sg * vb + lb;
        vLm0b += lLb, rb.aL += lLb, vRm0b += lRb, rb.aR += lRb;
    }
    for (int d = 0; d < 3; d++)
    {
        rb.v[d] += n[d] * vNb;
        rb.vL[d] += n[d] * vLm0b;
        rb.vR[d] += n[d] * vRm0b;
    }
}

// reverse of the wave strength a1 of roe_waves (Gas.hpp:1098-1109) with respect to incU and the Roe
// averages: adds a1b d a1/d(incU, r) to incUb, rb (and d a1 / d vRoe0 to vNb)
DNDSB_D void roe_a1_rev(const real *incU, const real *n, const RoeAvg &r, real gamma, real a1b, real *incUb, RoeBar &rb, real &vNb)
{
    real vN = dot3(r.v, n);
    real incU123N = incU[1] * n[0] + incU[2] * n[1] + incU[3] * n[2];
    real a23[3] = {incU[1] - incU[0] * r.v[0], incU[2] - incU[0] * r.v[1], incU[3] - incU[0] * r.v[2]};
    real a23n = dot3(a23, n);
    real a23T[3];
    for (int d = 0; d < 3; d++)
        a23T[d] = a23[d] - n[d] * a23n;
    real incU4b = incU[4] - dot3(a23T, r.v);
    real X = incU[0] * (r.H - vN * vN) + vN * incU123N - incU4b;
    real a1 = (gamma - 1) / r.asqr * X;
    real Xb = (gamma - 1) / r.asqr * a1b;
    rb.asqr += -a1 / r.asqr * a1b;
    incUb[0] += (r.H - vN * vN) * Xb;
    rb.H += incU[0] * Xb;
    vNb += (-2 * vN * incU[0] + incU123N) * Xb;
    real incU123Nb = vN * Xb;
    real incU4bb = -Xb;
    incUb[4] += incU4bb;
    real a23nb = 0, a23b[3];
    for (int d = 0; d < 3; d++)
    {
        real a23Tb = -r.v[d] * incU4bb;
        rb.v[d] += -a23T[d] * incU4bb;
        a23b[d] = a23Tb;
        a23nb -= n[d] * a23Tb;
    }
    for (int d = 0; d < 3; d++)
    {
        a23b[d] += n[d] * a23nb;
        incUb[1 + d] += a23b[d] + n[d] * incU123Nb;
        incUb[0] += -r.v[d] * a23b[d];
        rb.v[d] += -incU[0] * a23b[d];
    }
}

// d(a^2)/dU of the ideal gas (a^2 = gamma p / rho) times ab, added to Ub
DNDSB_D void asqr_rev(const real *U, real gamma, real ab, real *Ub)
{
    real ir = 1.0 / U[0];
    real m2 = U[1] * U[1] + U[2] * U[2] + U[3] * U[3];
    real p = (gamma - 1) * (U[4] - 0.5 * m2 * ir);
    real dpdr = (gamma - 1) * 0.5 * m2 * ir * ir;
    Ub[0] += ab * gamma * (dpdr * U[0] - p) * ir * ir;
    for (int d = 0; d < 3; d++)
        Ub[1 + d] += ab * gamma * ir * (-(gamma - 1) * U[1 + d] * ir);
    Ub[4] += ab * gamma * ir * (gamma - 1);
}

// HLLEPFlux_IdealGas (Gas.hpp:601-714) reversed: given Fbar, the cotangents of U_L, U_R (ULb, URb,
// set) and of the Roe-average fields (rb, accumulated); branch choices (min/max/|.|) follow the
// primal values, |x| at 0 takes the slope of x >= 0
DNDSB_D void hllep_rev(const real *UL, const real *UR, const real *n, const RoeAvg &r, real gamma, real dLambda, real fixScale,
                       const real *Fbar, real *ULb, real *URb, RoeBar &rb)
{
    real FL[5], FR[5], pL, pR, aL2, aR2;
    phys_flux(UL, n, gamma, FL, pL, aL2);
    phys_flux(UR, n, gamma, FR, pR, aR2);
    real vRoe0 = dot3(r.v, n), vLm0 = dot3(r.vL, n), vRm0 = dot3(r.vR, n);
    real incU[5];
    for (int i = 0; i < 5; i++)
        incU[i] = UR[i] - UL[i];
    RoeWavesT<real> w;
    roe_waves(incU, n, r, gamma, w);
    real sL = sqrt(aL2), sR = sqrt(aR2);
    real x1 = vRoe0 - r.a, x2 = vLm0 - sL, y1 = vRoe0 + r.a, y2 = vRm0 + sR;
    real SL = dmin(x1, x2), SR = dmax(y1, y2);
    real Mx = dmax(fabs(vRoe0), dLambda * fixScale);
    real dfix = r.a / (r.a + Mx);
    real SP = dmax(SR, 0.0), SM = dmin(SL, 0.0);
    real div = SP - SM;
    div = div + (div >= 0 ? 1 : -1) * kVerySmall;
    real id = 1.0 / div;
    real rv1[5] = {1.0, r.v[0], r.v[1], r.v[2], 0.5 * r.vsqr};
    real P = SP * SM * id;
    // F_i = (SP FL_i - SM FR_i) id + P X_i,  X_i = incU_i - dfix rv1_i a1
    real FLb[5], FRb[5], incUb[5], sumFrv = 0, G = 0, sumFX = 0, sumFFL = 0, sumFFR = 0;
    for (int i = 0; i < 5; i++)
    {
        real Xi = incU[i] - dfix * rv1[i] * w.a1;
        FLb[i] = SP * id * Fbar[i];
        FRb[i] = -SM * id * Fbar[i];
        incUb[i] = P * Fbar[i];
        sumFrv += Fbar[i] * rv1[i];
        sumFX += Fbar[i] * Xi;
        sumFFL += Fbar[i] * FL[i];
        sumFFR += Fbar[i] * FR[i];
        G += Fbar[i] * ((SP * FL[i] - SM * FR[i]) + SP * SM * Xi);
    }
    real a1b = -P * dfix * sumFrv;
    real dfixb = -P * w.a1 * sumFrv;
    for (int d = 0; d < 3; d++)
        rb.v[d] += -P * dfix * w.a1 * Fbar[1 + d];
    rb.vsqr += -P * dfix * w.a1 * Fbar[4] * 0.5;
    real SPb = sumFFL * id + SM * id * sumFX - id * id * G;
    real SMb = -sumFFR * id + SP * id * sumFX + id * id * G;
    real SRb = SR > 0.0 ? SPb : 0.0;
    real SLb = SL < 0.0 ? SMb : 0.0;
    real vNb = 0, vLm0b = 0, vRm0b = 0, aL2b = 0, aR2b = 0;
    if (x1 < x2)
        vNb += SLb, rb.a -= SLb;
    else
        vLm0b += SLb, aL2b += -SLb * 0.5 / sL;
    if (y1 > y2)
        vNb += SRb, rb.a += SRb;
    else
        vRm0b += SRb, aR2b += SRb * 0.5 / sR;
    // dfix = a / (a + Mx), Mx = max(|vRoe0|, dLambda fixScale)
    real den = r.a + Mx;
    rb.a += dfixb * Mx / (den * den);
    real Mxb = -dfixb * r.a / (den * den);
    if (fabs(vRoe0) > dLambda * fixScale)
        vNb += Mxb * (vRoe0 >= 0 ? 1.0 : -1.0);
    roe_a1_rev(incU, n, r, gamma, a1b, incUb, rb, vNb);
    // point states: physical fluxes, sound speeds, jump
    flux_jac_du_t<5>(UL, n, FLb, 0.0, gamma, ULb);
    flux_jac_du_t<5>(UR, n, FRb, 0.0, gamma, URb);
    asqr_rev(UL, gamma, aL2b, ULb);
    asqr_rev(UR, gamma, aR2b, URb);
    for (int i = 0; i < 5; i++)
        ULb[i] -= incUb[i], URb[i] += incUb[i];
    for (int d = 0; d < 3; d++)
    {
        rb.v[d] += n[d] * vNb;
        rb.vL[d] += n[d] * vLm0b;
        rb.vR[d] += n[d] * vRm0b;
    }
}
} // namespace roe_rev
} // namespace dndsb
