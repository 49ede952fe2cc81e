// Reverse of the compact viscous flux at one face Gauss point (5 variables, or 6 with the SA model), shared
// by the viscous derivative kernels (adjoint_visc.cu) and the Gauss-point-parallel face VJP (adjoint_fast.cu).
#pragma once
#include "solver.cuh"
#include "sa.cuh"

namespace dndsb
{
namespace visc_rev
{
constexpr int NV = 5;

// the 5-variable branch of point_viscous_flux (sa.cuh), on any scalar type
template <typename T>
DNDSB_D void visc_flux_t(const EulerSettingsD &s, const T *UM, const T *GP, const real *n, T *Fv)
{
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    T pM, a2M, HM;
    gas_thermal(UM[4], UM[0], (UM[1] * UM[1] + UM[2] * UM[2] + UM[3] * UM[3]) / (UM[0] * UM[0]), gamma, pM, a2M, HM);
    T Tm = pM / ((gamma - 1) / gamma * cp * UM[0]);
    T mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, UM[0], Tm);
    viscous_flux<NV>(UM, GP, n, false, gamma, mu, cp * mu / s.prGas, cp, Fv);
}

// bar[0..NV-1] = (dFv/dU_M)^T Fvbar and bar[NV..4 NV-1] = (dFv/d grad U_M)^T Fvbar at one point: the reverse
// sweep of point_viscous_flux after grad_cons2prim (Gas.hpp:1594-1655, 1677-1698), statement by statement,
// in real arithmetic (U_M = UM, grad U_M = GM [3][NV] conservative, interior faces: not adiabatic).  NV = 6
// adds the SA model (EulerEvaluator.hpp:791-877): the eddy viscosity mu_t(U5, mu) in the stress (mu + mu_t)
// and the heat flux (cp mu_t / 0.9 + cp mu / Pr), and the nuTilde diffusion flux
// (grad(U5 / rho) . n) (mu + U5 muRef fn) / sigma.
template <int NVV = 5>
DNDSB_D void visc_point_bar(const EulerSettingsD &s, const real *UM, const real *GM, const real *n, const real *Fvbar, real *bar)
{
    constexpr int N = NVV;
    const real gamma = s.gamma, gm1 = gamma - 1, cp = s.Rgas * gamma / gm1, kT = gamma / (gm1 * cp), cTm = gm1 / gamma * cp;
    const real rho = UM[0], ir = 1.0 / rho;
    const real v[3] = {UM[1] * ir, UM[2] * ir, UM[3] * ir};
    const real vv = dot3(v, v);
    const real p = gm1 * (UM[4] - rho * 0.5 * vv);
    const real Tm = p / (cTm * rho);
    const real mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, rho, Tm);
    const real dmudT = s.muModel == 1 ? mu * (1.5 / Tm - 1.0 / (Tm + s.CSutherland)) : 0.0;
    const real dmudr = s.muModel == 2 ? s.muGas : 0.0;
    // SA: chi0 = U5 muRef / mu, chi = chi0 below 10 smoothed by 0.05 log(1 + exp(20 chi0)), mu_t = mu f(chi),
    // f = chi^4 / (chi^3 + cnu1^3)
    real muT = 0, fT = 0, dfdchi = 0, chi0 = 0, dchi = 1;
    if constexpr (N == 6)
    {
        chi0 = UM[5] * s.muGas / mu;
        real chi = chi0;
        if (chi0 < 10)
        {
            const real e = exp(20 * chi0);
            chi = 0.05 * log(1 + e);
            dchi = e / (1 + e);
        }
        const real c3 = SAConst::cnu1 * SAConst::cnu1 * SAConst::cnu1, x3 = chi * chi * chi;
        fT = dmax(chi * x3 / (x3 + c3), 0.0);
        dfdchi = fT > 0 ? x3 * (x3 + 4 * c3) / ((x3 + c3) * (x3 + c3)) : 0.0;
        muT = mu * fT;
    }
    const real muS = mu + muT;                                              // viscosity of the stress
    const real k = N == 6 ? cp * muT / 0.9 + cp * mu / s.prGas : cp * mu / s.prGas; // heat conductivity
    // forward: primitive gradient, temperature gradient, stress
    real gp[3][N];
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        const real *g = GM + r * N;
        gp[r][0] = g[0];
        real sr = 0;
#pragma unroll
        for (int j = 0; j < 3; j++)
        {
            gp[r][1 + j] = (rho * g[1 + j] - g[0] * UM[1 + j]) * ir * ir;
            sr += g[1 + j] * v[j];
        }
#pragma unroll
        for (int j = 0; j < 3; j++)
            sr += gp[r][1 + j] * UM[1 + j];
        gp[r][4] = gm1 * (g[4] - 0.5 * sr);
        if constexpr (N == 6)
            gp[r][5] = (g[5] - g[0] * UM[5] * ir) * ir;
    }
    const real cT = kT * ir * ir;
    real gT[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        gT[i] = cT * (rho * gp[i][4] - p * gp[i][0]);
    const real tr = gp[0][1] + gp[1][2] + gp[2][3];
    const real lm = -2.0 / 3.0 * muS * tr;
    // reverse: Fv[1+i] = sum_j s_ij n_j, Fv[4] = sum_i (sum_j s_ij v_j + k gT_i) n_i
    real gpb[3][N], vb[3] = {0, 0, 0}, mb[3] = {0, 0, 0};
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < N; c++)
            gpb[r][c] = 0;
    real mub = 0, lmb = 0, kb = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
    {
        kb += Fvbar[4] * gT[i] * n[i];
#pragma unroll
        for (int j = 0; j < 3; j++)
        {
            const real sij = (gp[i][1 + j] + gp[j][1 + i]) * muS + (i == j ? lm : 0.0);
            vb[j] += Fvbar[4] * n[i] * sij;
            const real sb = Fvbar[1 + i] * n[j] + Fvbar[4] * n[i] * v[j];
            gpb[i][1 + j] += sb * muS;
            gpb[j][1 + i] += sb * muS;
            mub += sb * (gp[i][1 + j] + gp[j][1 + i]);
            if (i == j)
                lmb += sb;
        }
    }
    mub += -2.0 / 3.0 * tr * lmb;
    const real trb = -2.0 / 3.0 * muS * lmb;
    gpb[0][1] += trb, gpb[1][2] += trb, gpb[2][3] += trb;
    // gT_i = cT (rho gp_i4 - p gp_i0), gTb_i = Fvbar[4] k n_i
    real cTb = 0, rhob = 0, pb = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
    {
        const real gTb = Fvbar[4] * k * n[i];
        cTb += gTb * (rho * gp[i][4] - p * gp[i][0]);
        rhob += gTb * cT * gp[i][4];
        pb -= gTb * cT * gp[i][0];
        gpb[i][4] += gTb * cT * rho;
        gpb[i][0] -= gTb * cT * p;
    }
    real irb = cTb * kT * 2.0 * ir;
    // the laminar viscosity's cotangent through the stress, the heat flux and (SA) mu_t and the diffusion
    real mulb = mub + kb * cp / s.prGas, u5b = 0;
    if constexpr (N == 6)
    {
        const real muTb = mub + kb * cp / 0.9;
        // mu_t = mu f(chi(chi0)), chi0 = U5 muRef / mu
        mulb += muTb * fT;
        const real chi0b = muTb * mu * dfdchi * dchi;
        u5b += chi0b * s.muGas / mu;
        mulb -= chi0b * chi0 / mu;
        // Fv5 = gn5 D, D = (mu + U5 muRef fn) / sigma; fn = 1, or (cn1 + X) / (cn1 - X), X = chi0^3, for U5 < 0
        real gn5 = 0;
#pragma unroll
        for (int d = 0; d < 3; d++)
            gn5 += gp[d][5] * n[d];
        real fn = 1, dfn = 0;
        if (UM[5] < 0)
        {
            const real X = chi0 * chi0 * chi0, den = SAConst::cn1 - X;
            fn = (SAConst::cn1 + X) / den;
            dfn = 2 * SAConst::cn1 / (den * den) * 3 * chi0 * chi0; // d fn / d chi0
        }
        const real D = (mu + UM[5] * s.muGas * fn) / SAConst::sigma;
#pragma unroll
        for (int d = 0; d < 3; d++)
            gpb[d][5] += Fvbar[5] * D * n[d];
        const real Db = Fvbar[5] * gn5 / SAConst::sigma;
        mulb += Db;
        u5b += Db * s.muGas * fn;
        const real chi0b2 = Db * UM[5] * s.muGas * dfn;
        u5b += chi0b2 * s.muGas / mu;
        mulb -= chi0b2 * chi0 / mu;
    }
    // mu = mu(rho, T), T = p / (cTm rho)
    const real Tb = mulb * dmudT;
    rhob += mulb * dmudr;
    pb += Tb / (cTm * rho);
    rhob -= Tb * Tm / rho;
    // primitive gradient -> conservative gradient and state
    real *Gb = bar + N;
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        const real *g = GM + r * N;
        real *gb = Gb + r * N;
        const real srb = -0.5 * gm1 * gpb[r][4];
        gb[4] = gm1 * gpb[r][4];
        gb[0] = gpb[r][0];
#pragma unroll
        for (int j = 0; j < 3; j++)
        {
            vb[j] += srb * g[1 + j];
            mb[j] += srb * gp[r][1 + j];
            const real a = gpb[r][1 + j] + srb * UM[1 + j];
            gb[1 + j] = srb * v[j] + a * ir;
            gb[0] -= a * UM[1 + j] * ir * ir;
            rhob += a * g[1 + j] * ir * ir;
            mb[j] -= a * g[0] * ir * ir;
            irb += a * (rho * g[1 + j] - g[0] * UM[1 + j]) * 2.0 * ir;
        }
        if constexpr (N == 6)
        {
            // gp5 = g5 ir - g0 U5 ir^2
            const real a = gpb[r][5];
            gb[5] = a * ir;
            gb[0] -= a * UM[5] * ir * ir;
            u5b -= a * g[0] * ir * ir;
            irb += a * (g[5] - 2.0 * g[0] * UM[5] * ir);
        }
    }
    // p = (gamma - 1) (E - m.m / (2 rho)); v = m / rho; ir = 1 / rho
    rhob += gm1 * 0.5 * vv * pb;
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
        mb[j] += -gm1 * v[j] * pb + vb[j] * ir;
        irb += vb[j] * UM[1 + j];
    }
    rhob -= irb * ir * ir;
    bar[0] = rhob;
    bar[1] = mb[0], bar[2] = mb[1], bar[3] = mb[2];
    bar[4] = gm1 * pb;
    if constexpr (N == 6)
        bar[5] = u5b;
}
} // namespace visc_rev
} // namespace dndsb
