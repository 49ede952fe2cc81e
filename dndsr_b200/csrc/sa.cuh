// Spalart-Allmaras model terms of the NS_SA model (6 conservative variables, the sixth being
// rho nuTilde / muRef): eddy viscosity, the nuTilde diffusion flux, the passive-scalar upwind flux
// and the source term with its diagonal Jacobian.  Settings are the reference defaults (SADESMode
// 1 IDDES shielding, rotation correction on, SAVersion 0) and its compiled options (negative-SA
// model, ft2 term).
#pragma once
#include "solver.cuh"

namespace dndsb
{
struct SAConst
{
    static constexpr real cb1 = 0.1355, cb2 = 0.622, sigma = 2.0 / 3.0, cnu1 = 7.1, cnu2 = 0.7, cnu3 = 0.9, cw2 = 0.3, cw3 = 2,
                          kappa = 0.41, rlim = 10, cn1 = 16.0, ct3 = 1.2, ct4 = 0.5;
};

// EulerEvaluator.hpp:791-833 getMuTur (chi smoothed below 10 by the negative-SA model)
DNDSB_HD real sa_mu_tur(const real *U, real muRef, real muf)
{
    real Chi = U[5] * muRef / muf;
    if (Chi < 10)
        Chi = 0.05 * log(1 + exp(20 * Chi));
    real Chi3 = Chi * Chi * Chi;
    real fnu1 = Chi3 / (Chi3 + SAConst::cnu1 * SAConst::cnu1 * SAConst::cnu1);
    return muf * dmax(Chi * fnu1, 0.0);
}

// EulerEvaluator.hpp:835-877 visFluxTurVariable: the nuTilde diffusion flux through n (GP is the
// primitive gradient [3][6], the sixth column d(U5 / rho))
DNDSB_HD real sa_diffusion_flux(const real *U, const real *GP, const real *n, real muRef, real mufPhy)
{
    real fn = 1;
    if (U[5] < 0)
    {
        real Chi = U[5] * muRef / mufPhy;
        fn = (SAConst::cn1 + Chi * Chi * Chi) / (SAConst::cn1 - Chi * Chi * Chi);
    }
    return (GP[0 * 6 + 5] * n[0] + GP[1 * 6 + 5] * n[1] + GP[2 * 6 + 5] * n[2]) * (mufPhy + U[5] * muRef * fn) / SAConst::sigma;
}

// EulerEvaluator_EvaluateDt.hxx:1413-1425: upwind flux of the SA variable with the Riemann
// solver's lam123 as dissipation speed (ransEigScheme 0)
DNDSB_HD real sa_convective_flux(const real *UL, const real *UR, const real *n, real lam123)
{
    real vnL = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) / UL[0];
    real vnR = (UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2]) / UR[0];
    return ((vnL * UL[5] + vnR * UR[5]) - (UR[5] - UL[5]) * lam123) * 0.5;
}

// RANS_ke.hpp:985-1195 GetSource_SA: mode 0 the source of the SA equation, mode 1 its diagonal
// Jacobian; G is the conservative gradient [3][6]
DNDSB_HD real sa_source(const real *U, const real *G, real muRef, real mufPhy, real d, real lLES, real hMax, int mode)
{
    using C = SAConst;
    const real cw1 = C::cb1 / (C::kappa * C::kappa) + (1 + C::cb2) / C::sigma;
    const real k2 = C::kappa * C::kappa;
    real nuh = U[5] * muRef / U[0];
    real Chi = U[5] * muRef / mufPhy;
    real Chi3 = Chi * Chi * Chi;
    real fnu1 = Chi3 / (Chi3 + C::cnu1 * C::cnu1 * C::cnu1);
    real fnu2 = 1 - Chi / (1 + Chi * fnu1);
    real velo[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
    real diffRho[3], diffNu[3], diffU[3][3];
    for (int i = 0; i < 3; i++)
    {
        diffRho[i] = G[i * 6 + 0];
        diffNu[i] = (G[i * 6 + 5] * muRef - nuh * diffRho[i]) / U[0];
        for (int j = 0; j < 3; j++)
            diffU[i][j] = (G[i * 6 + 1 + j] - diffRho[i] * velo[j]) / U[0];
    }
    real om2 = 0, ss2 = 0, du2 = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
        {
            real o = 0.5 * (diffU[j][i] - diffU[i][j]);
            real sij = diffU[i][j] + diffU[j][i];
            om2 += o * o, ss2 += sij * sij, du2 += diffU[i][j] * diffU[i][j];
        }
    real S = sqrt(om2) * sqrt(2.0);
    real SS = sqrt(ss2) * (1. / sqrt(2.0));
    real SRotCor = 2.0 * dmin(0.0, S - SS);
    real diffUNorm = sqrt(du2);
    real ft2 = C::ct3 * exp(-C::ct4 * Chi * Chi);
    // DDES shielding, then the IDDES blend (SADESMode 1)
    real lRANS = d;
    real nuTur = mufPhy / U[0] * dmax(Chi * fnu1, 0.0);
    real nufPhy = mufPhy / U[0];
    real den = k2 * d * d * dmax(kSmall, diffUNorm);
    real rd = (nuTur + nufPhy) / den;
    real fd = 1. - tanh(pow(8 * rd, 3.0));
    real psiSqr = Chi <= 0 ? 100.0 : dmin(100.0, (1 - C::cb1 / (cw1 * k2 * 0.424) * (ft2 + (1 - ft2) * fnu2)) / (fnu1 * dmax(kSmall, 1 - ft2)));
    real psi = sqrt(dmax(psiSqr, 1.0));
    real lDES = lRANS - fd * dmax(0., lRANS - lLES * psi);
    {
        real alphaIDDES = 0.25 - d / hMax;
        real fB = dmin(2 * exp(-9. * alphaIDDES * alphaIDDES), 1.0);
        const real cl = 3.55, ct = 1.63;
        real rdt = nuTur / den, rdl = nufPhy / den;
        real ft = tanh(pow(ct * ct * rdt, 3.0));
        real flt = (cl * cl * rdl) * (cl * cl * rdl);
        real fl = tanh((flt * flt) * (flt * flt) * flt);
        real fe1 = 2. * exp(-(alphaIDDES >= 0 ? 11.09 : 9.0) * alphaIDDES * alphaIDDES);
        real fe2 = 1. - dmax(ft, fl);
        real fe = dmax(fe1 - 1., 0.) * psi * fe2;
        real fdTilde = dmax(fB, tanh(pow(8 * rdt, 3.0)));
        real lIDDES = fdTilde * (1 + fe) * lRANS + (1 - fdTilde) * lLES * psi;
        lDES = dmax(lLES * kSmall, lIDDES);
    }
    d = lDES;
    real Sbar = nuh / (k2 * d * d) * fnu2;
    real Sh = Sbar < -C::cnu2 * S ? S + S * (C::cnu2 * C::cnu2 * S + C::cnu3 * Sbar) / ((C::cnu3 - 2 * C::cnu2) * S - Sbar) : S + Sbar;
    real r = dmin(nuh / (Sh * (C::kappa * d) * (C::kappa * d) + kVerySmall), C::rlim);
    real g = r + C::cw2 * (pow(r, 6.0) - r);
    real cw36 = pow(C::cw3, 6.0);
    real fw = g * pow((1 + cw36) / (pow(g, 6.0) + cw36), 1. / 6.);
    real D = (cw1 * fw - C::cb1 / k2 * ft2) * (nuh / lDES) * (nuh / lDES);
    real P = C::cb1 * (1 - ft2) * (Sh + SRotCor) * nuh;
    real fn = 1;
    if (U[5] < 0)
    {
        real Chi_ = U[5] * muRef / mufPhy;
        fn = (C::cn1 + pow(Chi_, 3.0)) / (C::cn1 - pow(Chi_, 3.0));
        D = -cw1 * (nuh / lDES) * (nuh / lDES);
        P = C::cb1 * (1 - C::ct3) * fabs(S + SRotCor) * nuh;
    }
    real dd = diffRho[0] * diffNu[0] + diffRho[1] * diffNu[1] + diffRho[2] * diffNu[2];
    real nn = diffNu[0] * diffNu[0] + diffNu[1] * diffNu[1] + diffNu[2] * diffNu[2];
    if (mode == 0)
        return U[0] * (P - D + nn * C::cb2 / C::sigma) / muRef - (U[5] * fn * muRef + mufPhy) / (U[0] * C::sigma) * dd / muRef;
    return -dmin(U[0] * (dmin(P, 0.0) * 1 - D * 2) / muRef / (fabs(U[5]) + kVerySmall), -kVerySmall);
}
// fluxFace viscous part at one point (EvaluateDt.hxx:1167-1209): laminar plus, for the SA model,
// mu_t (with Pr_t = 0.9 heat conduction) and the nuTilde diffusion flux
template <int NV>
DNDSB_D void point_viscous_flux(const EulerSettingsD &s, const real *UM, const real *GP, const real *n, bool adiabatic, real *Fv)
{
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    real pM, a2M, HM;
    gas_thermal(UM[4], UM[0], (UM[1] * UM[1] + UM[2] * UM[2] + UM[3] * UM[3]) / (UM[0] * UM[0]), gamma, pM, a2M, HM);
    real Tm = pM / ((gamma - 1) / gamma * cp * UM[0]);
    real mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, UM[0], Tm);
    if (NV == 6)
    {
        real muTur = sa_mu_tur(UM, s.muGas, mu);
        viscous_flux<NV>(UM, GP, n, adiabatic, gamma, mu + muTur, cp * muTur / 0.9 + cp * mu / s.prGas, cp, Fv);
        Fv[NV - 1] = sa_diffusion_flux(UM, GP, n, s.muGas, mu);
    }
    else
        viscous_flux<NV>(UM, GP, n, adiabatic, gamma, mu, cp * mu / s.prGas, cp, Fv);
}
} // namespace dndsb
