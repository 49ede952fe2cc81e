// Spalart-Allmaras model terms of the NS_SA model (6 conservative variables, the sixth being
// rho nuTilde / muRef): eddy viscosity, the nuTilde diffusion flux, the passive-scalar upwind flux
// and the source term with its diagonal Jacobian.  Settings are the reference defaults (SADESMode
// 1 IDDES shielding, rotation correction on, SAVersion 0) and its compiled options (negative-SA
// model, ft2 term).  The state-dependent routines are templated on the scalar type: real for the
// residual, dual numbers for its derivatives.
#pragma once
#include "solver.cuh"
#include "dual.cuh"

namespace dndsb
{
struct SAConst
{
    static constexpr real cb1 = 0.1355, cb2 = 0.622, sigma = 2.0 / 3.0, cnu1 = 7.1, cnu2 = 0.7, cnu3 = 0.9, cw2 = 0.3, cw3 = 2,
                          kappa = 0.41, rlim = 10, cn1 = 16.0, ct3 = 1.2, ct4 = 0.5;
};

// EulerEvaluator.hpp:791-833 getMuTur (chi smoothed below 10 by the negative-SA model)
template <typename T>
DNDSB_HD T sa_mu_tur(const T *U, real muRef, const T &muf)
{
    T Chi = U[5] * muRef / muf;
    if (Chi < 10)
        Chi = 0.05 * log(1 + exp(20 * Chi));
    T Chi3 = Chi * Chi * Chi;
    T fnu1 = Chi3 / (Chi3 + SAConst::cnu1 * SAConst::cnu1 * SAConst::cnu1);
    return muf * dmax(Chi * fnu1, 0.0);
}

// EulerEvaluator.hpp:835-877 visFluxTurVariable: the nuTilde diffusion flux through n (GP is the
// primitive gradient [3][6], the sixth column d(U5 / rho))
template <typename T>
DNDSB_HD T sa_diffusion_flux(const T *U, const T *GP, const real *n, real muRef, const T &mufPhy)
{
    T fn = 1;
    if (U[5] < 0)
    {
        T Chi = U[5] * muRef / mufPhy;
        fn = (SAConst::cn1 + Chi * Chi * Chi) / (SAConst::cn1 - Chi * Chi * Chi);
    }
    return (GP[0 * 6 + 5] * n[0] + GP[1 * 6 + 5] * n[1] + GP[2 * 6 + 5] * n[2]) * (mufPhy + U[5] * muRef * fn) / SAConst::sigma;
}

// EulerEvaluator_EvaluateDt.hxx:1413-1425: upwind flux of the SA variable with the Riemann
// solver's lam123 as dissipation speed (ransEigScheme 0)
template <typename T>
DNDSB_HD T sa_convective_flux(const T *UL, const T *UR, const real *n, const T &lam123)
{
    T vnL = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) / UL[0];
    T vnR = (UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2]) / UR[0];
    return ((vnL * UL[5] + vnR * UR[5]) - (UR[5] - UL[5]) * lam123) * 0.5;
}

// RANS_ke.hpp:985-1195 GetSource_SA: mode 0 the source of the SA equation, mode 1 its diagonal
// Jacobian; G is the conservative gradient [3][6]
template <typename T>
DNDSB_HD T sa_source(const T *U, const T *G, real muRef, const T &mufPhy, real d, real lLES, real hMax, int mode)
{
    using C = SAConst;
    const real cw1 = C::cb1 / (C::kappa * C::kappa) + (1 + C::cb2) / C::sigma;
    const real k2 = C::kappa * C::kappa;
    T nuh = U[5] * muRef / U[0];
    T Chi = U[5] * muRef / mufPhy;
    T Chi3 = Chi * Chi * Chi;
    T fnu1 = Chi3 / (Chi3 + C::cnu1 * C::cnu1 * C::cnu1);
    T fnu2 = 1 - Chi / (1 + Chi * fnu1);
    T velo[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
    T diffRho[3], diffNu[3], diffU[3][3];
    for (int i = 0; i < 3; i++)
    {
        diffRho[i] = G[i * 6 + 0];
        diffNu[i] = (G[i * 6 + 5] * muRef - nuh * diffRho[i]) / U[0];
        for (int j = 0; j < 3; j++)
            diffU[i][j] = (G[i * 6 + 1 + j] - diffRho[i] * velo[j]) / U[0];
    }
    T om2 = 0, ss2 = 0, du2 = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
        {
            T o = 0.5 * (diffU[j][i] - diffU[i][j]);
            T sij = diffU[i][j] + diffU[j][i];
            om2 += o * o, ss2 += sij * sij, du2 += diffU[i][j] * diffU[i][j];
        }
    T S = sqrt(om2) * sqrt(2.0);
    T SS = sqrt(ss2) * (1. / sqrt(2.0));
    T SRotCor = 2.0 * dmin(0.0, S - SS);
    T diffUNorm = sqrt(du2);
    T ft2 = C::ct3 * exp(-C::ct4 * Chi * Chi);
    // DDES shielding, then the IDDES blend (SADESMode 1)
    T lRANS = d;
    T nuTur = mufPhy / U[0] * dmax(Chi * fnu1, 0.0);
    T nufPhy = mufPhy / U[0];
    T den = k2 * d * d * dmax(kSmall, diffUNorm);
    T rd = (nuTur + nufPhy) / den;
    T fd = 1. - tanh(pow(8 * rd, 3.0));
    T psiSqr = Chi <= 0 ? T(100.0) : dmin(100.0, (1 - C::cb1 / (cw1 * k2 * 0.424) * (ft2 + (1 - ft2) * fnu2)) / (fnu1 * dmax(kSmall, 1 - ft2)));
    T psi = sqrt(dmax(psiSqr, 1.0));
    T lDES = lRANS - fd * dmax(0., lRANS - lLES * psi);
    {
        real alphaIDDES = 0.25 - d / hMax;
        real fB = dmin(2 * exp(-9. * alphaIDDES * alphaIDDES), 1.0);
        const real cl = 3.55, ct = 1.63;
        T rdt = nuTur / den, rdl = nufPhy / den;
        T ft = tanh(pow(ct * ct * rdt, 3.0));
        T flt = (cl * cl * rdl) * (cl * cl * rdl);
        T fl = tanh((flt * flt) * (flt * flt) * flt);
        real fe1 = 2. * exp(-(alphaIDDES >= 0 ? 11.09 : 9.0) * alphaIDDES * alphaIDDES);
        T fe2 = 1. - dmax(ft, fl);
        T fe = dmax(fe1 - 1., 0.) * psi * fe2;
        T fdTilde = dmax(fB, tanh(pow(8 * rdt, 3.0)));
        T lIDDES = fdTilde * (1 + fe) * lRANS + (1 - fdTilde) * lLES * psi;
        lDES = dmax(lLES * kSmall, lIDDES);
    }
    const T dL = lDES; // d = lDES in the reference
    T Sbar = nuh / (k2 * dL * dL) * fnu2;
    T Sh = Sbar < -C::cnu2 * S ? T(S + S * (C::cnu2 * C::cnu2 * S + C::cnu3 * Sbar) / ((C::cnu3 - 2 * C::cnu2) * S - Sbar)) : T(S + Sbar);
    T r = dmin(nuh / (Sh * (C::kappa * dL) * (C::kappa * dL) + kVerySmall), C::rlim);
    T g = r + C::cw2 * (pow(r, 6.0) - r);
    real cw36 = pow(C::cw3, 6.0);
    T fw = g * pow((1 + cw36) / (pow(g, 6.0) + cw36), 1. / 6.);
    T D = (cw1 * fw - C::cb1 / k2 * ft2) * (nuh / lDES) * (nuh / lDES);
    T P = C::cb1 * (1 - ft2) * (Sh + SRotCor) * nuh;
    T fn = 1;
    if (U[5] < 0)
    {
        T Chi_ = U[5] * muRef / mufPhy;
        fn = (C::cn1 + pow(Chi_, 3.0)) / (C::cn1 - pow(Chi_, 3.0));
        D = -cw1 * (nuh / lDES) * (nuh / lDES);
        P = C::cb1 * (1 - C::ct3) * fabs(S + SRotCor) * nuh;
    }
    T dd = diffRho[0] * diffNu[0] + diffRho[1] * diffNu[1] + diffRho[2] * diffNu[2];
    T nn = diffNu[0] * diffNu[0] + diffNu[1] * diffNu[1] + diffNu[2] * diffNu[2];
    if (mode == 0)
        return U[0] * (P - D + nn * C::cb2 / C::sigma) / muRef - (U[5] * fn * muRef + mufPhy) / (U[0] * C::sigma) * dd / muRef;
    return -dmin(U[0] * (dmin(P, 0.0) * 1 - D * 2) / muRef / (fabs(U[5]) + kVerySmall), -kVerySmall);
}
// fluxFace viscous part at one point (EvaluateDt.hxx:1167-1209): laminar plus, for the SA model,
// mu_t (with Pr_t = 0.9 heat conduction) and the nuTilde diffusion flux
template <int NV, typename T>
DNDSB_D void point_viscous_flux(const EulerSettingsD &s, const T *UM, const T *GP, const real *n, bool adiabatic, T *Fv)
{
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    T pM, a2M, HM;
    gas_thermal(UM[4], UM[0], T((UM[1] * UM[1] + UM[2] * UM[2] + UM[3] * UM[3]) / (UM[0] * UM[0])), gamma, pM, a2M, HM);
    T Tm = pM / ((gamma - 1) / gamma * cp * UM[0]);
    T mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, UM[0], Tm);
    if (NV == 6)
    {
        T muTur = sa_mu_tur(UM, s.muGas, mu);
        viscous_flux<NV>(UM, GP, n, adiabatic, gamma, mu + muTur, cp * muTur / 0.9 + cp * mu / s.prGas, cp, Fv);
        Fv[NV - 1] = sa_diffusion_flux(UM, GP, n, s.muGas, mu);
    }
    else
        viscous_flux<NV>(UM, GP, n, adiabatic, gamma, mu, cp * mu / s.prGas, cp, Fv);
}
} // namespace dndsb
