// Positivity-preserving increment limiting of the implicit update (EulerSolver.hxx:696-738):
//   EvaluateCellRHSAlpha (EulerEvaluator.hxx:1938-2062) -- per-cell alpha that keeps the density and
//     the pressure of u + alpha inc above relaxed floors, with the quadratic pressure bound of
//     IdealGasGetCompressionRatioPressure (Gas.hpp:1750-1860, scheme 0);
//   EvaluateCellRHSAlphaExpansion (EulerEvaluator.hxx:2064-2140);
//   AddFixedIncrement (EulerEvaluator.hpp:1795-1857) -- u += CompressInc(u, alpha inc)
//     (EulerEvaluator.hpp:1645-1773).
// One thread per cell.  The reference's assertions set DE_NONPHYSICAL in the error word instead of
// aborting.  The count of limited cells and the minima are integer and min reductions (atomicAdd
// on an integer, atomicMin on the bits of a non-negative double), so they do not depend on order.
#include "solver.cuh"

#include <cmath>
#include <cstring>

namespace dndsb
{
namespace
{
constexpr real kPPSmall = 1e-10; // DNDS/Defines.hpp:201 smallReal

DNDSB_D real pp_rhoE(const real *u) { return u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]; }

DNDSB_D void atomic_min_nonneg(unsigned long long *bits, real v)
{
    atomicMin(bits, (unsigned long long)__double_as_longlong(v));
}

// Gas.hpp:1750-1860, scheme 0: the largest alpha keeping rho e of u + alpha inc above newRhoE
DNDSB_D real compression_ratio_pressure(const real *u, const real *inc, real newRhoE, bool &bad)
{
    const real safety = 1 - 1e-5;
    real r[5], un[5];
    for (int i = 0; i < 5; i++)
        r[i] = inc[i], un[i] = u[i] + inc[i];
    const real m2 = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
    const real rhoEOld = u[4] - m2 / (u[0] + kVerySmall) * 0.5;
    newRhoE = fmax(kPPSmall * rhoEOld, newRhoE);
    const real rhoENew = un[4] - (un[1] * un[1] + un[2] * un[2] + un[3] * un[3]) / (un[0] + kVerySmall) * 0.5;
    real alpha;
    const real c0 = 2 * u[4] * u[0] - m2 - 2 * u[0] * newRhoE;
    const real c1 = 2 * u[4] * r[0] + 2 * u[0] * r[4] - 2 * (u[1] * r[1] + u[2] * r[2] + u[3] * r[3]) - 2 * r[0] * newRhoE;
    real c2 = 2 * r[4] * r[0] - (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    c2 += (c2 >= 0 ? 1 : -1) * kVerySmall;
    real dC = c1 * c1 - 4 * c0 * c2;
    if (dC <= -c0 * c0 * kPPSmall)
        bad = true;
    dC = fmax(0.0, dC);
    const real aL = (-sqrt(dC) - c1) / (2 * c2);
    (void)rhoENew;
    if (fabs(c2) < 1e-10 * c0)
        alpha = fabs(c1) < 1e-10 * c0 ? 0.0 : fmin(-c0 / c1, 1.0);
    else
        alpha = fmin(aL, 1.0);
    alpha = fmax(0.0, alpha) * safety;
    if (alpha < kPPSmall)
        alpha = 0;
    for (int i = 0; i < 5; i++)
        r[i] *= alpha;
    int it = 0;
    for (; it < 1000; it++)
    {
        const real s0 = u[1] + r[1], s1 = u[2] + r[2], s2 = u[3] + r[3];
        const real ek = 0.5 * (s0 * s0 + s1 * s1 + s2 * s2) / (u[0] + r[0] + kVerySmall);
        if (r[4] + u[4] - ek < newRhoE)
        {
            for (int i = 0; i < 5; i++)
                r[i] *= 1 - 1e-2;
            alpha *= 1 - 1e-2;
        }
        else
            break;
    }
    if (it >= 1000)
        bad = true;
    return alpha;
}

DNDSB_GLOBAL void k_cell_rhs_alpha(int64_t nCell, int nv, real gamma, const real *__restrict__ u, const real *__restrict__ res,
                                   real *__restrict__ alpha, real rhoEps, real pEps, real relax, real power, unsigned long long *nLim,
                                   unsigned long long *aMinBits, int *err)
{
    const real safety = 1 - 1e-5;
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        const real *uc = u + c * nv;
        real ucl[5], inc[5];
        for (int i = 0; i < 5; i++)
            ucl[i] = uc[i], inc[i] = res[c * nv + i];
        bool bad = !(ucl[0] >= rhoEps);
        real aRho = 1;
        const real relRho = rhoEps * relax + ucl[0] * (1 - relax);
        if (inc[0] < 0)
            aRho = fmin(1.0, (ucl[0] - relRho) / (-inc[0] - kPPSmall * inc[0]));
        bad = bad || !(aRho >= 0 && aRho <= 1);
        real un[5];
        for (int i = 0; i < 5; i++)
            inc[i] *= aRho, un[i] = ucl[i] + inc[i];
        const real pNew = pp_rhoE(un) * (gamma - 1), pOld = pp_rhoE(ucl) * (gamma - 1);
        real relP = pEps;
        if (pNew < pOld)
            relP = pEps + (pOld - pEps) * (1 - relax);
        real aP = 1;
        if (pNew < relP)
            aP = fmin(aP, compression_ratio_pressure(ucl, inc, relP / (gamma - 1), bad));
        real a = aRho * aP;
        if (a < 1)
        {
            a = pow(a, power);
            atomicAdd(nLim, 1ull);
            a *= safety;
            atomic_min_nonneg(aMinBits, a);
        }
        alpha[c] = a;
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}

// flags EvaluateCellRHSAlpha_MIN_IF_NOT_ONE (1) and _MIN_ALL (2) with the reduced minimum
DNDSB_GLOBAL void k_alpha_flags(int64_t nCell, int flag, real *__restrict__ alpha, const unsigned long long *aMinBits)
{
    const real aMin = __longlong_as_double((long long)*aMinBits);
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        if ((flag & 1) && alpha[c] < 1)
            alpha[c] = aMin;
        if (flag & 2)
            alpha[c] = aMin;
    }
}

DNDSB_GLOBAL void k_alpha_expansion(int64_t nCell, int nv, real gamma, const real *__restrict__ u, const real *__restrict__ res,
                                    real *__restrict__ alpha, real rhoEps, real pEps, real alphaMin)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        real un[5];
        for (int i = 0; i < 5; i++)
            un[i] = u[c * nv + i] + res[c * nv + i];
        if (pp_rhoE(un) * (gamma - 1) < pEps || un[0] < rhoEps)
            alpha[c] = alphaMin;
    }
}

// EulerEvaluator.hpp:1645-1773 CompressInc, then u += it (AddFixedIncrement)
DNDSB_GLOBAL void k_add_fixed_increment(int64_t nCell, int nv, real gamma, real *__restrict__ u, const real *__restrict__ inc, real alpha,
                                        real rhoEps, real pEps, unsigned long long *fixMinBits, int *err)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        real uc[6], ret[6], a0;
        for (int i = 0; i < nv; i++)
            uc[i] = u[c * nv + i], ret[i] = inc[c * nv + i] * alpha;
        a0 = ret[0];
        bool bad = !(uc[0] > 0);
        if (uc[0] + ret[0] <= rhoEps)
        {
            const real f = (rhoEps - uc[0]) / (ret[0] - kVerySmall);
            for (int i = 0; i < nv; i++)
                ret[i] *= f;
        }
        const real rhoEint = uc[4] - 0.5 * (uc[1] * uc[1] + uc[2] * uc[2] + uc[3] * uc[3]) / (uc[0] + kVerySmall);
        bad = bad || !(rhoEint > 0);
        auto ek_of = [&]()
        {
            const real s0 = uc[1] + ret[1], s1 = uc[2] + ret[2], s2 = uc[3] + ret[3];
            return 0.5 * (s0 * s0 + s1 * s1 + s2 * s2) / (uc[0] + ret[0] + kVerySmall);
        };
        const real rhoEintNew = uc[4] + ret[4] - ek_of();
        if (rhoEintNew <= pEps)
        {
            const real e = pEps / (gamma - 1);
            const real m2 = uc[1] * uc[1] + uc[2] * uc[2] + uc[3] * uc[3];
            const real c0 = 2 * uc[4] * uc[0] - m2 - 2 * uc[0] * e;
            const real c1 = 2 * uc[4] * ret[0] + 2 * uc[0] * ret[4] - 2 * (uc[1] * ret[1] + uc[2] * ret[2] + uc[3] * ret[3]) - 2 * ret[0] * e;
            const real c2 = 2 * ret[4] * ret[0] - (ret[1] * ret[1] + ret[2] * ret[2] + ret[3] * ret[3]);
            const real dC = c1 * c1 - 4 * c0 * c2;
            bad = bad || !(dC > 0);
            const real al = fmax(0.0, fmin((-sqrt(fmax(dC, 0.0)) - c1) / (2 * c2), 1.0));
            for (int i = 0; i < nv; i++)
                ret[i] *= al * 0.99;
            for (int it = 0; it < 1000; it++)
            {
                if (ret[4] + uc[4] - ek_of() < e)
                    for (int i = 0; i < nv; i++)
                        ret[i] *= 1 - 1e-1;
                else
                    break;
            }
            bad = bad || ret[4] + uc[4] - ek_of() < e * 0.5;
        }
        if (nv > 5 && uc[5] + ret[5] < 0)
        {
            bad = bad || uc[5] < 0;
            const real nu = fmax(1e-6, uc[5] * exp(ret[5] / (uc[5] + 1e-6)));
            ret[5] = nu - uc[5];
        }
        real na = fabs(ret[0]) / fabs(a0);
        if (fabs(a0) < kVerySmall)
            na = 1.;
        atomic_min_nonneg(fixMinBits, na);
        for (int i = 0; i < nv; i++)
            u[c * nv + i] = uc[i] + ret[i];
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}

// rho and p floors of the reference: smallReal * refUPrim * 0.1
void pp_eps(real refRho, real refP, real &rhoEps, real &pEps)
{
    rhoEps = kPPSmall * refRho * 1e-1, pEps = kPPSmall * refP * 1e-1;
}

// the reductions' words live in the evaluator's reduction scratch: [0] count, [1] minimum bits
int pp_read(EvalD &ev, int64_t *count, real *minOut, cudaStream_t st)
{
    unsigned long long h[2] = {0, 0};
    int e = 0;
    d2h(h, ev.redBuf, sizeof(h), st);
    d2h(&e, ev.errWord, sizeof(int), st);
    if (last_error() != cudaSuccess || dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    if (count)
        *count = (int64_t)h[0];
    if (minOut)
    {
        long long b = (long long)h[1];
        std::memcpy(minOut, &b, sizeof(real));
    }
    return (e & DE_NONPHYSICAL) ? ST_NONPHYSICAL : ST_OK;
}

int pp_init(EvalD &ev, cudaStream_t st)
{
    static const unsigned long long init[2] = {0ull, 0x3FF0000000000000ull}; // 0 and the bits of 1.0
    if (h2d(ev.redBuf, init, sizeof(init), st) != cudaSuccess || dev_zero(ev.errWord, sizeof(int), st) != cudaSuccess)
        return ST_CUDA;
    return ST_OK;
}
} // namespace

int cell_rhs_alpha(const MeshD &m, EvalD &ev, const real *u, const real *res, real *alpha, real refRho, real refP, real relax, int compress,
                   real compressPower, int ppEpsIsRelaxed, int flag, int64_t *nLim, real *alphaMin, cudaStream_t st)
{
    real rhoEps, pEps;
    pp_eps(refRho, refP, rhoEps, pEps);
    if (ppEpsIsRelaxed)
        pEps *= 0, rhoEps *= 0;
    if (pp_init(ev, st) != ST_OK)
        return ST_CUDA;
    const real power = (real)(compress * (int)std::lround(compressPower));
    auto *words = (unsigned long long *)ev.redBuf;
    DNDSB_LAUNCH(k_cell_rhs_alpha, m.nCell, 256, st, m.nCell, ev.s.nVars, ev.s.gamma, u, res, alpha, rhoEps, pEps, relax, power, words, words + 1,
                 ev.errWord);
    if (flag & 3)
        DNDSB_LAUNCH(k_alpha_flags, m.nCell, 256, st, m.nCell, flag, alpha, words + 1);
    return pp_read(ev, nLim, alphaMin, st);
}

int cell_rhs_alpha_expansion(const MeshD &m, EvalD &ev, const real *u, const real *res, real *alpha, real refRho, real refP, real alphaMin,
                             cudaStream_t st)
{
    real rhoEps, pEps;
    pp_eps(refRho, refP, rhoEps, pEps);
    DNDSB_LAUNCH(k_alpha_expansion, m.nCell, 256, st, m.nCell, ev.s.nVars, ev.s.gamma, u, res, alpha, rhoEps, pEps, alphaMin);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int add_fixed_increment(const MeshD &m, EvalD &ev, real *u, const real *inc, real alpha, real refRho, real refP, int ppEpsIsRelaxed,
                        real *alphaFixMin, cudaStream_t st)
{
    real rhoEps, pEps;
    pp_eps(refRho, refP, rhoEps, pEps);
    if (ppEpsIsRelaxed)
        pEps *= kVerySmall, rhoEps *= kVerySmall;
    if (pp_init(ev, st) != ST_OK)
        return ST_CUDA;
    auto *words = (unsigned long long *)ev.redBuf;
    DNDSB_LAUNCH(k_add_fixed_increment, m.nCell, 256, st, m.nCell, ev.s.nVars, ev.s.gamma, u, inc, alpha, rhoEps, pEps, words + 1, ev.errWord);
    return pp_read(ev, nullptr, alphaFixMin, st);
}
} // namespace dndsb
