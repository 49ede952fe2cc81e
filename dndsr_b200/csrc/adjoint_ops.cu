// Building blocks of the steady adjoint solve.
//
// * The transposed LU-SGS operator: LUSGSMatrixVec (EulerEvaluator.hxx:175-274) is
//     (A x)_c = D_c x_c + sum_o w_co (J(u_o; n_co) - lambda_f I) x_o,   w_co = alpha A_f / (2 V_c),
//   with J(u; n) dU the flux-increment Jacobian of Gas.hpp:462-513.  Its transpose is
//     (A^T y)_q = D_q y_q + sum_c w_cq (J(u_q; n_cq) - lambda_f I)^T y_c,
//   where n_cq is the normal out of the neighbour c.  k_matvec_t applies it; k_sgs_color_t is one
//   multicolour Gauss-Seidel sweep on A^T y = b, the transpose of UpdateSGS (EulerEvaluator.hxx:550-693).
//   A forward sweep followed by a backward one is the symmetric Gauss-Seidel preconditioner of A^T.
// * The pressure-force objective on one boundary zone and its gradient with respect to u and uRec.
//
// One thread per cell (per boundary cell for the objective); fixed loop orders, no atomics on data.
#include "solver.cuh"
#include "basis_eval.cuh"
#include "flux_t.cuh"

namespace dndsb
{
namespace
{
// contribution of neighbour slot k (neighbour c, possibly q itself across a periodic face) to (A^T y)_q:
// w_cq (J(u_q; n_cq) - lambda)^T y_c, with n_cq the normal out of c and w_cq = alpha A_f / (2 V_c)
template <int NV>
DNDSB_D void neighbour_term_t(const MeshD &m, const GeomD &g, real gamma, const real *lamFace, real alphaDiag, int64_t q, int k, int64_t c,
                              const real *u, const real *yc, real *t)
{
    int fp = m.cell2face[q * m.nf + k];
    int64_t f = fp >> 1;
    real sg = (fp & 1) ? 1.0 : -1.0;
    real n[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
    real r[NV];
    flux_jac_du_t<NV>(u + q * NV, n, yc, lamFace[f], gamma, r);
    real w = 0.5 * alphaDiag * g.faceArea[f] / g.vol[c];
    for (int v = 0; v < NV; v++)
        t[v] = w * r[v];
}

template <int NV>
DNDSB_GLOBAL void k_matvec_t(MeshD m, GeomD g, real gamma, const real *__restrict__ lamFace, real alphaDiag, const real *__restrict__ u,
                             const real *__restrict__ y, const real *__restrict__ jdiag, real *ATy)
{
    DNDSB_KERNEL_LOOP(q, m.nCell)
    {
        real buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = 0;
        for (int k = 0; k < m.nf; k++)
        {
            int64_t c = m.cellNbr[q * m.nf + k];
            if (c < 0)
                continue;
            real t[NV];
            neighbour_term_t<NV>(m, g, gamma, lamFace, alphaDiag, q, k, c, u, y + c * NV, t);
            for (int v = 0; v < NV; v++)
                buf[v] += t[v];
        }
        for (int v = 0; v < NV; v++)
            ATy[q * NV + v] = jdiag[NV == 6 ? q * NV + v : q] * y[q * NV + v] + buf[v];
    }
}

// TY: the precision of b, y and yNew (the transposed sweep as an FP32 preconditioner reads and writes
// float vectors; the operator coefficients come from the FP64 state and are applied in FP64)
template <int NV, typename TY>
DNDSB_GLOBAL void k_sgs_color_t(MeshD m, GeomD g, real gamma, const real *__restrict__ lamFace, const int32_t *__restrict__ cellColor,
                                int64_t cBeg, int64_t cEnd, int color, real alphaDiag, const TY *__restrict__ b, const real *__restrict__ u,
                                const TY *__restrict__ y, TY *yNew, const real *__restrict__ jdiag, int forward, int gsUpdate)
{
    DNDSB_KERNEL_LOOP(ii, cEnd - cBeg)
    {
        int64_t q = m.colorCells[cBeg + ii];
        real buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = (real)b[q * NV + v];
        for (int k = 0; k < m.nf; k++)
        {
            int o = m.cellNbr[q * m.nf + k];
            if (o < 0 || o == q)
                continue;
            int oc = cellColor[o];
            bool useNew = gsUpdate && (forward ? oc < color : oc > color);
            const TY *src = (useNew ? yNew : y) + (int64_t)o * NV;
            real yo[NV], t[NV];
            for (int v = 0; v < NV; v++)
                yo[v] = (real)src[v];
            neighbour_term_t<NV>(m, g, gamma, lamFace, alphaDiag, q, k, o, u, yo, t);
            for (int v = 0; v < NV; v++)
                buf[v] -= t[v];
        }
        for (int v = 0; v < NV; v++)
            yNew[q * NV + v] = (TY)(buf[v] / jdiag[NV == 6 ? q * NV + v : q]);
    }
}

// J = sum over the zone's faces and Gauss points of |J| w p(U_L) (n . dir), U_L = u + phi . uRec of the
// face's cell; per boundary cell: its share of J and its rows of dJ/du, dJ/duRec
template <int DIM, int P, int NV>
DNDSB_GLOBAL void k_pressure_force(MeshD m, GeomD g, VRD vr, real gamma, int zone, real d0, real d1, real d2, const real *__restrict__ u,
                                   const real *__restrict__ uRec, real *Jpart, real *gU, real *gRec)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(ii, m.nBndCell)
    {
        int64_t c = m.bndCell[ii];
        real Jc = 0, aU[NV], aR[R * NV];
        for (int v = 0; v < NV; v++)
            aU[v] = 0;
        for (int j = 0; j < R * NV; j++)
            aR[j] = 0;
        bool any = false;
        for (int k = 0; k < m.nf; k++)
        {
            if (m.cellNbr[c * m.nf + k] >= 0)
                continue;
            int64_t f = m.cell2face[c * m.nf + k] >> 1;
            if (m.faceZone[f] != zone)
                continue;
            any = true;
            for (int q = 0; q < g.nGf; q++)
            {
                const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
                const real *p0 = &g.facePP[(f * g.nGf + q) * 3];
                real T0[NDOF];
                cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], &vr.baseMoment[c * NDOF], vr.s.anisotropicLengths, p0, 1, T0);
                real UL[NV];
                for (int v = 0; v < NV; v++)
                {
                    real a = 0;
                    for (int j = 0; j < R; j++)
                        a += T0[1 + j] * uRec[(c * R + j) * NV + v];
                    UL[v] = u[c * NV + v] + a;
                }
                real vel[3] = {UL[1] / UL[0], UL[2] / UL[0], UL[3] / UL[0]};
                real pr = (gamma - 1) * (UL[4] - 0.5 * UL[0] * dot3(vel, vel));
                real wt = g.faceJDet[f * g.nGf + q] * g.faceQw[q] * (n[0] * d0 + n[1] * d1 + n[2] * d2);
                Jc += wt * pr;
                real dp[NV];
                for (int v = 0; v < NV; v++)
                    dp[v] = 0;
                dp[0] = (gamma - 1) * 0.5 * dot3(vel, vel);
                for (int d = 0; d < 3; d++)
                    dp[1 + d] = -(gamma - 1) * vel[d];
                dp[4] = gamma - 1;
                for (int v = 0; v < NV; v++)
                {
                    aU[v] += wt * dp[v];
                    for (int j = 0; j < R; j++)
                        aR[j * NV + v] += wt * T0[1 + j] * dp[v];
                }
            }
        }
        Jpart[ii] = Jc;
        if (any && gU)
            for (int v = 0; v < NV; v++)
                gU[c * NV + v] = aU[v];
        if (any && gRec)
            for (int j = 0; j < R * NV; j++)
                gRec[c * R * NV + j] = aR[j];
    }
}

template <int DIM, int NV>
int launch_force(int P, const MeshD &m, const GeomD &g, const VRD &vr, real gamma, int zone, const real *dir, const real *u, const real *uRec,
                 real *Jpart, real *gU, real *gRec, cudaStream_t st)
{
    switch (P)
    {
    case 1:
        DNDSB_LAUNCH((k_pressure_force<DIM, 1, NV>), m.nBndCell, 64, st, m, g, vr, gamma, zone, dir[0], dir[1], dir[2], u, uRec, Jpart, gU, gRec);
        return ST_OK;
    case 2:
        DNDSB_LAUNCH((k_pressure_force<DIM, 2, NV>), m.nBndCell, 64, st, m, g, vr, gamma, zone, dir[0], dir[1], dir[2], u, uRec, Jpart, gU, gRec);
        return ST_OK;
    case 3:
        DNDSB_LAUNCH((k_pressure_force<DIM, 3, NV>), m.nBndCell, 64, st, m, g, vr, gamma, zone, dir[0], dir[1], dir[2], u, uRec, Jpart, gU, gRec);
        return ST_OK;
    }
    return ST_UNSUPPORTED;
}
} // namespace

int lusgs_matvec_t(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *y, const real *jdiag, real *ATy,
                   cudaStream_t st)
{
    if (ev.s.nVars == 5)
        DNDSB_LAUNCH(k_matvec_t<5>, m.nCell, 256, st, m, g, ev.s.gamma, ev.lambdaFace, alphaDiag, u, y, jdiag, ATy);
    else if (ev.s.nVars == 6)
        DNDSB_LAUNCH(k_matvec_t<6>, m.nCell, 256, st, m, g, ev.s.gamma, ev.lambdaFace, alphaDiag, u, y, jdiag, ATy);
    else
        return ST_UNSUPPORTED;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int update_sgs_t(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const void *b, const real *u, const void *y, void *yNew,
                 const real *jdiag, int forward, int gsUpdate, int fp32, cudaStream_t st)
{
    int nv = ev.s.nVars;
    for (int ci = 0; ci < m.nColor; ci++)
    {
        int col = forward ? ci : m.nColor - 1 - ci;
        int64_t bb = m.colorStart[col], e = m.colorStart[col + 1];
#define DNDSB_SGST(NVV, TY)                                                                                                               \
    DNDSB_LAUNCH((k_sgs_color_t<NVV, TY>), e - bb, 128, st, m, g, ev.s.gamma, ev.lambdaFace, m.cellColor, bb, e, col, alphaDiag, (const TY *)b, u, \
                 (const TY *)y, (TY *)yNew, jdiag, forward, gsUpdate)
        if (nv == 5 && !fp32)
            DNDSB_SGST(5, real);
        else if (nv == 5)
            DNDSB_SGST(5, float);
        else if (nv == 6 && !fp32)
            DNDSB_SGST(6, real);
        else if (nv == 6)
            DNDSB_SGST(6, float);
        else
            return ST_UNSUPPORTED;
#undef DNDSB_SGST
    }
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int pressure_force(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, int zone, const real *dir, const real *u, const real *uRec,
                   real *Jhost, real *gU, real *gRec, cudaStream_t st)
{
    int nv = ev.s.nVars;
    if (gU && dev_zero(gU, sizeof(real) * m.nCell * nv, st) != cudaSuccess)
        return ST_CUDA;
    if (gRec && dev_zero(gRec, sizeof(real) * m.nCell * vr.R * nv, st) != cudaSuccess)
        return ST_CUDA;
    if (m.nBndCell == 0)
    {
        *Jhost = 0;
        return ST_OK;
    }
    // per boundary cell shares in the [nFace][nv] scratch (nBndCell <= nFace)
    real *Jpart = ev.faceFlux;
    int rc = ST_UNSUPPORTED;
    if (m.dim == 2 && nv == 5)
        rc = launch_force<2, 5>(vr.P, m, g, vr, ev.s.gamma, zone, dir, u, uRec, Jpart, gU, gRec, st);
    else if (m.dim == 3 && nv == 5)
        rc = launch_force<3, 5>(vr.P, m, g, vr, ev.s.gamma, zone, dir, u, uRec, Jpart, gU, gRec, st);
    else if (m.dim == 3 && nv == 6)
        rc = launch_force<3, 6>(vr.P, m, g, vr, ev.s.gamma, zone, dir, u, uRec, Jpart, gU, gRec, st);
    if (rc != ST_OK)
        return rc;
    return reduce_norm(m.nBndCell, 1, Jpart, nullptr, 0, 0, ev.redBuf, Jhost, st);
}
} // namespace dndsb
