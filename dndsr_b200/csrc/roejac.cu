// LU-SGS operators in block mode (useScalarJacobian = false, optionally useRoeJacobian): LUSGSMatrixInit
// (EulerEvaluator.hxx:37-159), UpdateSGS (:550-693), UpdateLUSGSForward / Backward (:376-529) and
// LUSGSMatrixVec (:175-274) with a block jdiag [nCell][2][NV][NV] (block, inverse) and, with the Roe
// term, the flux increments of roejac.cuh.  One thread per cell; sweeps colour by colour as in the
// scalar kernels, so the sweep order and results match the reference's sequential sweep on a mesh
// numbered colour by colour.
#include "roejac.cuh"
#include "ilu.cuh"

namespace dndsb
{
namespace
{
using namespace roej;

template <int NV>
DNDSB_GLOBAL void k_lusgs_init_blk(MeshD m, GeomD g, BoundaryD bnd, EvalD ev, int roe, const real *__restrict__ dTau, real dt, real alphaDiag,
                                   const real *__restrict__ u, real *jd, int *err)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real B[NV * NV], Bi[NV * NV];
        cell_block<NV>(m, g, bnd, ev, roe != 0, dTau, dt, alphaDiag, u, c, B);
        bool ok = block_inv<NV>(B, Bi);
        bool fin = true;
        for (int i = 0; i < NV * NV; i++)
            fin = fin && isfinite(Bi[i]);
        if (!ok || !fin)
        {
            atomicOr(err, (int)DE_SINGULAR);
            for (int i = 0; i < NV * NV; i++)
                Bi[i] = 0;
        }
        real *o = jd + c * 2 * NV * NV;
        for (int i = 0; i < NV * NV; i++)
            o[i] = B[i], o[NV * NV + i] = Bi[i];
    }
}

// sum over the selected neighbours of w dF(u_o; dU_o), subtracted from buf (sel: 0 all, 1 GS of UpdateSGS, 2 LU-SGS lower/upper)
template <int NV>
DNDSB_D void nbr_sum(const MeshD &m, const GeomD &g, const EvalD &ev, bool roe, int64_t c, real alphaDiag, const real *u, const real *x0,
                     const real *x1, const int32_t *cellColor, int color, int forward, int gsUpdate, int uIncIsZero, int sel, real *buf)
{
    const real cf = 0.5 * alphaDiag / g.vol[c];
    for (int k = 0; k < m.nf; k++)
    {
        int o = m.cellNbr[c * m.nf + k];
        if (o < 0)
            continue;
        const real *dU;
        if (sel == 1)
        {
            if (o == c)
                continue;
            int oc = cellColor[o];
            bool useNew = gsUpdate && (forward ? oc < color : oc > color);
            if (uIncIsZero && !useNew)
                continue;
            dU = (useNew ? x1 : x0) + (int64_t)o * NV;
        }
        else if (sel == 2)
        {
            if (!(forward ? o < c : o > c))
                continue;
            dU = x0 + (int64_t)o * NV;
        }
        else
            dU = x0 + (int64_t)o * NV;
        int pk = m.cell2face[c * m.nf + k];
        int64_t f = pk >> 1;
        int side = pk & 1;
        real sg = side ? -1.0 : 1.0;
        real n[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
        FaceLam L;
        if (roe)
            L = face_lam(ev, f, side);
        else
            L.main = ev.lambdaFace[f], L.l0 = L.l123 = L.l4 = L.vis = 0;
        real dF[NV];
        nbr_inc<NV>(roe, u + (int64_t)o * NV, u + c * NV, n, dU, L, ev.s.gamma, dF);
        real w = cf * g.faceArea[f];
        for (int v = 0; v < NV; v++)
            buf[v] -= w * dF[v];
    }
}

template <int NV>
DNDSB_GLOBAL void k_sgs_color_blk(MeshD m, GeomD g, EvalD ev, int roe, int64_t cBeg, int64_t cEnd, int color, real alphaDiag,
                                  const real *__restrict__ rhs, const real *__restrict__ u, const real *__restrict__ uInc, real *uIncNew,
                                  const real *__restrict__ jd, int forward, int gsUpdate, int uIncIsZero, real *absInc)
{
    DNDSB_KERNEL_LOOP(ii, cEnd - cBeg)
    {
        int64_t c = m.colorCells[cBeg + ii];
        real buf[NV], x[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = rhs[c * NV + v];
        nbr_sum<NV>(m, g, ev, roe != 0, c, alphaDiag, u, uInc, uIncNew, m.cellColor, color, forward, gsUpdate, uIncIsZero, 1, buf);
        block_mul<NV>(jd + c * 2 * NV * NV + NV * NV, buf, x);
        for (int v = 0; v < NV; v++)
        {
            absInc[c * NV + v] = fabs(x[v] - uIncNew[c * NV + v]);
            uIncNew[c * NV + v] = x[v];
        }
    }
}

template <int NV>
DNDSB_GLOBAL void k_lusgs_sweep_blk(MeshD m, GeomD g, EvalD ev, int roe, const int32_t *__restrict__ cells, int64_t cBeg, int64_t cEnd,
                                    real alphaDiag, const real *__restrict__ rhs, const real *__restrict__ u, const real *uInc, real *uIncNew,
                                    const real *__restrict__ jd, int forward)
{
    DNDSB_KERNEL_LOOP(ii, cEnd - cBeg)
    {
        int64_t c = cells ? (int64_t)cells[cBeg + ii] : cBeg + ii;
        real buf[NV], x[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = forward ? rhs[c * NV + v] : 0.0;
        nbr_sum<NV>(m, g, ev, roe != 0, c, alphaDiag, u, uInc, nullptr, nullptr, 0, forward, 0, 0, 2, buf);
        block_mul<NV>(jd + c * 2 * NV * NV + NV * NV, buf, x);
        for (int v = 0; v < NV; v++)
            uIncNew[c * NV + v] = forward ? x[v] : uIncNew[c * NV + v] + x[v];
    }
}

template <int NV>
DNDSB_GLOBAL void k_matvec_blk(MeshD m, GeomD g, EvalD ev, int roe, real alphaDiag, const real *__restrict__ u, const real *__restrict__ uInc,
                               const real *__restrict__ jd, real *AuInc)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real buf[NV], y[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = 0;
        nbr_sum<NV>(m, g, ev, roe != 0, c, alphaDiag, u, uInc, nullptr, nullptr, 0, 0, 0, 0, 0, buf);
        block_mul<NV>(jd + c * 2 * NV * NV, uInc + c * NV, y);
        for (int v = 0; v < NV; v++)
            AuInc[c * NV + v] = y[v] - buf[v];
    }
}
// the slot blocks (alpha/2)(A_f/V_c) dF/dU_o of LUSGSMatrixToJacobianLU (EulerEvaluator.hxx:290-359), cell order
template <int NV>
DNDSB_GLOBAL void k_lu_assemble(MeshD m, GeomD g, EvalD ev, int roe, real alphaDiag, const real *__restrict__ u, real *off)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        const real cf = 0.5 * alphaDiag / g.vol[c];
        for (int k = 0; k < m.nf; k++)
        {
            real *ob = off + (c * m.nf + k) * NV * NV;
            int o = m.cellNbr[c * m.nf + k];
            if (o < 0 || o == c)
            {
                for (int i = 0; i < NV * NV; i++)
                    ob[i] = 0;
                continue;
            }
            int pk = m.cell2face[c * m.nf + k];
            int64_t f = pk >> 1;
            int side = pk & 1;
            real sg = side ? -1.0 : 1.0;
            real n[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
            FaceLam L;
            if (roe)
                L = face_lam(ev, f, side);
            else
                L.main = ev.lambdaFace[f], L.l0 = L.l123 = L.l4 = L.vis = 0;
            real w = cf * g.faceArea[f];
            for (int i = 0; i < NV; i++)
            {
                real e[NV], col[NV];
                for (int v = 0; v < NV; v++)
                    e[v] = v == i ? 1.0 : 0.0;
                nbr_inc<NV>(roe != 0, u + (int64_t)o * NV, u + c * NV, n, e, L, ev.s.gamma, col);
                for (int v = 0; v < NV; v++)
                    ob[v * NV + i] = w * col[v];
            }
        }
    }
}

// the scalar Jacobian's diagonal (one value, or one per variable) as diagonal blocks
template <int NV>
DNDSB_GLOBAL void k_diag_blocks(int64_t nCell, const real *__restrict__ jd, int nd, real *out)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        for (int i = 0; i < NV; i++)
            for (int j = 0; j < NV; j++)
                out[c * NV * NV + i * NV + j] = i == j ? jd[c * nd + (nd > 1 ? i : 0)] : 0.0;
    }
}

DNDSB_GLOBAL void k_sub(int64_t n, const real *__restrict__ a, const real *__restrict__ b, real *c)
{
    DNDSB_KERNEL_LOOP(i, n)
    c[i] = a[i] - b[i];
}

DNDSB_GLOBAL void k_abs_add(int64_t n, const real *x, real *absOut, const real *__restrict__ add, real *y) // y may be x
{
    DNDSB_KERNEL_LOOP(i, n)
    {
        absOut[i] = fabs(x[i]);
        if (add)
            y[i] = x[i] + add[i];
    }
}

// jd: the block jdiag [nCell][2][NV][NV], or (scalar Jacobian) ev.luDiag [nCell][NV][NV]
template <int NV, int NF>
void lu_factor_colors(const MeshD &m, EvalD &ev, const real *jd, cudaStream_t st)
{
    auto kf = ilu::k_ilu_factor<real, NV, NF>;
    constexpr int64_t NN = NV * NV;
    const ilu::BlockLay DL{ev.jacMode ? 2 * NN : NN, 0};
    for (int ci = 0; ci < m.nColor; ci++)
        DNDSB_LAUNCH(kf, m.colorStart[ci + 1] - m.colorStart[ci], 64, st, m.colorStart[ci], m.colorStart[ci + 1], m.colorCells, m.cellNbr,
                     m.cellColor, (const real *)ev.luOff, jd, ilu::BlockLay{NF * NN, 0}, ilu::BlockLay{NN, 0}, DL, ev.luOff, ev.luDinv, ev.errWord,
                     (int32_t *)nullptr, (int32_t *)nullptr);
}

template <int NV, int NF>
void lu_solve_colors(const MeshD &m, EvalD &ev, real *x, cudaStream_t st)
{
    auto kl = ilu::k_ilu_lower<real, NV, NF>;
    auto ku = ilu::k_ilu_upper<real, NV, NF>;
    constexpr int64_t NN = NV * NV;
    const ilu::BlockLay offL{NF * NN, 0}, dL{NN, 0};
    for (int ci = 0; ci < m.nColor; ci++)
        DNDSB_LAUNCH(kl, m.colorStart[ci + 1] - m.colorStart[ci], 128, st, m.colorStart[ci], m.colorStart[ci + 1], m.colorCells, m.cellNbr,
                     m.cellColor, (const real *)ev.luOff, offL, (const real *)x, x);
    for (int ci = m.nColor - 1; ci >= 0; ci--)
        DNDSB_LAUNCH(ku, m.colorStart[ci + 1] - m.colorStart[ci], 128, st, m.colorStart[ci], m.colorStart[ci + 1], m.colorCells, m.cellNbr,
                     m.cellColor, (const real *)ev.luOff, offL, (const real *)ev.luDinv, dL, x);
}

template <int NV>
int lu_dispatch(const MeshD &m, EvalD &ev, const real *jd, real *x, bool factor, cudaStream_t st)
{
    switch (m.nf)
    {
    case 3:
        factor ? lu_factor_colors<NV, 3>(m, ev, jd, st) : lu_solve_colors<NV, 3>(m, ev, x, st);
        return ST_OK;
    case 4:
        factor ? lu_factor_colors<NV, 4>(m, ev, jd, st) : lu_solve_colors<NV, 4>(m, ev, x, st);
        return ST_OK;
    case 6:
        factor ? lu_factor_colors<NV, 6>(m, ev, jd, st) : lu_solve_colors<NV, 6>(m, ev, x, st);
        return ST_OK;
    }
    return ST_UNSUPPORTED;
}
} // namespace

int jacobian_lu(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *jd, cudaStream_t st)
{
    int nv = ev.s.nVars;
    if (ev.jacMode == 2 && !ev.lambdaFace0)
        return ST_BADARG;
    if (nv != 5 && nv != 6)
        return ST_UNSUPPORTED;
    if (!ev.luOff && (dev_alloc((void **)&ev.luOff, sizeof(real) * nv * nv * m.nCell * m.nf) != cudaSuccess ||
                      dev_alloc((void **)&ev.luDinv, sizeof(real) * nv * nv * m.nCell) != cudaSuccess))
        return ST_CUDA;
    if (ev.jacMode == 0) // JDiag.getValue of the scalar Jacobian: its diagonal as blocks
    {
        if (!ev.luDiag && dev_alloc((void **)&ev.luDiag, sizeof(real) * nv * nv * m.nCell) != cudaSuccess)
            return ST_CUDA;
        if (nv == 5)
            DNDSB_LAUNCH(k_diag_blocks<5>, m.nCell, 256, st, m.nCell, jd, 1, ev.luDiag);
        else
            DNDSB_LAUNCH(k_diag_blocks<6>, m.nCell, 256, st, m.nCell, jd, 6, ev.luDiag);
        jd = ev.luDiag;
    }
    cudaMemsetAsync(ev.errWord, 0, sizeof(int), st);
    int roe = ev.jacMode == 2;
    if (nv == 5)
        DNDSB_LAUNCH(k_lu_assemble<5>, m.nCell, 128, st, m, g, ev, roe, alphaDiag, u, ev.luOff);
    else
        DNDSB_LAUNCH(k_lu_assemble<6>, m.nCell, 128, st, m, g, ev, roe, alphaDiag, u, ev.luOff);
    int rc = nv == 5 ? lu_dispatch<5>(m, ev, jd, nullptr, true, st) : lu_dispatch<6>(m, ev, jd, nullptr, true, st);
    if (rc != ST_OK)
        return rc;
    if (last_error() != cudaSuccess)
        return ST_CUDA;
    int e = 0;
    d2h(&e, ev.errWord, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    return (e & DE_SINGULAR) ? ST_NONFINITE : ST_OK;
}

int solve_jacobian_lu(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc, real *uIncNew,
                      const real *jd, int uIncIsZero, real *sumIncHost, cudaStream_t st)
{
    int nv = ev.s.nVars;
    if (!ev.luOff)
        return ST_BADARG;
    int64_t n = m.nCell * nv;
    if (uIncIsZero)
        d2d(uIncNew, rhs, sizeof(real) * n, st);
    else
    {
        real *ax = ev.faceFlux; // [nCell][nv] fits in the [nFace][nv] scratch
        int rc = ev.jacMode ? lusgs_matvec_block(m, g, ev, alphaDiag, u, uInc, jd, ax, st) : lusgs_matvec(m, g, ev, alphaDiag, u, uInc, jd, ax, st);
        if (rc != ST_OK)
            return rc;
        DNDSB_LAUNCH(k_sub, n, 256, st, n, rhs, (const real *)ax, uIncNew);
    }
    int rc = nv == 5 ? lu_dispatch<5>(m, ev, jd, uIncNew, false, st) : lu_dispatch<6>(m, ev, jd, uIncNew, false, st);
    if (rc != ST_OK)
        return rc;
    real *absX = ev.faceFlux;
    DNDSB_LAUNCH(k_abs_add, n, 256, st, n, (const real *)uIncNew, absX, uIncIsZero ? nullptr : uInc, uIncNew);
    if (sumIncHost)
    {
        real *res = reduce_cols(0, m.nCell, nv, absX, nullptr, 0, ev.redBuf, st);
        d2h(sumIncHost, res, sizeof(real) * nv, st);
        if (dev_sync(st) != cudaSuccess)
            return ST_CUDA;
    }
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int lusgs_init_block(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *dTau, real dt, real alphaDiag, const real *u,
                     real *jd, cudaStream_t st)
{
    int nv = ev.s.nVars;
    bool roe = ev.jacMode == 2;
    if (roe && !ev.lambdaFace0)
        return ST_BADARG;
    if (roe && m.nBndFace > 0 && !vr.bnd.type)
        return ST_BADARG;
    if (nv == 6 && !ev.jSource)
        return ST_BADARG;
    cudaMemsetAsync(ev.errWord, 0, sizeof(int), st);
    if (nv == 5)
        DNDSB_LAUNCH(k_lusgs_init_blk<5>, m.nCell, 128, st, m, g, vr.bnd, ev, (int)roe, dTau, dt, alphaDiag, u, jd, ev.errWord);
    else if (nv == 6)
        DNDSB_LAUNCH(k_lusgs_init_blk<6>, m.nCell, 128, st, m, g, vr.bnd, ev, (int)roe, dTau, dt, alphaDiag, u, jd, ev.errWord);
    else
        return ST_UNSUPPORTED;
    if (last_error() != cudaSuccess)
        return ST_CUDA;
    int e = 0;
    d2h(&e, ev.errWord, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    return (e & DE_SINGULAR) ? ST_NONFINITE : ST_OK;
}

int update_sgs_block(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc, real *uIncNew,
                     const real *jd, int forward, int gsUpdate, int uIncIsZero, real *sumIncHost, cudaStream_t st)
{
    int nv = ev.s.nVars;
    int roe = ev.jacMode == 2;
    real *absInc = ev.faceFlux; // [nCell][nv] fits in the [nFace][nv] scratch
    for (int ci = 0; ci < m.nColor; ci++)
    {
        int col = forward ? ci : m.nColor - 1 - ci;
        int64_t b = m.colorStart[col], e = m.colorStart[col + 1];
        if (nv == 5)
            DNDSB_LAUNCH(k_sgs_color_blk<5>, e - b, 128, st, m, g, ev, roe, b, e, col, alphaDiag, rhs, u, uInc, uIncNew, jd, forward, gsUpdate,
                         uIncIsZero, absInc);
        else if (nv == 6)
            DNDSB_LAUNCH(k_sgs_color_blk<6>, e - b, 128, st, m, g, ev, roe, b, e, col, alphaDiag, rhs, u, uInc, uIncNew, jd, forward, gsUpdate,
                         uIncIsZero, absInc);
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

int update_lusgs_block(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc,
                       real *uIncNew, const real *jd, int forward, cudaStream_t st)
{
    int nv = ev.s.nVars;
    int roe = ev.jacMode == 2;
    if (nv != 5 && nv != 6)
        return ST_UNSUPPORTED;
    auto launch = [&](const int32_t *cells, int64_t b, int64_t e)
    {
        if (nv == 5)
            DNDSB_LAUNCH(k_lusgs_sweep_blk<5>, e - b, 128, st, m, g, ev, roe, cells, b, e, alphaDiag, rhs, u, uInc, uIncNew, jd, forward);
        else
            DNDSB_LAUNCH(k_lusgs_sweep_blk<6>, e - b, 128, st, m, g, ev, roe, cells, b, e, alphaDiag, rhs, u, uInc, uIncNew, jd, forward);
    };
    if (uInc != uIncNew)
        launch(nullptr, 0, m.nCell);
    else
        for (int ci = 0; ci < m.nColor; ci++)
        {
            int col = forward ? ci : m.nColor - 1 - ci;
            launch(m.colorCells, m.colorStart[col], m.colorStart[col + 1]);
        }
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int lusgs_matvec_block(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *uInc, const real *jd, real *AuInc,
                       cudaStream_t st)
{
    int roe = ev.jacMode == 2;
    if (ev.s.nVars == 5)
        DNDSB_LAUNCH(k_matvec_blk<5>, m.nCell, 128, st, m, g, ev, roe, alphaDiag, u, uInc, jd, AuInc);
    else if (ev.s.nVars == 6)
        DNDSB_LAUNCH(k_matvec_blk<6>, m.nCell, 128, st, m, g, ev, roe, alphaDiag, u, uInc, jd, AuInc);
    else
        return ST_UNSUPPORTED;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
