// Boundary faces of the VR sweep and of the right-hand side.
//
// Boundary faces are few (the walls and far-field of a channel are a few
// percent of the faces), so they run in their own kernels after the interior
// kernels: one thread per boundary cell adds the boundary term of the VR sweep,
// one thread per boundary face writes the boundary face flux.  Both are
// deterministic (fixed loop orders, no atomics on data).
#include "solver.cuh"
#include "basis_eval.cuh"
#include "bc.cuh"
#include "sa.cuh"

namespace dndsb
{
namespace
{
// VariationalReconstruction_Reconstruction.hxx:19-176 GetBoundaryRHS with the Euler FBoundary of
// EulerSolver.hxx:163-175, applied as in :568-586:
//   BCC = sum_{bc faces} sum_q w0^2 phi(x_q) (uBV(compress(u + phi . uRec)) - u) |J| w_q
//   uRecNew += relax A^-1 BCC     (recordInc: -= A^-1 BCC, nothing when uRecIsZero)
template <int DIM, int P, int NV, typename TC>
DNDSB_GLOBAL void k_vr_bc(MeshD m, GeomD g, VRD vr, const TC *__restrict__ AAInvB, const real *__restrict__ uRec, real *uRecNew,
                          const real *__restrict__ u, real relax, int recordInc)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(ii, m.nBndCell)
    {
        int64_t c = m.bndCell[ii];
        const real *uc = u + c * NV, *rc = uRec + c * R * NV;
        real BCC[R * NV];
        for (int i = 0; i < R * NV; i++)
            BCC[i] = 0;
        for (int k = 0; k < m.nf; k++)
        {
            if (m.cellNbr[c * m.nf + k] >= 0)
                continue;
            int64_t f = m.cell2face[c * m.nf + k] >> 1;
            real w0 = vr.faceWeight[f * (P + 1)];
            if (w0 == 0)
                continue;
            int zone = m.faceZone[f];
            for (int q = 0; q < g.nGf; q++)
            {
                const real *p = &g.facePP[(f * g.nGf + q) * 3];
                const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
                real T[NDOF];
                cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], &vr.baseMoment[c * NDOF], vr.s.anisotropicLengths, p, 1, T);
                real UL[NV], ULf[NV], UB[NV];
                for (int v = 0; v < NV; v++)
                {
                    real a = uc[v];
                    for (int j = 0; j < R; j++)
                        a += T[1 + j] * rc[j * NV + v];
                    UL[v] = a;
                }
                compress_rec<NV>(uc, UL, ULf);
                if (!bc_value_fix<NV>(vr.bnd, zone, ULf, n, UB))
                    for (int v = 0; v < NV; v++)
                        UB[v] = ULf[v];
                real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q] * w0 * w0;
                for (int i = 0; i < R; i++)
                    for (int v = 0; v < NV; v++)
                        BCC[i * NV + v] += T[1 + i] * (UB[v] - uc[v]) * JW;
            }
        }
        const TC *Ai = AAInvB + c * (m.nf + 1) * R * R;
        real sgn = recordInc ? -1.0 : relax;
        for (int i = 0; i < R; i++)
        {
            real acc[NV];
            for (int v = 0; v < NV; v++)
                acc[v] = 0;
            for (int j = 0; j < R; j++)
            {
                real a = (real)Ai[i * R + j];
                for (int v = 0; v < NV; v++)
                    acc[v] += a * BCC[j * NV + v];
            }
            for (int v = 0; v < NV; v++)
                uRecNew[(c * R + i) * NV + v] += sgn * acc[v];
        }
    }
}

// DoReconstructionIter with SORInstead (VariationalReconstruction_Reconstruction.hxx:534-611): one colour class of an
// in-place sweep, row_c = (1 - relax) row_c + relax sum over faces in cell2face order of A^-1 B_k uRec_o + A^-1 b_k (u_o - u_c)
// (interior) or A^-1 GetBoundaryRHS (boundary, evaluated from the cell's partially updated row, as the reference's
// in-place update reads it).  Cells of one colour are not adjacent, so a colour is one launch and the sweep equals the
// reference's sequential one on a mesh numbered colour by colour.
template <int DIM, int P, int NV>
DNDSB_GLOBAL void k_vr_sor(MeshD m, GeomD g, VRD vr, int64_t cBeg, int64_t cEnd, real *uRec, const real *__restrict__ u, real relax)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(ii, cEnd - cBeg)
    {
        int64_t c = m.colorCells[cBeg + ii];
        const real *uc = u + c * NV;
        real row[R * NV];
        for (int i = 0; i < R * NV; i++)
            row[i] = uRec[c * R * NV + i] * (1 - relax);
        for (int k = 0; k < m.nf; k++)
        {
            int o = m.cellNbr[c * m.nf + k];
            real t[R * NV];
            if (o >= 0)
            {
                const real *M = vr.AAInvB + ((c * (m.nf + 1) + 1 + k) * R) * R;
                const real *b = vr.AInvb + (c * m.nf + k) * R;
                const real *ro = o == c ? row : uRec + (int64_t)o * R * NV; // a periodic image of itself: the current row
                for (int i = 0; i < R; i++)
                    for (int v = 0; v < NV; v++)
                    {
                        real acc = 0;
                        for (int j = 0; j < R; j++)
                            acc += M[i * R + j] * ro[j * NV + v];
                        t[i * NV + v] = acc + b[i] * (u[(int64_t)o * NV + v] - uc[v]);
                    }
            }
            else
            {
                int64_t f = m.cell2face[c * m.nf + k] >> 1;
                real BCC[R * NV];
                for (int i = 0; i < R * NV; i++)
                    BCC[i] = 0;
                real w0 = vr.faceWeight[f * (P + 1)];
                int zone = m.faceZone[f];
                if (w0 != 0)
                    for (int q = 0; q < g.nGf; q++)
                    {
                        const real *p = &g.facePP[(f * g.nGf + q) * 3];
                        const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
                        real T[NDOF];
                        cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], &vr.baseMoment[c * NDOF], vr.s.anisotropicLengths, p, 1, T);
                        real UL[NV], ULf[NV], UB[NV];
                        for (int v = 0; v < NV; v++)
                        {
                            real a = uc[v];
                            for (int j = 0; j < R; j++)
                                a += T[1 + j] * row[j * NV + v];
                            UL[v] = a;
                        }
                        compress_rec<NV>(uc, UL, ULf);
                        if (!bc_value_fix<NV>(vr.bnd, zone, ULf, n, UB))
                            for (int v = 0; v < NV; v++)
                                UB[v] = ULf[v];
                        real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q] * w0 * w0;
                        for (int i = 0; i < R; i++)
                            for (int v = 0; v < NV; v++)
                                BCC[i * NV + v] += T[1 + i] * (UB[v] - uc[v]) * JW;
                    }
                const real *Ai = vr.AAInvB + c * (m.nf + 1) * R * R;
                for (int i = 0; i < R; i++)
                    for (int v = 0; v < NV; v++)
                    {
                        real acc = 0;
                        for (int j = 0; j < R; j++)
                            acc += Ai[i * R + j] * BCC[j * NV + v];
                        t[i * NV + v] = acc;
                    }
            }
            for (int i = 0; i < R * NV; i++)
                row[i] += relax * t[i];
        }
        for (int i = 0; i < R * NV; i++)
            uRec[c * R * NV + i] = row[i];
    }
}

template <int DIM, int NV>
int vr_sor_p(const MeshD &m, const GeomD &g, const VRD &vr, real *uRec, const real *u, cudaStream_t st)
{
    for (int ci = 0; ci < m.nColor; ci++)
    {
        int64_t b = m.colorStart[ci], e = m.colorStart[ci + 1];
        switch (vr.P)
        {
        case 1:
            DNDSB_LAUNCH((k_vr_sor<DIM, 1, NV>), e - b, 64, st, m, g, vr, b, e, uRec, u, vr.s.jacobiRelax);
            break;
        case 2:
            DNDSB_LAUNCH((k_vr_sor<DIM, 2, NV>), e - b, 64, st, m, g, vr, b, e, uRec, u, vr.s.jacobiRelax);
            break;
        case 3:
            DNDSB_LAUNCH((k_vr_sor<DIM, 3, NV>), e - b, 64, st, m, g, vr, b, e, uRec, u, vr.s.jacobiRelax);
            break;
        default:
            return ST_UNSUPPORTED;
        }
    }
    return ST_OK;
}

// EulerEvaluator_EvaluateRHS.hxx:171-562 on a boundary face: ghost state at every Gauss
// point, Roe means from the ghost of the cell mean at the face centre (:198-210), the inner
// gradient on both sides (:360-362), GRP distance from the face centre (:363-386) and no
// viscous flux on slip, far-field and outflow faces (:423-430, EvaluateDt.hxx:1203-1207)
template <int DIM, int P, int NV>
// lam (may be nullptr): [3][nFace] face integrals of the eigenvalues l0, l123, l4 divided by the area (useRoeJacobian)
DNDSB_GLOBAL void k_rhs_bc(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ u, const real *__restrict__ uRec,
                           const real *__restrict__ uRecG, const real *__restrict__ dLamCell, real *__restrict__ faceFlux, int *err,
                           real *__restrict__ lam)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real gamma = s.gamma;
    DNDSB_KERNEL_LOOP(ii, m.nBndFace)
    {
        int64_t f = m.bndFace[ii];
        int64_t c0 = m.face2cell[f * 2];
        int zone = m.faceZone[f];
        int type = zone >= 0 && zone < vr.bnd.nZone ? vr.bnd.type[zone] : 0;
        const real *ULm = u + c0 * NV, *r0 = uRec + c0 * R * NV, *q0 = uRecG + c0 * R * NV; // values, gradients
        real URm[NV];
        bool bad = false;
        if (!bc_value<NV>(vr.bnd, zone, ULm, &g.faceMeanNorm[f * 3], URm))
            for (int v = 0; v < NV; v++)
                URm[v] = ULm[v];
        real dLambda = dLamCell[c0];
        bool zeroGrad = type == BC_WALL_INVIS || type == BC_OUT || type == BC_FAR || type == BC_SYM;
        bool slip = type == BC_WALL_INVIS || type == BC_SYM;
        real dc[3];
        for (int d = 0; d < 3; d++)
            dc[d] = g.faceCent[f * 3 + d] - g.cellBary[c0 * 3 + d];
        real fluxEs[NV], lamEs[3] = {0, 0, 0};
        for (int v = 0; v < NV; v++)
            fluxEs[v] = 0;
        for (int q = 0; q < g.nGf; q++)
        {
            const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
            const real *p0 = &g.facePP[(f * g.nGf + q) * 3];
            real T0[(DIM + 1) * NDOF];
            cell_basis<DIM, NDOF>(&g.cellCent[c0 * 3], &g.cellScale[c0 * 3], &vr.baseMoment[c0 * NDOF], vr.s.anisotropicLengths, p0, DIM + 1,
                                  T0);
            real UL[NV], UR[NV], GL[3 * NV];
            for (int v = 0; v < NV; v++)
            {
                real a = ULm[v];
                real ga[3] = {0, 0, 0};
                for (int j = 0; j < R; j++)
                {
                    real x0 = r0[j * NV + v], y0 = q0[j * NV + v];
                    a += T0[1 + j] * x0;
                    for (int d = 0; d < DIM; d++)
                        ga[d] += T0[(1 + d) * NDOF + 1 + j] * y0;
                }
                UL[v] = a;
                for (int d = 0; d < 3; d++)
                    GL[d * NV + v] = ga[d];
            }
            if (!bc_value_fix<NV>(vr.bnd, zone, UL, n, UR))
                for (int v = 0; v < NV; v++)
                    UR[v] = UL[v];
            real Fv[NV];
            for (int v = 0; v < NV; v++)
                Fv[v] = 0;
            if (!s.ignoreVis && !zeroGrad)
            {
                real distBaryPerp = fabs(dot3(dc, n)) * 2.;
                real distGRP = g.vol[c0] / g.faceArea[f] * 2;
                distGRP = dmax(dmin(distBaryPerp, distGRP * 2), distGRP * 0.25);
                real iD = 1.0 / distGRP;
                real UM[NV], GM[3 * NV], GP[3 * NV];
                for (int v = 0; v < NV; v++)
                    UM[v] = 0.5 * (UL[v] + UR[v]);
                for (int d = 0; d < 3; d++)
                    for (int v = 0; v < NV; v++)
                        GM[d * NV + v] = GL[d * NV + v] + iD * (n[d] * (UR[v] - UL[v]));
                grad_cons2prim<NV>(UM, GM, GP, gamma);
                if (!slip)
                    point_viscous_flux<NV>(s, UM, GP, n, type == BC_WALL, Fv);
            }
            real F[NV], l0, l1, l4;
            for (int v = 0; v < NV; v++)
                F[v] = 0;
            bad |= !riemann_flux(s.rsType, UL, UR, ULm, URm, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4,
                                 s.rsMeanValueEig ? &g.faceMeanNorm[f * 3] : nullptr);
            if (NV == 6)
                F[NV - 1] = sa_convective_flux(UL, UR, n, l1);
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            for (int v = 0; v < NV; v++)
                fluxEs[v] -= (F[v] - Fv[v]) * JW;
            lamEs[0] += l0 * JW, lamEs[1] += l1 * JW, lamEs[2] += l4 * JW;
        }
        if (lam)
            for (int i = 0; i < 3; i++)
                lam[i * m.nFace + f] = lamEs[i] / g.faceArea[f];
        bool fin = true;
        for (int v = 0; v < NV; v++)
            fin = fin && isfinite(fluxEs[v]);
        if (bad || !fin)
            atomicOr(err, bad ? (int)DE_NONPHYSICAL : (int)DE_NONFINITE);
        for (int v = 0; v < NV; v++)
            faceFlux[f * NV + v] = fluxEs[v];
    }
}

template <int DIM, int P, int NV>
void launch_vr_bc(const MeshD &m, const GeomD &g, const VRD &vr, const real *uRec, real *uRecNew, const real *u, int recordInc, int useFP32,
                  cudaStream_t st)
{
    if (useFP32)
    {
        auto k = k_vr_bc<DIM, P, NV, float>;
        DNDSB_LAUNCH(k, m.nBndCell, 64, st, m, g, vr, vr.AAInvB32, uRec, uRecNew, u, vr.s.jacobiRelax, recordInc);
    }
    else
    {
        auto k = k_vr_bc<DIM, P, NV, real>;
        DNDSB_LAUNCH(k, m.nBndCell, 64, st, m, g, vr, vr.AAInvB, uRec, uRecNew, u, vr.s.jacobiRelax, recordInc);
    }
}

template <int DIM, int NV>
int vr_bc_p(const MeshD &m, const GeomD &g, const VRD &vr, const real *uRec, real *uRecNew, const real *u, int recordInc, int useFP32,
            cudaStream_t st)
{
    switch (vr.P)
    {
    case 1:
        launch_vr_bc<DIM, 1, NV>(m, g, vr, uRec, uRecNew, u, recordInc, useFP32, st);
        return ST_OK;
    case 2:
        launch_vr_bc<DIM, 2, NV>(m, g, vr, uRec, uRecNew, u, recordInc, useFP32, st);
        return ST_OK;
    case 3:
        launch_vr_bc<DIM, 3, NV>(m, g, vr, uRec, uRecNew, u, recordInc, useFP32, st);
        return ST_OK;
    }
    return ST_UNSUPPORTED;
}

template <int DIM, int NV>
int rhs_bc_p(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *u, const real *uRec, const real *uRecG, real *ff,
             cudaStream_t st)
{
    switch (vr.P)
    {
    case 1:
    {
        auto k = k_rhs_bc<DIM, 1, NV>;
        DNDSB_LAUNCH(k, m.nBndFace, 64, st, m, g, vr, ev.s, u, uRec, uRecG, ev.deltaLambdaCell, ff, ev.errWord,
                     ev.jacMode == 2 ? ev.lambdaFace0 : nullptr);
        return ST_OK;
    }
    case 2:
    {
        auto k = k_rhs_bc<DIM, 2, NV>;
        DNDSB_LAUNCH(k, m.nBndFace, 64, st, m, g, vr, ev.s, u, uRec, uRecG, ev.deltaLambdaCell, ff, ev.errWord,
                     ev.jacMode == 2 ? ev.lambdaFace0 : nullptr);
        return ST_OK;
    }
    case 3:
    {
        auto k = k_rhs_bc<DIM, 3, NV>;
        DNDSB_LAUNCH(k, m.nBndFace, 64, st, m, g, vr, ev.s, u, uRec, uRecG, ev.deltaLambdaCell, ff, ev.errWord,
                     ev.jacMode == 2 ? ev.lambdaFace0 : nullptr);
        return ST_OK;
    }
    }
    return ST_UNSUPPORTED;
}
} // namespace

int vr_iter_bc(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *uRec, real *uRecNew, const real *u, int recordInc,
               int uRecIsZero, int useFP32, cudaStream_t st)
{
    if (m.nBndCell == 0 || (recordInc && uRecIsZero))
        return ST_OK;
    int rc = ST_UNSUPPORTED;
    if (nv == 5)
        rc = m.dim == 2 ? vr_bc_p<2, 5>(m, g, vr, uRec, uRecNew, u, recordInc, useFP32, st)
                        : vr_bc_p<3, 5>(m, g, vr, uRec, uRecNew, u, recordInc, useFP32, st);
    else if (nv == 6)
        rc = m.dim == 2 ? vr_bc_p<2, 6>(m, g, vr, uRec, uRecNew, u, recordInc, useFP32, st)
                        : vr_bc_p<3, 6>(m, g, vr, uRec, uRecNew, u, recordInc, useFP32, st);
    if (rc != ST_OK)
        return rc;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int vr_iter_sor(const MeshD &m, const GeomD &g, const VRD &vr, int nv, real *uRec, const real *u, cudaStream_t st)
{
    if (m.nBndFace > 0 && !vr.bnd.type)
        return ST_BADARG;
    int rc = ST_UNSUPPORTED;
    if (nv == 5)
        rc = m.dim == 2 ? vr_sor_p<2, 5>(m, g, vr, uRec, u, st) : vr_sor_p<3, 5>(m, g, vr, uRec, u, st);
    else if (nv == 6)
        rc = m.dim == 2 ? vr_sor_p<2, 6>(m, g, vr, uRec, u, st) : vr_sor_p<3, 6>(m, g, vr, uRec, u, st);
    if (rc != ST_OK)
        return rc;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int rhs_bc(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *u, const real *uRec, const real *uRecG, real *ff,
           cudaStream_t st)
{
    if (m.nBndFace == 0)
        return ST_OK;
    int rc = ST_UNSUPPORTED;
    if (ev.s.nVars == 5)
        rc = m.dim == 2 ? rhs_bc_p<2, 5>(m, g, vr, ev, u, uRec, uRecG, ff, st) : rhs_bc_p<3, 5>(m, g, vr, ev, u, uRec, uRecG, ff, st);
    else if (ev.s.nVars == 6)
        rc = m.dim == 2 ? rhs_bc_p<2, 6>(m, g, vr, ev, u, uRec, uRecG, ff, st) : rhs_bc_p<3, 6>(m, g, vr, ev, u, uRec, uRecG, ff, st);
    if (rc != ST_OK)
        return rc;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
