#pragma once
// Kernels of the forward-mode derivatives for the SA model and viscous boundary zones, included by the
// instantiation units adjoint_generic_p{1,2}n{5,6}.cu (one VR degree and variable count each, compiled
// in parallel); the entry points are in adjoint_generic.cu.
//
// Derivatives of the residual path for the configurations the specialised kernels of adjoint.cu,
// adjoint_roe.cu and adjoint_visc.cu do not cover: the SA model (6 variables: the SA convective and
// diffusion fluxes, the eddy viscosity in the viscous flux, the source term) and boundary zones with
// a viscous flux (no-slip and isothermal walls, inflow, pressure outflow), for 5 or 6 variables.
//
// Forward mode throughout.  Per face Gauss point the integrand of EvaluateRHS (EvaluateRHS.hxx:224-525:
// F(UL, UR; ULm, URm) minus the viscous flux of the compact gradient) is evaluated in dual numbers
// with 2 NV seeds per pass: the two point states, the two cell means, then the two point gradients
// along each axis; on a boundary face the ghost states are formed inside the pass (the point state
// and the cell mean are seeded together).  The pass results are contracted with the face cotangent
// and carried through the reconstruction basis to (u, uRec) of both cells; the per-face cotangents
// are gathered per cell in a fixed order, as in the specialised kernels.  The SA source is
// differentiated per cell Gauss point in four passes (the point state, then the gradient along each
// axis).  The JVPs are the same computations with one seed.  The entropy-fix scale deltaLambdaCell
// is held fixed.  One Jacobi sweep of the reconstruction and its boundary term are differentiated as
// in adjoint.cu, for NV variables.
#include "solver.cuh"
#include "basis_eval.cuh"
#include "bc.cuh"
#include "sa.cuh"

namespace dndsb
{
namespace
{
// F - Fv at one point of an interior face (the integrand of fluxEs, EvaluateRHS.hxx:369-525)
// (parts: 1 the inviscid flux, 2 the viscous flux, 3 both; a pass whose seeds one part does not depend on
// skips that part)
template <int NV, typename T>
DNDSB_D bool interior_point_flux(const EulerSettingsD &s, const T *UL, const T *UR, const T *ULm, const T *URm, const T *GL, const T *GR,
                                 const real *n, const real *nMV, real distGRP, real dLambda, T *out, int parts = 3)
{
    const real gamma = s.gamma;
    T Fv[NV];
    for (int v = 0; v < NV; v++)
        Fv[v] = 0.0;
    if (!s.ignoreVis && (parts & 2))
    {
        real iD = 1.0 / distGRP;
        T UM[NV], GM[3 * NV], GP[3 * NV];
        for (int v = 0; v < NV; v++)
            UM[v] = 0.5 * (UL[v] + UR[v]);
        for (int d = 0; d < 3; d++)
            for (int v = 0; v < NV; v++)
                GM[d * NV + v] = (GR[d * NV + v] + GL[d * NV + v]) * 0.5 + iD * (n[d] * (UR[v] - UL[v]));
        grad_cons2prim<NV>(UM, GM, GP, gamma);
        point_viscous_flux<NV>(s, UM, GP, n, false, Fv);
    }
    T F[NV], l0, l1, l4;
    for (int v = 0; v < NV; v++)
        F[v] = 0.0;
    bool ok = true;
    if (parts & 1)
    {
        ok = riemann_flux(s.rsType, UL, UR, ULm, URm, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4, nMV);
        if (NV == 6)
            F[NV - 1] = sa_convective_flux(UL, UR, n, l1);
    }
    for (int v = 0; v < NV; v++)
        out[v] = F[v] - Fv[v];
    return ok;
}

// F - Fv at one point of a boundary face (bc.cu k_rhs_bc): ghost states of the point state and of the
// cell mean (at the face centre), the inner gradient, no viscous flux on slip, far-field and outflow faces
template <int NV, typename T>
DNDSB_D bool boundary_point_flux(const EulerSettingsD &s, const BoundaryD &bnd, int zone, int type, const T *ULin, const T *ULm,
                                 const real *nMean, const T *GL, const real *n, const real *nMV, real distGRP, real dLambda, T *out)
{
    const real gamma = s.gamma;
    T UL[NV], UR[NV], URm[NV];
    for (int v = 0; v < NV; v++)
        UL[v] = ULin[v];
    if (!bc_value<NV>(bnd, zone, ULm, nMean, URm))
        for (int v = 0; v < NV; v++)
            URm[v] = ULm[v];
    if (!bc_value_fix<NV>(bnd, zone, UL, n, UR))
        for (int v = 0; v < NV; v++)
            UR[v] = UL[v];
    const bool zeroGrad = type == BC_WALL_INVIS || type == BC_OUT || type == BC_FAR || type == BC_SYM;
    const bool slip = type == BC_WALL_INVIS || type == BC_SYM;
    T Fv[NV];
    for (int v = 0; v < NV; v++)
        Fv[v] = 0.0;
    if (!s.ignoreVis && !zeroGrad)
    {
        real iD = 1.0 / distGRP;
        T UM[NV], GM[3 * NV], GP[3 * NV];
        for (int v = 0; v < NV; v++)
            UM[v] = 0.5 * (UL[v] + UR[v]);
        for (int d = 0; d < 3; d++)
            for (int v = 0; v < NV; v++)
                GM[d * NV + v] = GL[d * NV + v] + iD * (n[d] * (UR[v] - UL[v]));
        grad_cons2prim<NV>(UM, GM, GP, gamma);
        if (!slip)
            point_viscous_flux<NV>(s, UM, GP, n, type == BC_WALL, Fv);
    }
    T F[NV], l0, l1, l4;
    for (int v = 0; v < NV; v++)
        F[v] = 0.0;
    bool ok = riemann_flux(s.rsType, UL, UR, ULm, URm, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4, nMV);
    if (NV == 6)
        F[NV - 1] = sa_convective_flux(UL, UR, n, l1);
    for (int v = 0; v < NV; v++)
        out[v] = F[v] - Fv[v];
    return ok;
}

// point value and gradient (rows 1..DIM of the basis table T) of one cell's reconstruction
template <int DIM, int NDOF, int NV>
DNDSB_D void recon_point_grad(const real *T, const real *u, const real *rec, real *U, real *G)
{
    constexpr int R = NDOF - 1;
    for (int v = 0; v < NV; v++)
    {
        real a = u[v], ga[3] = {0, 0, 0};
        for (int j = 0; j < R; j++)
        {
            real x = rec[j * NV + v];
            a += T[1 + j] * x;
            for (int d = 0; d < DIM; d++)
                ga[d] += T[(1 + d) * NDOF + 1 + j] * x;
        }
        U[v] = a;
        for (int d = 0; d < 3; d++)
            G[d * NV + v] = ga[d];
    }
}

// per-face geometry of the compact gradient: the distance of EvaluateRHS.hxx:363-386
DNDSB_D real grp_distance(const MeshD &m, const GeomD &g, int64_t f, int64_t c0, int64_t c1, const real *n)
{
    if (c1 >= 0)
    {
        real db[3];
        for (int d = 0; d < 3; d++)
            db[d] = g.cellBary[c1 * 3 + d] - m.facePShift[f * 3 + d] - g.cellBary[c0 * 3 + d];
        real dg = dmin(g.vol[c0], g.vol[c1]) * 2.0 / g.faceArea[f];
        return dmax(dmin(fabs(dot3(db, n)), dg * 2), dg * 0.25);
    }
    real dc[3];
    for (int d = 0; d < 3; d++)
        dc[d] = g.faceCent[f * 3 + d] - g.cellBary[c0 * 3 + d];
    real dg = g.vol[c0] / g.faceArea[f] * 2;
    return dmax(dmin(fabs(dot3(dc, n)) * 2., dg * 2), dg * 0.25);
}

DNDSB_D int zone_type(const BoundaryD &bnd, int zone) { return zone >= 0 && zone < bnd.nZone ? bnd.type[zone] : 0; }

// wall faces of the wall-flux integral (EvaluateRHS.hxx:599-607)
DNDSB_D bool is_wall(int type, real muGas) { return type == BC_WALL || type == BC_WALL_ISOTHERMAL || (type == BC_WALL_INVIS && muGas < 1e-99); }

// Face cotangents faceAdj[f][side][R+1][NV] (entry 0: d/du, 1+j: d/duRec_j) of
//   sum_c w_c . rhs_c   (objDir == nullptr), or of
//   sum over the wall faces of objDir . (minus their face flux), the wall-flux integral along objDir.
template <int DIM, int P, int NV>
DNDSB_GLOBAL void k_rhs_vjp_face_g(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ w, const real *__restrict__ objDir,
                                   const real *__restrict__ u, const real *__restrict__ uRec, const real *__restrict__ dLamCell,
                                   real *__restrict__ faceAdj, int *err, int bndOnly)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1, W = (R + 1) * NV;
    using DV = Dual<2 * NV>;
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        const int64_t c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        const bool bnd = c1 < 0;
        if (bndOnly && !bnd)
            continue; // the interior faces' records come from the Gauss-point-parallel kernel
        const int zone = m.faceZone[f], type = bnd ? zone_type(vr.bnd, zone) : 0;
        real *o0 = faceAdj + (f * 2) * W, *o1 = faceAdj + (f * 2 + 1) * W;
        for (int i = 0; i < W; i++)
            o0[i] = 0, o1[i] = 0;
        real gbar[NV];
        bool any = false;
        for (int v = 0; v < NV; v++)
        {
            if (objDir)
                gbar[v] = bnd && is_wall(type, s.muGas) ? -objDir[v] : 0.0;
            else
                gbar[v] = w[c0 * NV + v] / g.vol[c0] - (bnd ? 0.0 : w[c1 * NV + v] / g.vol[c1]);
            any = any || gbar[v] != 0.0;
        }
        if (!any)
            continue;
        const real *nMV = s.rsMeanValueEig ? &g.faceMeanNorm[f * 3] : nullptr;
        const real *ULm = u + c0 * NV, *URm = bnd ? nullptr : u + c1 * NV;
        const real dLambda = bnd ? dLamCell[c0] : dmax(dLamCell[c0], dLamCell[c1]);
        const bool vis = !s.ignoreVis && !(bnd && (type == BC_WALL_INVIS || type == BC_OUT || type == BC_FAR || type == BC_SYM));
        real ULbar[NV], URbar[NV], ULmbar[NV], URmbar[NV], GLbar[3 * NV], GRbar[3 * NV];
        for (int i = 0; i < NV; i++)
            ULbar[i] = URbar[i] = ULmbar[i] = URmbar[i] = 0;
        for (int i = 0; i < 3 * NV; i++)
            GLbar[i] = GRbar[i] = 0;
        bool bad = false;
        for (int q = 0; q < g.nGf; q++)
        {
            const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
            real p0[3], p1[3];
            for (int d = 0; d < 3; d++)
            {
                p0[d] = g.facePP[(f * g.nGf + q) * 3 + d];
                p1[d] = p0[d] + m.facePShift[f * 3 + d];
            }
            const real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            const real distGRP = grp_distance(m, g, f, c0, c1, n);
            real Fbar[NV];
            for (int v = 0; v < NV; v++)
                Fbar[v] = -JW * gbar[v];
            real T0[(DIM + 1) * NDOF], T1[(DIM + 1) * NDOF];
            real UL[NV], UR[NV], GL[3 * NV], GR[3 * NV];
            cell_basis<DIM, NDOF>(&g.cellCent[c0 * 3], &g.cellScale[c0 * 3], &vr.baseMoment[c0 * NDOF], vr.s.anisotropicLengths, p0, DIM + 1, T0);
            recon_point_grad<DIM, NDOF, NV>(T0, u + c0 * NV, uRec + c0 * R * NV, UL, GL);
            if (!bnd)
            {
                cell_basis<DIM, NDOF>(&g.cellCent[c1 * 3], &g.cellScale[c1 * 3], &vr.baseMoment[c1 * NDOF], vr.s.anisotropicLengths, p1, DIM + 1,
                                      T1);
                recon_point_grad<DIM, NDOF, NV>(T1, u + c1 * NV, uRec + c1 * R * NV, UR, GR);
            }
            const int npass = 2 + (vis ? DIM : 0);
            for (int pass = 0; pass < npass; pass++)
            {
                // pass 0: (UL, UR) [boundary: (UL, ULm)]; pass 1: (ULm, URm) [boundary: nothing]; 2 + d: (GL_d, GR_d)
                if (bnd && pass == 1)
                    continue;
                DV a[NV], b[NV], am[NV], bm[NV], ga[3 * NV], gb[3 * NV], out[NV];
                for (int v = 0; v < NV; v++)
                {
                    a[v] = DV(UL[v]), am[v] = DV(ULm[v]);
                    if (!bnd)
                        b[v] = DV(UR[v]), bm[v] = DV(URm[v]);
                }
                for (int i = 0; i < 3 * NV; i++)
                    ga[i] = DV(GL[i]), gb[i] = DV(bnd ? 0.0 : GR[i]);
                const int d = pass - 2;
                for (int v = 0; v < NV; v++)
                {
                    if (pass == 0)
                    {
                        a[v].d[v] = 1;
                        if (bnd)
                            am[v].d[NV + v] = 1;
                        else
                            b[v].d[NV + v] = 1;
                    }
                    else if (pass == 1)
                        am[v].d[v] = 1, bm[v].d[NV + v] = 1;
                    else
                        ga[d * NV + v].d[v] = 1, gb[d * NV + v].d[NV + v] = 1;
                }
                // on interior faces the means enter only the inviscid flux, the gradients only the viscous one
                bool ok = bnd ? boundary_point_flux<NV>(s, vr.bnd, zone, type, a, am, &g.faceMeanNorm[f * 3], ga, n, nMV, distGRP, dLambda, out)
                              : interior_point_flux<NV>(s, a, b, am, bm, ga, gb, n, nMV, distGRP, dLambda, out, pass == 0 ? 3 : pass == 1 ? 1 : 2);
                bad |= !ok;
                for (int i = 0; i < NV; i++)
                {
                    real x0 = 0, x1 = 0;
                    for (int v = 0; v < NV; v++)
                        x0 += out[v].d[i] * Fbar[v], x1 += out[v].d[NV + i] * Fbar[v];
                    if (pass == 0)
                    {
                        ULbar[i] += x0;
                        if (bnd)
                            ULmbar[i] += x1;
                        else
                            URbar[i] += x1;
                    }
                    else if (pass == 1)
                        ULmbar[i] += x0, URmbar[i] += x1;
                    else
                        GLbar[d * NV + i] += x0, GRbar[d * NV + i] += x1;
                }
            }
            // through the basis into (u, uRec) of both sides: U = u + sum_j T_j uRec_j, G_d = sum_j T_{d,j} uRec_j
            for (int v = 0; v < NV; v++)
            {
                o0[v] += ULbar[v];
                for (int j = 0; j < R; j++)
                {
                    real a = T0[1 + j] * ULbar[v];
                    for (int dd = 0; dd < DIM; dd++)
                        a += T0[(1 + dd) * NDOF + 1 + j] * GLbar[dd * NV + v];
                    o0[NV + j * NV + v] += a;
                }
                if (!bnd)
                {
                    o1[v] += URbar[v];
                    for (int j = 0; j < R; j++)
                    {
                        real a = T1[1 + j] * URbar[v];
                        for (int dd = 0; dd < DIM; dd++)
                            a += T1[(1 + dd) * NDOF + 1 + j] * GRbar[dd * NV + v];
                        o1[NV + j * NV + v] += a;
                    }
                }
                ULbar[v] = URbar[v] = 0;
            }
            for (int i = 0; i < 3 * NV; i++)
                GLbar[i] = GRbar[i] = 0;
        }
        for (int v = 0; v < NV; v++)
            o0[v] += ULmbar[v], o1[v] += URmbar[v];
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}

// tangent of the face integrand for tangents (du, duRec): ffd[f] = d(fluxEs_f)
template <int DIM, int P, int NV>
DNDSB_GLOBAL void k_rhs_jvp_face_g(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ du, const real *__restrict__ duRec,
                                   const real *__restrict__ u, const real *__restrict__ uRec, const real *__restrict__ dLamCell,
                                   real *__restrict__ ffd, int *err)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    using D1 = Dual<1>;
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        const int64_t c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        const bool bnd = c1 < 0;
        const int zone = m.faceZone[f], type = bnd ? zone_type(vr.bnd, zone) : 0;
        const real *nMV = s.rsMeanValueEig ? &g.faceMeanNorm[f * 3] : nullptr;
        const real dLambda = bnd ? dLamCell[c0] : dmax(dLamCell[c0], dLamCell[c1]);
        real acc[NV];
        for (int v = 0; v < NV; v++)
            acc[v] = 0;
        bool bad = false;
        D1 ULm[NV], URm[NV];
        for (int v = 0; v < NV; v++)
        {
            ULm[v] = D1(u[c0 * NV + v]), ULm[v].d[0] = du[c0 * NV + v];
            if (!bnd)
                URm[v] = D1(u[c1 * NV + v]), URm[v].d[0] = du[c1 * NV + v];
        }
        for (int q = 0; q < g.nGf; q++)
        {
            const real *n = &g.faceNorm[(f * g.nGf + q) * 3];
            real p0[3], p1[3];
            for (int d = 0; d < 3; d++)
            {
                p0[d] = g.facePP[(f * g.nGf + q) * 3 + d];
                p1[d] = p0[d] + m.facePShift[f * 3 + d];
            }
            const real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            const real distGRP = grp_distance(m, g, f, c0, c1, n);
            real T0[(DIM + 1) * NDOF], T1[(DIM + 1) * NDOF];
            real U[NV], G[3 * NV], dU[NV], dG[3 * NV];
            D1 UL[NV], UR[NV], GL[3 * NV], GR[3 * NV], out[NV];
            cell_basis<DIM, NDOF>(&g.cellCent[c0 * 3], &g.cellScale[c0 * 3], &vr.baseMoment[c0 * NDOF], vr.s.anisotropicLengths, p0, DIM + 1, T0);
            recon_point_grad<DIM, NDOF, NV>(T0, u + c0 * NV, uRec + c0 * R * NV, U, G);
            recon_point_grad<DIM, NDOF, NV>(T0, du + c0 * NV, duRec + c0 * R * NV, dU, dG);
            for (int v = 0; v < NV; v++)
                UL[v] = D1(U[v]), UL[v].d[0] = dU[v];
            for (int i = 0; i < 3 * NV; i++)
                GL[i] = D1(G[i]), GL[i].d[0] = dG[i];
            bool ok;
            if (bnd)
                ok = boundary_point_flux<NV>(s, vr.bnd, zone, type, UL, ULm, &g.faceMeanNorm[f * 3], GL, n, nMV, distGRP, dLambda, out);
            else
            {
                cell_basis<DIM, NDOF>(&g.cellCent[c1 * 3], &g.cellScale[c1 * 3], &vr.baseMoment[c1 * NDOF], vr.s.anisotropicLengths, p1, DIM + 1,
                                      T1);
                recon_point_grad<DIM, NDOF, NV>(T1, u + c1 * NV, uRec + c1 * R * NV, U, G);
                recon_point_grad<DIM, NDOF, NV>(T1, du + c1 * NV, duRec + c1 * R * NV, dU, dG);
                for (int v = 0; v < NV; v++)
                    UR[v] = D1(U[v]), UR[v].d[0] = dU[v];
                for (int i = 0; i < 3 * NV; i++)
                    GR[i] = D1(G[i]), GR[i].d[0] = dG[i];
                ok = interior_point_flux<NV>(s, UL, UR, ULm, URm, GL, GR, n, nMV, distGRP, dLambda, out);
            }
            bad |= !ok;
            for (int v = 0; v < NV; v++)
                acc[v] -= out[v].d[0] * JW;
        }
        for (int v = 0; v < NV; v++)
            ffd[f * NV + v] = acc[v];
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}

template <int W, int NV>
DNDSB_GLOBAL void k_adj_gather_g(int64_t nCell, int nf, const int32_t *__restrict__ c2f, const real *__restrict__ faceAdj, real *du, real *duRec)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        real acc[W];
        for (int i = 0; i < W; i++)
            acc[i] = 0;
        for (int k = 0; k < nf; k++)
        {
            int fp = c2f[c * nf + k];
            const real *src = faceAdj + ((int64_t)(fp >> 1) * 2 + (fp & 1)) * W;
            for (int i = 0; i < W; i++)
                acc[i] += src[i];
        }
        for (int v = 0; v < NV; v++)
            du[c * NV + v] = acc[v];
        for (int i = NV; i < W; i++)
            duRec[c * (W - NV) + i - NV] = acc[i];
    }
}

template <int NV>
DNDSB_GLOBAL void k_flux_gather_g(int64_t nCell, int nf, const int32_t *__restrict__ c2f, const real *__restrict__ vol, const real *__restrict__ ff,
                                  real *rhs)
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
                acc[v] += sg * ff[f * NV + v];
        }
        for (int v = 0; v < NV; v++)
            rhs[c * NV + v] = acc[v] * iv;
    }
}

// the SA source at the cell Gauss points (hotpath.cu k_sa_source): VJP (mode 0, cotangent w) adds into
// (du, duRec); JVP (mode 1, tangents du, duRec) adds into dRhs
template <int DIM, int P>
DNDSB_GLOBAL void k_sa_source_d(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ u, const real *__restrict__ uRec,
                                const real *__restrict__ dWall, int mode, const real *__restrict__ w, const real *__restrict__ tu,
                                const real *__restrict__ tRec, real *outU, real *outRec)
{
    constexpr int NV = 6, NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    using D6 = Dual<6>;
    using D1 = Dual<1>;
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        const real hMax = g.hMax[c];
        const real iv = 1.0 / g.vol[c];
        const real wb = mode == 0 ? w[c * NV + 5] * iv : 0.0;
        real aU[NV], aRec[R * NV], dS = 0;
        for (int i = 0; i < NV; i++)
            aU[i] = 0;
        for (int i = 0; i < R * NV; i++)
            aRec[i] = 0;
        for (int q = 0; q < g.nGc; q++)
        {
            real T[(DIM + 1) * NDOF];
            cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], &vr.baseMoment[c * NDOF], vr.s.anisotropicLengths,
                                  &g.cellPP[(c * g.nGc + q) * 3], DIM + 1, T);
            real U[NV], G[3 * NV];
            recon_point_grad<DIM, NDOF, NV>(T, u + c * NV, uRec + c * R * NV, U, G);
            const real d = dmin(dWall[c * g.nGc + q], pow(kVeryLarge, 1. / 6.));
            const real lLES = dmin(hMax * kVeryLarge, dmax(d, hMax));
            const real JW = g.cellJDet[c * g.nGc + q] * g.cellQw[q];
            if (mode == 0)
            {
                real Ubar[NV] = {0, 0, 0, 0, 0, 0}, Gbar[3 * NV];
                for (int i = 0; i < 3 * NV; i++)
                    Gbar[i] = 0;
                for (int pass = 0; pass <= DIM; pass++) // pass 0: U; pass 1 + d: G along axis d
                {
                    D6 Ud[NV], Gd[3 * NV];
                    for (int v = 0; v < NV; v++)
                        Ud[v] = D6(U[v]);
                    for (int i = 0; i < 3 * NV; i++)
                        Gd[i] = D6(G[i]);
                    for (int v = 0; v < NV; v++)
                    {
                        if (pass == 0)
                            Ud[v].d[v] = 1;
                        else
                            Gd[(pass - 1) * NV + v].d[v] = 1;
                    }
                    D6 pM, a2M, HM;
                    gas_thermal(Ud[4], Ud[0], D6((Ud[1] * Ud[1] + Ud[2] * Ud[2] + Ud[3] * Ud[3]) / (Ud[0] * Ud[0])), gamma, pM, a2M, HM);
                    D6 Tm = pM / ((gamma - 1) / gamma * cp * Ud[0]);
                    D6 mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, Ud[0], Tm);
                    D6 S = sa_source(Ud, Gd, s.muGas, mu, d, lLES, hMax, 0);
                    for (int v = 0; v < NV; v++)
                    {
                        if (pass == 0)
                            Ubar[v] += S.d[v] * JW * wb;
                        else
                            Gbar[(pass - 1) * NV + v] += S.d[v] * JW * wb;
                    }
                }
                for (int v = 0; v < NV; v++)
                {
                    aU[v] += Ubar[v];
                    for (int j = 0; j < R; j++)
                    {
                        real a = T[1 + j] * Ubar[v];
                        for (int dd = 0; dd < DIM; dd++)
                            a += T[(1 + dd) * NDOF + 1 + j] * Gbar[dd * NV + v];
                        aRec[j * NV + v] += a;
                    }
                }
            }
            else
            {
                real dU[NV], dG[3 * NV];
                recon_point_grad<DIM, NDOF, NV>(T, tu + c * NV, tRec + c * R * NV, dU, dG);
                D1 Ud[NV], Gd[3 * NV];
                for (int v = 0; v < NV; v++)
                    Ud[v] = D1(U[v]), Ud[v].d[0] = dU[v];
                for (int i = 0; i < 3 * NV; i++)
                    Gd[i] = D1(G[i]), Gd[i].d[0] = dG[i];
                D1 pM, a2M, HM;
                gas_thermal(Ud[4], Ud[0], D1((Ud[1] * Ud[1] + Ud[2] * Ud[2] + Ud[3] * Ud[3]) / (Ud[0] * Ud[0])), gamma, pM, a2M, HM);
                D1 Tm = pM / ((gamma - 1) / gamma * cp * Ud[0]);
                D1 mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, Ud[0], Tm);
                dS += sa_source(Ud, Gd, s.muGas, mu, d, lLES, hMax, 0).d[0] * JW;
            }
        }
        if (mode == 0)
        {
            for (int v = 0; v < NV; v++)
                outU[c * NV + v] += aU[v];
            for (int i = 0; i < R * NV; i++)
                outRec[c * R * NV + i] += aRec[i];
        }
        else
            outU[c * NV + 5] += dS * iv;
    }
}

// ---- one Jacobi sweep of the reconstruction, NV variables (the same algebra as adjoint.cu) ----
template <int R, int NV>
DNDSB_D void recon_value_g(const real *T, const real *u, const real *rec, real *U)
{
    for (int v = 0; v < NV; v++)
    {
        real a = u[v];
        for (int j = 0; j < R; j++)
            a += T[1 + j] * rec[j * NV + v];
        U[v] = a;
    }
}

// the boundary term BCC = sum_q w0^2 |J| w phi_q (UB_q - u_c), UB_q = ghost(compress(u_c, u_c + phi_q . uRec_c)):
// mode 0: VJP of its cotangent t into (vRec, vU); mode 1: JVP (dRec, du) -> dBCC
template <int DIM, int P, int NV>
DNDSB_D void bcc_derivative_g(const MeshD &m, const GeomD &g, const VRD &vr, int64_t c, const real *u, const real *uRec, int mode,
                              const real *t, real *vRec, real *vU, const real *dRec, const real *duc, real *dBCC)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    using DV = Dual<2 * NV>;
    const real *uc = u + c * NV, *rc = uRec + c * R * NV;
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
            real UL[NV];
            recon_value_g<R, NV>(T, uc, rc, UL);
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q] * w0 * w0;
            DV ULd[NV], umd[NV], ULf[NV], UB[NV];
            for (int v = 0; v < NV; v++)
                ULd[v] = DV::var(UL[v], v), umd[v] = DV::var(uc[v], NV + v);
            compress_rec<NV>(umd, ULd, ULf);
            if (!bc_value_fix<NV>(vr.bnd, zone, ULf, n, UB))
                for (int v = 0; v < NV; v++)
                    UB[v] = ULf[v];
            if (mode == 0)
            {
                real UBbar[NV];
                for (int v = 0; v < NV; v++)
                {
                    real a = 0;
                    for (int i = 0; i < R; i++)
                        a += T[1 + i] * t[i * NV + v];
                    UBbar[v] = a * JW;
                    vU[v] -= UBbar[v];
                }
                for (int i = 0; i < NV; i++)
                {
                    real gl = 0, gm = 0;
                    for (int v = 0; v < NV; v++)
                        gl += UB[v].d[i] * UBbar[v], gm += UB[v].d[NV + i] * UBbar[v];
                    vU[i] += gl + gm;
                    for (int j = 0; j < R; j++)
                        vRec[j * NV + i] += T[1 + j] * gl;
                }
            }
            else
            {
                real dUL[NV];
                for (int v = 0; v < NV; v++)
                {
                    real a = duc[v];
                    for (int j = 0; j < R; j++)
                        a += T[1 + j] * dRec[j * NV + v];
                    dUL[v] = a;
                }
                for (int v = 0; v < NV; v++)
                {
                    real dUB = 0;
                    for (int i = 0; i < NV; i++)
                        dUB += UB[v].d[i] * dUL[i] + UB[v].d[NV + i] * duc[i];
                    real dd = (dUB - duc[v]) * JW;
                    for (int i = 0; i < R; i++)
                        dBCC[i * NV + v] += T[1 + i] * dd;
                }
            }
        }
    }
}

template <int DIM, int P, int NV>
DNDSB_GLOBAL void k_vr_vjp_g(MeshD m, GeomD g, VRD vr, const real *__restrict__ v, const real *__restrict__ uRec, const real *__restrict__ u,
                             real *vRec, real *vU)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real om = vr.s.jacobiRelax;
    const int nf = m.nf;
    DNDSB_KERNEL_LOOP(o, m.nCell)
    {
        real aRec[R * NV], aU[NV];
        const real *vo = v + o * R * NV;
        for (int i = 0; i < R * NV; i++)
            aRec[i] = (1 - om) * vo[i];
        for (int x = 0; x < NV; x++)
            aU[x] = 0;
        bool hasBnd = false;
        for (int j = 0; j < nf; j++)
        {
            int i = m.cellNbr[o * nf + j];
            if (i < 0)
            {
                hasBnd = true;
                continue;
            }
            int k = m.nbrSlot[o * nf + j];
            const real *M = vr.AAInvB + ((int64_t)i * (nf + 1) + 1 + k) * R * R;
            const real *b = vr.AInvb + ((int64_t)i * nf + k) * R;
            const real *vi = v + (int64_t)i * R * NV;
            for (int r = 0; r < R; r++)
                for (int x = 0; x < NV; x++)
                {
                    real a = 0;
                    for (int l = 0; l < R; l++)
                        a += M[l * R + r] * vi[l * NV + x];
                    aRec[r * NV + x] += om * a;
                }
            const real *bo = vr.AInvb + (o * nf + j) * R;
            for (int x = 0; x < NV; x++)
            {
                real a = 0, a2 = 0;
                for (int l = 0; l < R; l++)
                    a += b[l] * vi[l * NV + x], a2 += bo[l] * vo[l * NV + x];
                aU[x] += om * (a - a2);
            }
        }
        if (hasBnd && vr.bnd.nZone > 0)
        {
            const real *Ai = vr.AAInvB + (o * (nf + 1)) * R * R;
            real t[R * NV];
            for (int r = 0; r < R; r++)
                for (int x = 0; x < NV; x++)
                {
                    real a = 0;
                    for (int l = 0; l < R; l++)
                        a += Ai[l * R + r] * vo[l * NV + x];
                    t[r * NV + x] = om * a;
                }
            bcc_derivative_g<DIM, P, NV>(m, g, vr, o, u, uRec, 0, t, aRec, aU, nullptr, nullptr, nullptr);
        }
        for (int i = 0; i < R * NV; i++)
            vRec[o * R * NV + i] = aRec[i];
        for (int x = 0; x < NV; x++)
            vU[o * NV + x] = aU[x];
    }
}

template <int DIM, int P, int NV>
DNDSB_GLOBAL void k_vr_jvp_g(MeshD m, GeomD g, VRD vr, const real *__restrict__ dRec, const real *__restrict__ du, const real *__restrict__ uRec,
                             const real *__restrict__ u, real *dNew)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real om = vr.s.jacobiRelax;
    const int nf = m.nf;
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real acc[R * NV];
        for (int i = 0; i < R * NV; i++)
            acc[i] = (1 - om) * dRec[c * R * NV + i];
        bool hasBnd = false;
        for (int k = 0; k < nf; k++)
        {
            int o = m.cellNbr[c * nf + k];
            if (o < 0)
            {
                hasBnd = true;
                continue;
            }
            const real *M = vr.AAInvB + (c * (nf + 1) + 1 + k) * R * R;
            const real *b = vr.AInvb + (c * nf + k) * R;
            for (int r = 0; r < R; r++)
                for (int x = 0; x < NV; x++)
                {
                    real a = b[r] * (du[(int64_t)o * NV + x] - du[c * NV + x]);
                    for (int l = 0; l < R; l++)
                        a += M[r * R + l] * dRec[((int64_t)o * R + l) * NV + x];
                    acc[r * NV + x] += om * a;
                }
        }
        if (hasBnd && vr.bnd.nZone > 0)
        {
            real dB[R * NV];
            for (int i = 0; i < R * NV; i++)
                dB[i] = 0;
            bcc_derivative_g<DIM, P, NV>(m, g, vr, c, u, uRec, 1, nullptr, nullptr, nullptr, dRec + c * R * NV, du + c * NV, dB);
            const real *Ai = vr.AAInvB + (c * (nf + 1)) * R * R;
            for (int r = 0; r < R; r++)
                for (int x = 0; x < NV; x++)
                {
                    real a = 0;
                    for (int l = 0; l < R; l++)
                        a += Ai[r * R + l] * dB[l * NV + x];
                    acc[r * NV + x] += om * a;
                }
        }
        for (int i = 0; i < R * NV; i++)
            dNew[c * R * NV + i] = acc[i];
    }
}
} // namespace

namespace gen
{
template <int DIM, int P, int NV>
int vjp_dp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *w, const real *objDir, const real *u, const real *uRec,
           real *du, real *duRec, cudaStream_t st)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1, W = (R + 1) * NV;
    // the SA model with plain Roe and the viscous flux: interior faces by the hand-reversed Gauss-point-parallel
    // kernel, boundary faces here
    int interiorDone = 0;
    if (NV == 6 && !objDir)
    {
        int rc = rhs_vjp_interior_fast_sa(m, g, vr, ev, w, u, uRec, ev.adjBuf, st);
        if (rc == ST_OK)
            interiorDone = 1;
        else if (rc != ST_UNSUPPORTED)
            return rc;
    }
    auto kf = k_rhs_vjp_face_g<DIM, P, NV>;
    DNDSB_LAUNCH(kf, m.nFace, 64, st, m, g, vr, ev.s, w, objDir, u, uRec, ev.deltaLambdaCell, ev.adjBuf, ev.errWord, interiorDone);
    auto kg = k_adj_gather_g<W, NV>;
    DNDSB_LAUNCH(kg, m.nCell, 128, st, m.nCell, m.nf, m.cell2face, ev.adjBuf, du, duRec);
    if (NV == 6 && !objDir)
    {
        auto ks = k_sa_source_d<DIM, P>;
        DNDSB_LAUNCH(ks, m.nCell, 64, st, m, g, vr, ev.s, u, uRec, ev.dWall, 0, w, nullptr, nullptr, du, duRec);
    }
    return ST_OK;
}

template <int DIM, int P, int NV>
int jvp_dp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *du, const real *duRec, const real *u, const real *uRec,
           real *dRhs, cudaStream_t st)
{
    auto kf = k_rhs_jvp_face_g<DIM, P, NV>;
    DNDSB_LAUNCH(kf, m.nFace, 64, st, m, g, vr, ev.s, du, duRec, u, uRec, ev.deltaLambdaCell, ev.adjBuf, ev.errWord);
    auto kg = k_flux_gather_g<NV>;
    DNDSB_LAUNCH(kg, m.nCell, 256, st, m.nCell, m.nf, m.cell2face, g.vol, ev.adjBuf, dRhs);
    if (NV == 6)
    {
        auto ks = k_sa_source_d<DIM, P>;
        DNDSB_LAUNCH(ks, m.nCell, 64, st, m, g, vr, ev.s, u, uRec, ev.dWall, 1, nullptr, du, duRec, dRhs, nullptr);
    }
    return ST_OK;
}

template <int DIM, int P, int NV>
int vr_vjp_dp_g(const MeshD &m, const GeomD &g, const VRD &vr, const real *v, const real *uRec, const real *u, real *vRec, real *vU, cudaStream_t st)
{
    auto k = k_vr_vjp_g<DIM, P, NV>;
    DNDSB_LAUNCH(k, m.nCell, 64, st, m, g, vr, v, uRec, u, vRec, vU);
    return ST_OK;
}

template <int DIM, int P, int NV>
int vr_jvp_dp_g(const MeshD &m, const GeomD &g, const VRD &vr, const real *dRec, const real *du, const real *uRec, const real *u, real *dNew,
                cudaStream_t st)
{
    auto k = k_vr_jvp_g<DIM, P, NV>;
    DNDSB_LAUNCH(k, m.nCell, 64, st, m, g, vr, dRec, du, uRec, u, dNew);
    return ST_OK;
}
} // namespace gen
} // namespace dndsb

// explicit instantiation of the launchers for 3-D meshes, VR degree P, NV variables
#define DNDSB_GEN_INSTANTIATE_RHS(P, NV)                                                                                                  \
    namespace dndsb::gen                                                                                                                \
    {                                                                                                                                   \
    template int vjp_dp<3, P, NV>(const MeshD &, const GeomD &, const VRD &, EvalD &, const real *, const real *, const real *,          \
                                  const real *, real *, real *, cudaStream_t);                                                           \
    template int jvp_dp<3, P, NV>(const MeshD &, const GeomD &, const VRD &, EvalD &, const real *, const real *, const real *,          \
                                  const real *, real *, cudaStream_t);                                                                   \
    }
#define DNDSB_GEN_INSTANTIATE_VR(P, NV)                                                                                                   \
    namespace dndsb::gen                                                                                                                \
    {                                                                                                                                   \
    template int vr_vjp_dp_g<3, P, NV>(const MeshD &, const GeomD &, const VRD &, const real *, const real *, const real *, real *,      \
                                       real *, cudaStream_t);                                                                            \
    template int vr_jvp_dp_g<3, P, NV>(const MeshD &, const GeomD &, const VRD &, const real *, const real *, const real *,              \
                                       const real *, real *, cudaStream_t);                                                              \
    }
