// Viscous part of the derivatives of EvaluateRHS (5 variables).
//
// The face Gauss-point viscous flux of EulerEvaluator_EvaluateRHS.hxx:369-430 is
//   Fv(U_M, grad U_M),  U_M = (U_L + U_R) / 2,
//   grad U_M = (grad U_L + grad U_R) / 2 + (U_R - U_L) (x) n / d_GRP,
// with grad U = D1 phi . uRec of each side and the flux of Gas.hpp:1594-1655 on the primitive
// gradient (Gas.hpp:1677-1698).  Fv depends on the 20 numbers (U_M, grad U_M).  Their cotangents
// (VJP): five Dual<1> passes for U_M at fixed gradient, and for grad U_M the transposes of the two
// maps that are linear in it (conservative -> primitive gradient, primitive gradient -> flux);
// the chain above carries them to (u, uRec) of both cells.  The JVP is one Dual<1> pass.  Both add to the
// inviscid face arrays before their per-cell gathers.  Boundary faces carry no viscous flux in
// the zone types allowed here (far-field, outflow, slip wall, symmetry).
#include "solver.cuh"
#include "basis_eval.cuh"
#include "visc_rev.cuh"

namespace dndsb
{
namespace
{
constexpr int NV = 5;
using D1 = Dual<1>;
using visc_rev::visc_flux_t;
using visc_rev::visc_point_bar;

// geometry of one interior face shared by its Gauss points
struct ViscFace
{
    int64_t c0, c1;
    real db[3], minVol, areaInv2;
};

DNDSB_D ViscFace visc_face(const MeshD &m, const GeomD &g, int64_t f)
{
    ViscFace F;
    F.c0 = m.face2cell[f * 2], F.c1 = m.face2cell[f * 2 + 1];
    for (int d = 0; d < 3; d++)
        F.db[d] = F.c1 >= 0 ? g.cellBary[F.c1 * 3 + d] - m.facePShift[f * 3 + d] - g.cellBary[F.c0 * 3 + d] : 0.0;
    F.minVol = F.c1 >= 0 ? dmin(g.vol[F.c0], g.vol[F.c1]) : g.vol[F.c0];
    F.areaInv2 = 2.0 / g.faceArea[f];
    return F;
}

// the Gauss-point states, gradients and basis rows of both sides (as the primal face kernel)
template <int DIM, int P>
DNDSB_D void visc_point(const MeshD &m, const GeomD &g, const VRD &vr, const ViscFace &F, int64_t f, int q, const real *u, const real *uRec,
                        real *T0, real *T1, real *UL, real *UR, real *GL, real *GR, real &iD, const real *&n)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    n = &g.faceNorm[(f * g.nGf + q) * 3];
    real p0[3], p1[3];
    for (int d = 0; d < 3; d++)
    {
        p0[d] = g.facePP[(f * g.nGf + q) * 3 + d];
        p1[d] = p0[d] + m.facePShift[f * 3 + d];
    }
    cell_basis<DIM, NDOF>(&g.cellCent[F.c0 * 3], &g.cellScale[F.c0 * 3], &vr.baseMoment[F.c0 * NDOF], vr.s.anisotropicLengths, p0, DIM + 1, T0);
    cell_basis<DIM, NDOF>(&g.cellCent[F.c1 * 3], &g.cellScale[F.c1 * 3], &vr.baseMoment[F.c1 * NDOF], vr.s.anisotropicLengths, p1, DIM + 1, T1);
    const real *r0 = uRec + F.c0 * R * NV, *r1 = uRec + F.c1 * R * NV;
    for (int v = 0; v < NV; v++)
    {
        real a = u[F.c0 * NV + v], b = u[F.c1 * NV + v];
        real ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
        for (int j = 0; j < R; j++)
        {
            real x0 = r0[j * NV + v], x1 = r1[j * NV + v];
            a += T0[1 + j] * x0;
            b += T1[1 + j] * x1;
            for (int d = 0; d < DIM; d++)
                ga[d] += T0[(1 + d) * NDOF + 1 + j] * x0, gb[d] += T1[(1 + d) * NDOF + 1 + j] * x1;
        }
        UL[v] = a, UR[v] = b;
        for (int d = 0; d < 3; d++)
            GL[d * NV + v] = ga[d], GR[d * NV + v] = gb[d];
    }
    real distBaryPerp = fabs(dot3(F.db, n));
    real distGRP = F.minVol * F.areaInv2;
    distGRP = dmax(dmin(distBaryPerp, distGRP * 2), distGRP * 0.25);
    iD = 1.0 / distGRP;
}

template <int DIM, int P>
DNDSB_GLOBAL void k_rhs_vjp_visc(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ w, const real *__restrict__ u,
                                 const real *__restrict__ uRec, real *__restrict__ faceAdj)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1, W = (R + 1) * NV;
    const real gamma = s.gamma;
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        if (m.face2cell[f * 2 + 1] < 0)
            continue;
        ViscFace F = visc_face(m, g, f);
        real *o0g = faceAdj + (f * 2) * W, *o1g = faceAdj + (f * 2 + 1) * W;
        // the face's two cotangent rows accumulated over its Gauss points, stored once
        real o0[W], o1[W];
        for (int i = 0; i < W; i++)
            o0[i] = o0g[i], o1[i] = o1g[i];
        real gbar[NV];
        for (int v = 0; v < NV; v++)
            gbar[v] = w[F.c0 * NV + v] / g.vol[F.c0] - w[F.c1 * NV + v] / g.vol[F.c1];
        for (int q = 0; q < g.nGf; q++)
        {
            real T0[(DIM + 1) * NDOF], T1[(DIM + 1) * NDOF], UL[NV], UR[NV], GL[3 * NV], GR[3 * NV], iD;
            const real *n;
            visc_point<DIM, P>(m, g, vr, F, f, q, u, uRec, T0, T1, UL, UR, GL, GR, iD, n);
            // the face flux is -(F - Fv) |J| w: the cotangent of Fv is +|J| w gbar.  bar[0..4]: the
            // cotangent of U_M (Dual<1> passes at fixed grad U_M); bar[5..19]: of grad U_M
            // (transposed linear maps at fixed U_M)
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            real UMr[NV], GMr[3 * NV], Fvbar[NV], bar[20];
            for (int v = 0; v < NV; v++)
                UMr[v] = 0.5 * (UL[v] + UR[v]), Fvbar[v] = JW * gbar[v];
            for (int d = 0; d < 3; d++)
                for (int v = 0; v < NV; v++)
                    GMr[d * NV + v] = (GR[d * NV + v] + GL[d * NV + v]) * 0.5 + iD * (n[d] * (UR[v] - UL[v]));
            visc_point_bar(s, UMr, GMr, n, Fvbar, bar);
            for (int v = 0; v < NV; v++)
            {
                real nG = 0;
                for (int d = 0; d < 3; d++)
                    nG += n[d] * bar[NV + d * NV + v];
                real ULbar = 0.5 * bar[v] - iD * nG, URbar = 0.5 * bar[v] + iD * nG;
                o0[v] += ULbar;
                o1[v] += URbar;
                for (int j = 0; j < R; j++)
                {
                    real a0 = T0[1 + j] * ULbar, a1 = T1[1 + j] * URbar;
                    for (int d = 0; d < DIM; d++)
                    {
                        real gmb = 0.5 * bar[NV + d * NV + v];
                        a0 += T0[(1 + d) * NDOF + 1 + j] * gmb;
                        a1 += T1[(1 + d) * NDOF + 1 + j] * gmb;
                    }
                    o0[NV + j * NV + v] += a0;
                    o1[NV + j * NV + v] += a1;
                }
            }
        }
        for (int i = 0; i < W; i++)
            o0g[i] = o0[i], o1g[i] = o1[i];
    }
}

template <int DIM, int P>
DNDSB_GLOBAL void k_rhs_jvp_visc(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ du, const real *__restrict__ duRec,
                                 const real *__restrict__ u, const real *__restrict__ uRec, real *__restrict__ ffd)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real gamma = s.gamma;
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        if (m.face2cell[f * 2 + 1] < 0)
            continue;
        ViscFace F = visc_face(m, g, f);
        real acc[NV] = {0, 0, 0, 0, 0};
        for (int q = 0; q < g.nGf; q++)
        {
            real T0[(DIM + 1) * NDOF], T1[(DIM + 1) * NDOF], UL[NV], UR[NV], GL[3 * NV], GR[3 * NV], iD;
            const real *n;
            visc_point<DIM, P>(m, g, vr, F, f, q, u, uRec, T0, T1, UL, UR, GL, GR, iD, n);
            // tangents of the point states and gradients of both sides
            real dUL[NV], dUR[NV], dGL[3 * NV], dGR[3 * NV];
            for (int v = 0; v < NV; v++)
            {
                real a = du[F.c0 * NV + v], b = du[F.c1 * NV + v];
                real ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
                for (int j = 0; j < R; j++)
                {
                    real x0 = duRec[(F.c0 * R + j) * NV + v], x1 = duRec[(F.c1 * R + j) * NV + v];
                    a += T0[1 + j] * x0;
                    b += T1[1 + j] * x1;
                    for (int d = 0; d < DIM; d++)
                        ga[d] += T0[(1 + d) * NDOF + 1 + j] * x0, gb[d] += T1[(1 + d) * NDOF + 1 + j] * x1;
                }
                dUL[v] = a, dUR[v] = b;
                for (int d = 0; d < 3; d++)
                    dGL[d * NV + v] = ga[d], dGR[d * NV + v] = gb[d];
            }
            D1 UM[NV], GM[3 * NV], GP[3 * NV], Fv[NV];
            for (int v = 0; v < NV; v++)
            {
                UM[v] = D1(0.5 * (UL[v] + UR[v]));
                UM[v].d[0] = 0.5 * (dUL[v] + dUR[v]);
            }
            for (int d = 0; d < 3; d++)
                for (int v = 0; v < NV; v++)
                {
                    int i = d * NV + v;
                    GM[i] = D1((GR[i] + GL[i]) * 0.5 + iD * (n[d] * (UR[v] - UL[v])));
                    GM[i].d[0] = (dGR[i] + dGL[i]) * 0.5 + iD * (n[d] * (dUR[v] - dUL[v]));
                }
            grad_cons2prim<NV>(UM, GM, GP, gamma);
            visc_flux_t(s, UM, GP, n, Fv);
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            for (int v = 0; v < NV; v++)
                acc[v] += Fv[v].d[0] * JW;
        }
        for (int v = 0; v < NV; v++)
            ffd[f * NV + v] += acc[v];
    }
}

template <int DIM, int P>
void launch_visc(bool vjp, const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *a, const real *b, const real *u,
                 const real *uRec, real *out, cudaStream_t st)
{
    if (vjp)
        DNDSB_LAUNCH((k_rhs_vjp_visc<DIM, P>), m.nFace, 64, st, m, g, vr, ev.s, a, u, uRec, out);
    else
        DNDSB_LAUNCH((k_rhs_jvp_visc<DIM, P>), m.nFace, 64, st, m, g, vr, ev.s, a, b, u, uRec, out);
}

int dispatch(bool vjp, const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *a, const real *b, const real *u,
             const real *uRec, real *out, cudaStream_t st)
{
    if (m.dim == 2)
    {
        if (vr.P == 1)
            launch_visc<2, 1>(vjp, m, g, vr, ev, a, b, u, uRec, out, st);
        else if (vr.P == 2)
            launch_visc<2, 2>(vjp, m, g, vr, ev, a, b, u, uRec, out, st);
        else
            launch_visc<2, 3>(vjp, m, g, vr, ev, a, b, u, uRec, out, st);
    }
    else if (vr.P == 1)
        launch_visc<3, 1>(vjp, m, g, vr, ev, a, b, u, uRec, out, st);
    else if (vr.P == 2)
        launch_visc<3, 2>(vjp, m, g, vr, ev, a, b, u, uRec, out, st);
    else
        launch_visc<3, 3>(vjp, m, g, vr, ev, a, b, u, uRec, out, st);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace

int rhs_vjp_visc(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *w, const real *u, const real *uRec, real *faceAdj,
                 cudaStream_t st)
{
    if (ev.s.nVars != NV || !vr.bnd.viscFree)
        return ST_UNSUPPORTED;
    return dispatch(true, m, g, vr, ev, w, nullptr, u, uRec, faceAdj, st);
}

int rhs_jvp_visc(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *du, const real *duRec, const real *u,
                 const real *uRec, real *ffd, cudaStream_t st)
{
    if (ev.s.nVars != NV || !vr.bnd.viscFree)
        return ST_UNSUPPORTED;
    return dispatch(false, m, g, vr, ev, du, duRec, u, uRec, ffd, st);
}
} // namespace dndsb
