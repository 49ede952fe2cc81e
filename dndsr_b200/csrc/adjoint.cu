// Derivatives of the residual path: vector-Jacobian products (reverse mode) and
// Jacobian-vector products (forward mode) of EvaluateRHS and of one VR Jacobi
// sweep, with respect to the cell means u and the reconstruction uRec.
//
// Pointwise derivatives of the Riemann flux and of the boundary ghost states
// come from the templated gas routines instantiated on dual numbers (two
// 10-wide passes per Gauss point: the point states, then the cell means that
// feed the Roe averages); the Gauss-point states are recomputed, not stored.
// The mesh-level reverse sweep is explicit: per-face cotangents are written to
// a scratch array and gathered per cell in a fixed order (no atomics on data),
// and the transposed VR sweep gathers A^-1 B blocks of the neighbours through
// the face-slot map.  The entropy-fix scale deltaLambdaCell is held fixed.
// The viscous flux derivative is added by adjoint_visc.cu (boundary zones without a viscous
// flux only); the SA model and viscous boundary zones go to the forward-mode kernels of
// adjoint_generic.cu.
#include "solver.cuh"
#include "basis_eval.cuh"
#include "bc.cuh"

namespace dndsb
{
namespace
{
constexpr int NV = 5;
using D10 = Dual<10>;
using D1 = Dual<1>;

// u + phi . uRec at one point
template <int R>
DNDSB_D void recon_value(const real *T, const real *u, const real *rec, real *U)
{
    for (int v = 0; v < NV; v++)
    {
        real a = u[v];
        for (int j = 0; j < R; j++)
            a += T[1 + j] * rec[j * NV + v];
        U[v] = a;
    }
}

// cotangent of one interior or boundary face: faceAdj[f][side][(R+1)][NV], entry 0 = d/du, 1+j = d/duRec_j
template <int DIM, int P>
DNDSB_GLOBAL void k_rhs_vjp_face(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ w, const real *__restrict__ u,
                                 const real *__restrict__ uRec, const real *__restrict__ dLamCell, real *__restrict__ faceAdj, int *err,
                                 int boundaryOnly)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1, W = (R + 1) * NV;
    const real gamma = s.gamma;
    // boundaryOnly: the boundary faces of the list m.bndFace (the reverse-mode Roe kernel writes the others)
    DNDSB_KERNEL_LOOP(ii, boundaryOnly ? m.nBndFace : m.nFace)
    {
        const int64_t f = boundaryOnly ? (int64_t)m.bndFace[ii] : ii;
        const real *nMV = s.rsMeanValueEig ? &g.faceMeanNorm[f * 3] : nullptr; // batched mean-value eigenvalues
        int64_t c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        bool bnd = c1 < 0;
        int zone = m.faceZone[f];
        real *o0 = faceAdj + (f * 2) * W, *o1 = faceAdj + (f * 2 + 1) * W;
        for (int i = 0; i < W; i++)
            o0[i] = 0, o1[i] = 0;
        real gbar[NV];
        for (int v = 0; v < NV; v++)
            gbar[v] = w[c0 * NV + v] / g.vol[c0] - (bnd ? 0.0 : w[c1 * NV + v] / g.vol[c1]);
        const real *ULm = u + c0 * NV;
        const real *URm = bnd ? nullptr : u + c1 * NV;
        real dLambda = bnd ? dLamCell[c0] : dmax(dLamCell[c0], dLamCell[c1]);
        real ULmbar[NV] = {0, 0, 0, 0, 0}, URmbar[NV] = {0, 0, 0, 0, 0};
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
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            real Fbar[NV];
            for (int v = 0; v < NV; v++)
                Fbar[v] = -JW * gbar[v];
            real T0[NDOF], T1[NDOF];
            cell_basis<DIM, NDOF>(&g.cellCent[c0 * 3], &g.cellScale[c0 * 3], &vr.baseMoment[c0 * NDOF], vr.s.anisotropicLengths, p0, 1, T0);
            real UL[NV], UR[NV];
            recon_value<R>(T0, u + c0 * NV, uRec + c0 * R * NV, UL);
            real ULbar[NV] = {0, 0, 0, 0, 0}, URbar[NV] = {0, 0, 0, 0, 0};
            D10 F[NV], l0, l1, l4;
            if (!bnd)
            {
                cell_basis<DIM, NDOF>(&g.cellCent[c1 * 3], &g.cellScale[c1 * 3], &vr.baseMoment[c1 * NDOF], vr.s.anisotropicLengths, p1, 1, T1);
                recon_value<R>(T1, u + c1 * NV, uRec + c1 * R * NV, UR);
                // pass 1: point states UL (0..4), UR (5..9)
                D10 ULd[NV], URd[NV], ULmd[NV], URmd[NV];
                for (int v = 0; v < NV; v++)
                    ULd[v] = D10::var(UL[v], v), URd[v] = D10::var(UR[v], 5 + v), ULmd[v] = D10(ULm[v]), URmd[v] = D10(URm[v]);
                bad |= !riemann_flux(s.rsType, ULd, URd, ULmd, URmd, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4, nMV);
                for (int v = 0; v < NV; v++)
                    for (int i = 0; i < NV; i++)
                        ULbar[i] += F[v].d[i] * Fbar[v], URbar[i] += F[v].d[5 + i] * Fbar[v];
                // pass 2: cell means ULm (0..4), URm (5..9) through the Roe averages
                for (int v = 0; v < NV; v++)
                    ULd[v] = D10(UL[v]), URd[v] = D10(UR[v]), ULmd[v] = D10::var(ULm[v], v), URmd[v] = D10::var(URm[v], 5 + v);
                bad |= !riemann_flux(s.rsType, ULd, URd, ULmd, URmd, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4, nMV);
                for (int v = 0; v < NV; v++)
                    for (int i = 0; i < NV; i++)
                        ULmbar[i] += F[v].d[i] * Fbar[v], URmbar[i] += F[v].d[5 + i] * Fbar[v];
            }
            else
            {
                // boundary: UR = ghost(UL) at this point, URm = ghost(ULm) at the face centre
                D10 ULd[NV], URd[NV], ULmd[NV], URmd[NV];
                for (int v = 0; v < NV; v++)
                    ULd[v] = D10::var(UL[v], v), ULmd[v] = D10::var(ULm[v], 5 + v);
                if (!bc_value<NV>(vr.bnd, zone, ULd, n, URd))
                    for (int v = 0; v < NV; v++)
                        URd[v] = ULd[v];
                if (!bc_value<NV>(vr.bnd, zone, ULmd, &g.faceMeanNorm[f * 3], URmd))
                    for (int v = 0; v < NV; v++)
                        URmd[v] = ULmd[v];
                bad |= !riemann_flux(s.rsType, ULd, URd, ULmd, URmd, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4, nMV);
                for (int v = 0; v < NV; v++)
                    for (int i = 0; i < NV; i++)
                        ULbar[i] += F[v].d[i] * Fbar[v], ULmbar[i] += F[v].d[5 + i] * Fbar[v];
            }
            for (int v = 0; v < NV; v++)
            {
                o0[v] += ULbar[v];
                for (int j = 0; j < R; j++)
                    o0[NV + j * NV + v] += T0[1 + j] * ULbar[v];
                if (!bnd)
                {
                    o1[v] += URbar[v];
                    for (int j = 0; j < R; j++)
                        o1[NV + j * NV + v] += T1[1 + j] * URbar[v];
                }
            }
        }
        for (int v = 0; v < NV; v++)
            o0[v] += ULmbar[v], o1[v] += URmbar[v];
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}

// du_c = sum over the cell's faces of the face cotangents of its side (fixed face order)
template <int W>
DNDSB_GLOBAL void k_adj_gather(int64_t nCell, int nf, const int32_t *__restrict__ c2f, const real *__restrict__ faceAdj, real *du, real *duRec)
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

// tangent of the face flux for tangents (du, duRec) of (u, uRec)
template <int DIM, int P>
DNDSB_GLOBAL void k_rhs_jvp_face(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ du, const real *__restrict__ duRec,
                                 const real *__restrict__ u, const real *__restrict__ uRec, const real *__restrict__ dLamCell, real *__restrict__ ffd,
                                 int *err)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real gamma = s.gamma;
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        const real *nMV = s.rsMeanValueEig ? &g.faceMeanNorm[f * 3] : nullptr; // batched mean-value eigenvalues
        int64_t c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        bool bnd = c1 < 0;
        int zone = m.faceZone[f];
        D1 ULm[NV], URm[NV];
        for (int v = 0; v < NV; v++)
        {
            ULm[v] = D1(u[c0 * NV + v]);
            ULm[v].d[0] = du[c0 * NV + v];
        }
        if (bnd)
        {
            if (!bc_value<NV>(vr.bnd, zone, ULm, &g.faceMeanNorm[f * 3], URm))
                for (int v = 0; v < NV; v++)
                    URm[v] = ULm[v];
        }
        else
            for (int v = 0; v < NV; v++)
            {
                URm[v] = D1(u[c1 * NV + v]);
                URm[v].d[0] = du[c1 * NV + v];
            }
        real dLambda = bnd ? dLamCell[c0] : dmax(dLamCell[c0], dLamCell[c1]);
        real acc[NV] = {0, 0, 0, 0, 0};
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
            real T0[NDOF];
            cell_basis<DIM, NDOF>(&g.cellCent[c0 * 3], &g.cellScale[c0 * 3], &vr.baseMoment[c0 * NDOF], vr.s.anisotropicLengths, p0, 1, T0);
            D1 UL[NV], UR[NV];
            for (int v = 0; v < NV; v++)
            {
                real a = u[c0 * NV + v], da = du[c0 * NV + v];
                for (int j = 0; j < R; j++)
                    a += T0[1 + j] * uRec[(c0 * R + j) * NV + v], da += T0[1 + j] * duRec[(c0 * R + j) * NV + v];
                UL[v] = D1(a);
                UL[v].d[0] = da;
            }
            if (bnd)
            {
                if (!bc_value<NV>(vr.bnd, zone, UL, n, UR))
                    for (int v = 0; v < NV; v++)
                        UR[v] = UL[v];
            }
            else
            {
                real T1[NDOF];
                cell_basis<DIM, NDOF>(&g.cellCent[c1 * 3], &g.cellScale[c1 * 3], &vr.baseMoment[c1 * NDOF], vr.s.anisotropicLengths, p1, 1, T1);
                for (int v = 0; v < NV; v++)
                {
                    real a = u[c1 * NV + v], da = du[c1 * NV + v];
                    for (int j = 0; j < R; j++)
                        a += T1[1 + j] * uRec[(c1 * R + j) * NV + v], da += T1[1 + j] * duRec[(c1 * R + j) * NV + v];
                    UR[v] = D1(a);
                    UR[v].d[0] = da;
                }
            }
            D1 F[NV], l0, l1, l4;
            bad |= !riemann_flux(s.rsType, UL, UR, ULm, URm, n, gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4, nMV);
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
            for (int v = 0; v < NV; v++)
                acc[v] -= F[v].d[0] * JW;
        }
        for (int v = 0; v < NV; v++)
            ffd[f * NV + v] = acc[v];
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}

DNDSB_GLOBAL void k_flux_gather(int64_t nCell, int nf, const int32_t *__restrict__ c2f, const real *__restrict__ vol, const real *__restrict__ ff,
                                real *rhs)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        real acc[NV] = {0, 0, 0, 0, 0};
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

// ---------------------------------------------------------------------------
// one Jacobi sweep uRecNew = S(uRec, u) (VariationalReconstruction_Reconstruction.hxx:485-615):
//   uRecNew_i = (1-w) uRec_i + w sum_k [M_ik uRec_k + b_ik (u_k - u_i)] + w A_i^-1 BCC_i(u_i, uRec_i)
// ---------------------------------------------------------------------------
// derivative of the boundary term of cell c: BCC = sum_q w0^2 |J| w phi_q (UB_q - u_c) with
// UB_q = ghost(compress(u_c, u_c + phi_q . uRec_c)); mode 0: VJP of t (R x NV cotangent of BCC)
// into (vRec, vU); mode 1: JVP (dRec, du) -> dBCC
template <int DIM, int P>
DNDSB_D void bcc_derivative(const MeshD &m, const GeomD &g, const VRD &vr, int64_t c, const real *u, const real *uRec, int mode, const real *t,
                            real *vRec, real *vU, const real *dRec, const real *duc, real *dBCC)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
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
            recon_value<R>(T, uc, rc, UL);
            real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q] * w0 * w0;
            // UB as a function of (UL, u_c): independents 0..4 and 5..9
            D10 ULd[NV], umd[NV], ULf[NV], UB[NV];
            for (int v = 0; v < NV; v++)
                ULd[v] = D10::var(UL[v], v), umd[v] = D10::var(uc[v], 5 + v);
            compress_rec<NV>(umd, ULd, ULf);
            if (!bc_value<NV>(vr.bnd, zone, ULf, n, UB))
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
                        gl += UB[v].d[i] * UBbar[v], gm += UB[v].d[5 + i] * UBbar[v];
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
                        dUB += UB[v].d[i] * dUL[i] + UB[v].d[5 + i] * duc[i];
                    real dd = (dUB - duc[v]) * JW;
                    for (int i = 0; i < R; i++)
                        dBCC[i * NV + v] += T[1 + i] * dd;
                }
            }
        }
    }
}

// VJP of the sweep: v = cotangent of uRecNew -> vRec (of uRec), vU (of u); gathered per cell o
template <int DIM, int P>
DNDSB_GLOBAL void k_vr_vjp(MeshD m, GeomD g, VRD vr, const real *__restrict__ v, const real *__restrict__ uRec, const real *__restrict__ u,
                           real *vRec, real *vU)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const real om = vr.s.jacobiRelax;
    const int nf = m.nf;
    DNDSB_KERNEL_LOOP(o, m.nCell)
    {
        real aRec[R * NV], aU[NV] = {0, 0, 0, 0, 0};
        const real *vo = v + o * R * NV;
        for (int i = 0; i < R * NV; i++)
            aRec[i] = (1 - om) * vo[i];
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
            // neighbour i's row k reads uRec_o and u_o: transpose into o
            for (int r = 0; r < R; r++)
                for (int x = 0; x < NV; x++)
                {
                    real a = 0;
                    for (int l = 0; l < R; l++)
                        a += M[l * R + r] * vi[l * NV + x];
                    aRec[r * NV + x] += om * a;
                }
            // b_ik (u_o - u_i): + into o, and o's own row: - b_oj (u_o) for its own slot j
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
            // t = w A_o^-T v_o, the cotangent of BCC_o
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
            bcc_derivative<DIM, P>(m, g, vr, o, u, uRec, 0, t, aRec, aU, nullptr, nullptr, nullptr);
        }
        for (int i = 0; i < R * NV; i++)
            vRec[o * R * NV + i] = aRec[i];
        for (int x = 0; x < NV; x++)
            vU[o * NV + x] = aU[x];
    }
}

// JVP of the sweep: tangents (dRec, du) -> tangent of uRecNew
template <int DIM, int P>
DNDSB_GLOBAL void k_vr_jvp(MeshD m, GeomD g, VRD vr, const real *__restrict__ dRec, const real *__restrict__ du, const real *__restrict__ uRec,
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
            bcc_derivative<DIM, P>(m, g, vr, c, u, uRec, 1, nullptr, nullptr, nullptr, dRec + c * R * NV, du + c * NV, dB);
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

template <int DIM, int P>
int rhs_vjp_dp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *w, const real *u, const real *uRec, real *du, real *duRec,
               cudaStream_t st)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1, W = (R + 1) * NV;
    auto kf = k_rhs_vjp_face<DIM, P>;
    // the hand-reversed Roe kernel takes the point-normal eigenvalues; the batched mean-value variant
    // (rsMeanValueEig with Roe_M1..M5) runs through the forward-mode face kernel on every face
    const int roe = roe_scheme_of(ev.s.rsType) >= 0 && !(ev.s.rsMeanValueEig && ev.s.rsType >= RS_Roe_M1 && ev.s.rsType <= RS_Roe_M1 + 4);
    DNDSB_LAUNCH(kf, roe ? m.nBndFace : m.nFace, 64, st, m, g, vr, ev.s, w, u, uRec, ev.deltaLambdaCell, ev.adjBuf, ev.errWord, roe);
    bool viscDone = false;
    if (roe)
    {
        int rc = rhs_vjp_roe_interior(m, g, vr, ev, w, u, uRec, ev.adjBuf, st, &viscDone);
        if (rc != ST_OK)
            return rc;
    }
    if (!ev.s.ignoreVis && !viscDone)
    {
        int rc = rhs_vjp_visc(m, g, vr, ev, w, u, uRec, ev.adjBuf, st);
        if (rc != ST_OK)
            return rc;
    }
    auto kg = k_adj_gather<W>;
    DNDSB_LAUNCH(kg, m.nCell, 128, st, m.nCell, m.nf, m.cell2face, ev.adjBuf, du, duRec);
    return ST_OK;
}

template <int DIM, int P>
int rhs_jvp_dp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *du, const real *duRec, const real *u, const real *uRec,
               real *dRhs, cudaStream_t st)
{
    auto kf = k_rhs_jvp_face<DIM, P>;
    DNDSB_LAUNCH(kf, m.nFace, 64, st, m, g, vr, ev.s, du, duRec, u, uRec, ev.deltaLambdaCell, ev.adjBuf, ev.errWord);
    if (!ev.s.ignoreVis)
    {
        int rc = rhs_jvp_visc(m, g, vr, ev, du, duRec, u, uRec, ev.adjBuf, st);
        if (rc != ST_OK)
            return rc;
    }
    DNDSB_LAUNCH(k_flux_gather, m.nCell, 256, st, m.nCell, m.nf, m.cell2face, g.vol, ev.adjBuf, dRhs);
    return ST_OK;
}

#define DNDSB_DP_DISPATCH(FN, ...)                                                                         \
    do                                                                                                     \
    {                                                                                                      \
        if (m.dim == 2)                                                                                    \
            return vr.P == 1 ? FN<2, 1>(__VA_ARGS__) : vr.P == 2 ? FN<2, 2>(__VA_ARGS__) : FN<2, 3>(__VA_ARGS__); \
        return vr.P == 1 ? FN<3, 1>(__VA_ARGS__) : vr.P == 2 ? FN<3, 2>(__VA_ARGS__) : FN<3, 3>(__VA_ARGS__);     \
    } while (0)

int ensure_adj(const MeshD &m, const VRD &vr, EvalD &ev)
{
    size_t n = (size_t)m.nFace * 2 * (vr.R + 1) * NV;
    if (ev.adjBuf && ev.adjBufLen >= n)
        return ST_OK;
    dev_free(ev.adjBuf);
    ev.adjBuf = nullptr;
    if (dev_alloc((void **)&ev.adjBuf, sizeof(real) * n) != cudaSuccess)
        return ST_CUDA;
    ev.adjBufLen = n;
    return ST_OK;
}

template <int DIM, int P>
int vr_vjp_dp(const MeshD &m, const GeomD &g, const VRD &vr, const real *v, const real *uRec, const real *u, real *vRec, real *vU,
              cudaStream_t st)
{
    auto k = k_vr_vjp<DIM, P>;
    DNDSB_LAUNCH(k, m.nCell, 64, st, m, g, vr, v, uRec, u, vRec, vU);
    return ST_OK;
}

template <int DIM, int P>
int vr_jvp_dp(const MeshD &m, const GeomD &g, const VRD &vr, const real *dRec, const real *du, const real *uRec, const real *u, real *dNew,
              cudaStream_t st)
{
    auto k = k_vr_jvp<DIM, P>;
    DNDSB_LAUNCH(k, m.nCell, 64, st, m, g, vr, dRec, du, uRec, u, dNew);
    return ST_OK;
}
} // namespace

int rhs_vjp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *w, const real *u, const real *uRec, real *du, real *duRec,
            cudaStream_t st)
{
    // the SA model and viscous boundary zones: the forward-mode kernels of adjoint_generic.cu
    if (ev.s.nVars != NV || (!ev.s.ignoreVis && !vr.bnd.viscFree))
        return rhs_vjp_generic(m, g, vr, ev, w, nullptr, u, uRec, du, duRec, st);
    if (ensure_adj(m, vr, ev) != ST_OK)
        return ST_CUDA;
    dev_zero(ev.errWord, sizeof(int), st);
    int rc = ST_OK;
    auto run = [&]() { DNDSB_DP_DISPATCH(rhs_vjp_dp, m, g, vr, ev, w, u, uRec, du, duRec, st); };
    rc = run();
    if (rc != ST_OK)
        return rc;
    int e = 0;
    d2h(&e, ev.errWord, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess || last_error() != cudaSuccess)
        return ST_CUDA;
    return e ? ST_NONPHYSICAL : ST_OK;
}

int rhs_jvp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *du, const real *duRec, const real *u, const real *uRec,
            real *dRhs, cudaStream_t st)
{
    if (ev.s.nVars != NV || (!ev.s.ignoreVis && !vr.bnd.viscFree))
        return rhs_jvp_generic(m, g, vr, ev, du, duRec, u, uRec, dRhs, st);
    if (ensure_adj(m, vr, ev) != ST_OK)
        return ST_CUDA;
    dev_zero(ev.errWord, sizeof(int), st);
    auto run = [&]() { DNDSB_DP_DISPATCH(rhs_jvp_dp, m, g, vr, ev, du, duRec, u, uRec, dRhs, st); };
    int rc = run();
    if (rc != ST_OK)
        return rc;
    int e = 0;
    d2h(&e, ev.errWord, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess || last_error() != cudaSuccess)
        return ST_CUDA;
    return e ? ST_NONPHYSICAL : ST_OK;
}

int vr_vjp(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *v, const real *uRec, const real *u, real *vRec, real *vU,
           cudaStream_t st)
{
    if (nv != NV)
        return vr_vjp_generic(m, g, vr, nv, v, uRec, u, vRec, vU, st);
    auto run = [&]() { DNDSB_DP_DISPATCH(vr_vjp_dp, m, g, vr, v, uRec, u, vRec, vU, st); };
    int rc = run();
    if (rc != ST_OK)
        return rc;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int vr_jvp(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *dRec, const real *du, const real *uRec, const real *u,
           real *dRecNew, cudaStream_t st)
{
    if (nv != NV)
        return vr_jvp_generic(m, g, vr, nv, dRec, du, uRec, u, dRecNew, st);
    auto run = [&]() { DNDSB_DP_DISPATCH(vr_jvp_dp, m, g, vr, dRec, du, uRec, u, dRecNew, st); };
    int rc = run();
    if (rc != ST_OK)
        return rc;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
