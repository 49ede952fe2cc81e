// WBAP_C limiter of the reconstruction (EulerSolver.hxx:455-556 with smoothIndicatorProcedure 0,
// limiterProcedure 1, limiterBiwayAlter 0, normWBAP false), 3-D, 5 or 6 variables, VR degree 1-2:
//   k_lim_secondary     VariationalReconstruction.cpp:840-866 matrixSecondary: per interior face the
//                       maps between the two cells' derivative bases at the face centre
//                       (DiffI^-1 DiffJ and DiffJ^-1 DiffI), built once per reconstruction;
//   k_smooth_face/_gather  VariationalReconstruction_LimiterProcedure.hxx:40-108 (density and energy),
//                       each interior face's terms once, then summed per cell;
//   k_limiter_wbap_c    VariationalReconstruction_LimiterProcedure.hxx:188-334 with the WBAP-L2 biway
//                       and multiway functions (Limiters.hpp:361-470) in the characteristic variables of
//                       the face (Gas.hpp:120-200 eigenvectors, Geometric.hpp:135-160 normal frame).
// One thread per face or cell; the per-cell work (orders from the highest down, each face's
// neighbour mapped, projected, limited and projected back, then the multiway average) is local.
#include "solver.cuh"
#include "basis_eval.cuh"

namespace dndsb
{
namespace
{
constexpr real kPDiP = 1e-50; // verySmallReal^(1/4), Limiters.hpp

template <int P>
DNDSB_GLOBAL void k_lim_secondary(MeshD m, GeomD g, VRD vr, real *__restrict__ sec, int *err)
{
    constexpr int NDOF = ndof_of<3>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        const int cL = m.face2cell[f * 2], cR = m.face2cell[f * 2 + 1];
        if (cR < 0)
            continue;
        real T[NDOF * NDOF], DI[R * R], DJ[R * R], A[R * R], Ai[R * R];
        real p[3];
        for (int d = 0; d < 3; d++)
            p[d] = g.faceCent[f * 3 + d];
        cell_basis<3, NDOF>(&g.cellCent[cL * 3], &g.cellScale[cL * 3], &vr.baseMoment[(int64_t)cL * NDOF], vr.s.anisotropicLengths, p, NDOF, T);
        for (int r = 0; r < R; r++)
            for (int j = 0; j < R; j++)
                DI[r * R + j] = T[(r + 1) * NDOF + 1 + j];
        for (int d = 0; d < 3; d++)
            p[d] += m.facePShift[f * 3 + d];
        cell_basis<3, NDOF>(&g.cellCent[cR * 3], &g.cellScale[cR * 3], &vr.baseMoment[(int64_t)cR * NDOF], vr.s.anisotropicLengths, p, NDOF, T);
        for (int r = 0; r < R; r++)
            for (int j = 0; j < R; j++)
                DJ[r * R + j] = T[(r + 1) * NDOF + 1 + j];
        for (int side = 0; side < 2; side++)
        {
            const real *X = side ? DJ : DI, *Y = side ? DI : DJ;
            for (int i = 0; i < R * R; i++)
                A[i] = X[i];
            if (!invert_gj<R>(A, Ai))
            {
                atomicOr(err, (int)DE_SINGULAR);
                continue;
            }
            real *S = sec + ((int64_t)f * 2 + side) * R * R;
            for (int i = 0; i < R; i++)
                for (int j = 0; j < R; j++)
                {
                    real a = 0;
                    for (int l = 0; l < R; l++)
                        a += Ai[i * R + l] * Y[l * R + j];
                    S[i * R + j] = a;
                }
        }
    }
}

// face functional weights of order o: w^2 L^(2o) (VariationalReconstruction.hpp:460-590)
template <int P>
DNDSB_D void lim_w2L(const VRD &vr, int64_t f, real *w2L)
{
    const real L = vr.faceL[f];
    real Lp = 1;
    for (int o = 0; o <= P; o++)
    {
        const real w = vr.faceWeight[f * (P + 1) + o];
        w2L[o] = w * w * (L == 0 ? 1.0 : Lp);
        Lp *= L * L;
    }
}

// per interior face: the jump and mean functionals of density and energy at the face centre, times
// the face area (the terms both cells of the face add); boundary faces contribute nothing
template <int P>
DNDSB_GLOBAL void k_smooth_face(MeshD m, GeomD g, VRD vr, int nv, const real *__restrict__ u, const real *__restrict__ uRec,
                                real *__restrict__ faceTerm)
{
    constexpr int NDOF = ndof_of<3>(P), R = NDOF - 1;
    const int vs[2] = {0, 4};
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        const int c1 = m.face2cell[f * 2 + 1];
        real *out = faceTerm + f * 4;
        if (c1 < 0)
        {
            for (int i = 0; i < 4; i++)
                out[i] = 0;
            continue;
        }
        real val[2][NDOF * 2];
        for (int sd = 0; sd < 2; sd++)
        {
            const int64_t cc = m.face2cell[f * 2 + sd];
            real p[3], T[NDOF * NDOF];
            for (int d = 0; d < 3; d++)
                p[d] = g.faceCent[f * 3 + d] + (sd ? m.facePShift[f * 3 + d] : 0.0);
            cell_basis<3, NDOF>(&g.cellCent[cc * 3], &g.cellScale[cc * 3], &vr.baseMoment[cc * NDOF], vr.s.anisotropicLengths, p, NDOF, T);
            for (int r = 0; r < NDOF; r++)
                for (int q = 0; q < 2; q++)
                {
                    real a = 0;
                    for (int j = 0; j < R; j++)
                        a += T[r * NDOF + 1 + j] * uRec[(cc * R + j) * nv + vs[q]];
                    if (r == 0)
                        a += u[cc * nv + vs[q]];
                    val[sd][r * 2 + q] = a;
                }
        }
        real w2L[P + 1];
        lim_w2L<P>(vr, f, w2L);
        real IJ[2] = {0, 0}, IS[2] = {0, 0};
        for (int ob = P; ob >= 0; ob--)
            for (int kk = Basis<3>::order_start(ob); kk < Basis<3>::order_start(ob + 1); kk++)
                for (int q = 0; q < 2; q++)
                {
                    const real jm = (val[0][kk * 2 + q] - val[1][kk * 2 + q]) * 0.5, av = (val[0][kk * 2 + q] + val[1][kk * 2 + q]) * 0.5;
                    IJ[q] += jm * jm * Basis<3>::ncomb(kk) * w2L[ob];
                    IS[q] += av * av * Basis<3>::ncomb(kk) * w2L[ob];
                }
        for (int q = 0; q < 2; q++)
            out[q] = IJ[q] * g.faceArea[f], out[2 + q] = IS[q] * g.faceArea[f];
    }
}

// per cell: the sums over its faces, si = sqrt(max over the two variables of IJ / IS) maxOrder^2
DNDSB_GLOBAL void k_smooth_gather(MeshD m, int maxOrder, const real *__restrict__ faceTerm, real *__restrict__ si)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real S[4] = {0, 0, 0, 0};
        for (int k = 0; k < m.nf; k++)
        {
            const int64_t f = m.cell2face[c * m.nf + k] >> 1;
            for (int i = 0; i < 4; i++)
                S[i] += faceTerm[f * 4 + i];
        }
        real sm = 0;
        for (int q = 0; q < 2; q++)
            sm = fmax(sm, fabs(S[q] / (S[2 + q] + kVerySmall)));
        si[c] = sqrt(sm) * (real)(maxOrder * maxOrder);
    }
}

// the face's characteristic projection (toChar: left eigenvectors) or its inverse (right
// eigenvectors) at the mean of the two cell states, in the normal-aligned frame
DNDSB_D void lim_char_matrix(const real *uL, const real *uR, const real *n, real gamma, bool toChar, real M[5][5])
{
    real UC[5];
    for (int i = 0; i < 5; i++)
        UC[i] = (uL[i] + uR[i]) * 0.5;
    // Geometric.hpp:135-160: columns n, t1 = -(n x e_z) (or -(n x e_y)) normalised, t2 = n x t1 normalised
    real B[3][3], t[3];
    if (fabs(n[2]) < 0.9)
        t[0] = -n[1], t[1] = n[0], t[2] = 0;
    else
        t[0] = n[2], t[1] = 0, t[2] = -n[0];
    const real tn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    for (int d = 0; d < 3; d++)
        t[d] /= tn;
    real s[3] = {n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2], n[0] * t[1] - n[1] * t[0]};
    const real sn = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (int d = 0; d < 3; d++)
        B[d][0] = n[d], B[d][1] = t[d], B[d][2] = s[d] / sn;
    const real m0 = UC[1], m1 = UC[2], m2 = UC[3];
    for (int d = 0; d < 3; d++)
        UC[1 + d] = B[0][d] * m0 + B[1][d] * m1 + B[2][d] * m2;
    const real v[3] = {UC[1] / UC[0], UC[2] / UC[0], UC[3] / UC[0]};
    const real vsq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const real p = (gamma - 1) * (UC[4] - 0.5 * UC[0] * vsq);
    const real a2 = gamma * p / UC[0], a = sqrt(a2), H = (UC[4] + p) / UC[0], gb = gamma - 1;
    real E[5][5];
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++)
            E[i][j] = 0;
    if (toChar)
    {
        // Gas.hpp:160-200 left eigenvectors, then columns 1..3 times B^T
        const real sc = gb / (2 * a2);
        E[0][0] = H + a / gb * (v[0] - a), E[0][1] = -v[0] - a / gb, E[0][2] = -v[1], E[0][3] = -v[2], E[0][4] = 1;
        E[1][0] = -2 * H + 4 / gb * a2, E[1][1] = 2 * v[0], E[1][2] = 2 * v[1], E[1][3] = 2 * v[2], E[1][4] = -2;
        E[2][0] = v[1] * (-2 * a2 / gb), E[3][0] = v[2] * (-2 * a2 / gb);
        E[2][2] = E[3][3] = 2 * a2 / gb;
        E[4][0] = H - a / gb * (v[0] + a), E[4][1] = -v[0] + a / gb, E[4][2] = -v[1], E[4][3] = -v[2], E[4][4] = 1;
        for (int i = 0; i < 5; i++)
        {
            for (int j = 0; j < 5; j++)
                E[i][j] *= sc;
            M[i][0] = E[i][0], M[i][4] = E[i][4];
            for (int d = 0; d < 3; d++)
                M[i][1 + d] = E[i][1] * B[d][0] + E[i][2] * B[d][1] + E[i][3] * B[d][2];
        }
    }
    else
    {
        // Gas.hpp:120-158 right eigenvectors, then rows 1..3 = B times them
        E[0][0] = E[0][1] = E[0][4] = 1;
        E[2][2] = E[3][3] = 1;
        for (int d = 0; d < 3; d++)
            E[1 + d][0] = v[d], E[1 + d][1] = v[d], E[1 + d][4] = v[d];
        E[1][0] -= a, E[1][4] += a;
        E[4][0] = H - v[0] * a, E[4][4] = H + v[0] * a, E[4][1] = 0.5 * vsq, E[4][2] = v[1], E[4][3] = v[2];
        for (int j = 0; j < 5; j++)
        {
            M[0][j] = E[0][j], M[4][j] = E[4][j];
            for (int d = 0; d < 3; d++)
                M[1 + d][j] = B[d][0] * E[1][j] + B[d][1] * E[2][j] + B[d][2] * E[3][j];
        }
    }
}

template <int NV>
DNDSB_D void lim_apply(const real M[5][5], int rows, real *data)
{
    for (int r = 0; r < rows; r++)
    {
        real x[5], y[5];
        for (int i = 0; i < 5; i++)
            x[i] = data[r * NV + i];
        for (int i = 0; i < 5; i++)
        {
            y[i] = 0;
            for (int j = 0; j < 5; j++)
                y[i] += M[i][j] * x[j];
        }
        for (int i = 0; i < 5; i++)
            data[r * NV + i] = y[i];
    }
}

DNDSB_D real lim_sign(real x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

template <int P, int NV>
DNDSB_GLOBAL void __launch_bounds__(64) k_limiter_wbap_c(MeshD m, GeomD g, VRD vr, const real *__restrict__ sec, const real *__restrict__ u,
                                                         const real *__restrict__ uRec, const real *__restrict__ si, real *__restrict__ uRecNew,
                                                         real threshold, real nStd, int ifAll, real gamma)
{
    constexpr int NDOF = ndof_of<3>(P), R = NDOF - 1, NRMAX = P == 1 ? 3 : 6, MAXF = 6;
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        const real *rc = uRec + c * R * NV;
        real *out = uRecNew + c * R * NV;
        if (!ifAll && si[c] < threshold)
        {
            for (int i = 0; i < R * NV; i++)
                out[i] = rc[i];
            continue;
        }
        real uFaces[MAXF][R * NV];
        for (int cp = P; cp >= 1; cp--)
        {
            const int ls = Basis<3>::order_start(cp) - 1, le = Basis<3>::order_start(cp + 1) - 2, nr = le - ls + 1;
            real others[MAXF][NRMAX * NV];
            int nO = 0;
            for (int k = 0; k < m.nf; k++)
            {
                const int o = m.cellNbr[c * m.nf + k];
                if (o < 0)
                    continue;
                const int fp = m.cell2face[c * m.nf + k];
                const int64_t f = fp >> 1;
                const int side = fp & 1;
                const real *Mt = sec + ((int64_t)f * 2 + side) * R * R, *Mo = sec + ((int64_t)f * 2 + 1 - side) * R * R;
                const real *ro = uRec + (int64_t)o * R * NV;
                real uoo[R * NV];
                for (int i = 0; i < R * NV; i++)
                    uoo[i] = ro[i];
                // successive small reconstruction: the neighbour's higher orders from this face's limited ones
                for (int i = le + 1; i < R; i++)
                    for (int v = 0; v < NV; v++)
                    {
                        real a = 0;
                        for (int j = le + 1; j < R; j++)
                            a += Mo[i * R + j] * uFaces[k][j * NV + v];
                        uoo[i * NV + v] = a;
                    }
                real oin[NRMAX * NV], tin[NRMAX * NV];
                for (int i = 0; i < nr; i++)
                    for (int v = 0; v < NV; v++)
                    {
                        real a = 0;
                        for (int j = 0; j < R; j++)
                            a += Mt[(ls + i) * R + j] * uoo[j * NV + v];
                        oin[i * NV + v] = a;
                        tin[i * NV + v] = rc[(ls + i) * NV + v];
                    }
                const real *uL = side == 0 ? u + c * NV : u + (int64_t)o * NV, *uR = side == 0 ? u + (int64_t)o * NV : u + c * NV;
                const real *n = &g.faceMeanNorm[f * 3];
                real Ml[5][5], Mr[5][5];
                lim_char_matrix(uL, uR, n, gamma, true, Ml);
                lim_char_matrix(uL, uR, n, gamma, false, Mr);
                lim_apply<NV>(Ml, nr, oin);
                lim_apply<NV>(Ml, nr, tin);
                real *lim = others[nO];
                for (int i = 0; i < nr * NV; i++)
                {
                    const real u1 = tin[i], u2 = oin[i];
                    const real fr = u1 / (fabs(u2) + kPDiP) * lim_sign(u2);
                    const real t1 = fr * fr * fr, t2 = (fr * fr) * (fr * fr);
                    lim[i] = u1 * (1 + t1) / (1 + t2) * fabs(lim_sign(u2));
                }
                lim_apply<NV>(Mr, nr, lim);
                for (int i = 0; i < nr * NV; i++)
                    uFaces[k][ls * NV + i] = lim[i];
                nO++;
            }
            for (int i = 0; i < nr * NV; i++)
            {
                const real c0 = rc[ls * NV + i];
                real up = 0, down = 0, cent = c0;
                for (int q = 0; q < nO; q++)
                {
                    const real ti = c0 / (fabs(others[q][i]) + kPDiP) * lim_sign(others[q][i]);
                    down += (ti * ti) * (ti * ti);
                    up += ti * ti * ti;
                    cent *= fabs(lim_sign(others[q][i]));
                }
                out[ls * NV + i] = cent * (up + nStd) / (down + nStd);
            }
        }
    }
}
} // namespace

int lim_secondary_build(const MeshD &m, const GeomD &g, const VRD &vr, real **sec, int *errWord, cudaStream_t st)
{
    if (*sec)
        return ST_OK;
    if (m.dim != 3 || vr.P < 1 || vr.P > 2)
        return ST_UNSUPPORTED;
    const int R = vr.R;
    if (dev_alloc((void **)sec, sizeof(real) * m.nFace * 2 * R * R) != cudaSuccess)
        return ST_CUDA;
    dev_zero(*sec, sizeof(real) * m.nFace * 2 * R * R, st);
    dev_zero(errWord, sizeof(int), st);
    if (vr.P == 1)
        DNDSB_LAUNCH(k_lim_secondary<1>, m.nFace, 128, st, m, g, vr, *sec, errWord);
    else
        DNDSB_LAUNCH(k_lim_secondary<2>, m.nFace, 128, st, m, g, vr, *sec, errWord);
    int e = 0;
    d2h(&e, errWord, sizeof(int), st);
    if (last_error() != cudaSuccess || dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    if (e & DE_SINGULAR)
    {
        dev_free(*sec);
        *sec = nullptr;
        return ST_NONFINITE;
    }
    return ST_OK;
}

int smooth_indicator(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *u, const real *uRec, real **faceTerm, real *si,
                     cudaStream_t st)
{
    if (m.dim != 3 || vr.P < 1 || vr.P > 2 || (nv != 5 && nv != 6))
        return ST_UNSUPPORTED;
    if (!*faceTerm && dev_alloc((void **)faceTerm, sizeof(real) * 4 * m.nFace) != cudaSuccess)
        return ST_CUDA;
    if (vr.P == 1)
        DNDSB_LAUNCH(k_smooth_face<1>, m.nFace, 128, st, m, g, vr, nv, u, uRec, *faceTerm);
    else
        DNDSB_LAUNCH(k_smooth_face<2>, m.nFace, 128, st, m, g, vr, nv, u, uRec, *faceTerm);
    DNDSB_LAUNCH(k_smooth_gather, m.nCell, 256, st, m, vr.s.maxOrder, *faceTerm, si);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int limiter_wbap_c(const MeshD &m, const GeomD &g, const VRD &vr, const real *sec, int nv, real gamma, const real *u, const real *uRec,
                   const real *si, real *uRecNew, real threshold, real nStd, int ifAll, cudaStream_t st)
{
    if (m.dim != 3 || vr.P < 1 || vr.P > 2 || (nv != 5 && nv != 6) || m.nf > 6)
        return ST_UNSUPPORTED;
#define DNDSB_LIM(PP, NVV) \
    DNDSB_LAUNCH((k_limiter_wbap_c<PP, NVV>), m.nCell, 64, st, m, g, vr, sec, u, uRec, si, uRecNew, threshold, nStd, ifAll, gamma)
    if (vr.P == 1)
    {
        if (nv == 5)
            DNDSB_LIM(1, 5);
        else
            DNDSB_LIM(1, 6);
    }
    else if (nv == 5)
        DNDSB_LIM(2, 5);
    else
        DNDSB_LIM(2, 6);
#undef DNDSB_LIM
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
