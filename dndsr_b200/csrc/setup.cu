// Setup kernels: geometry metrics, variational-reconstruction base moments,
// face weights and the A^-1 B / A^-1 b coefficient blocks.  One thread per
// cell or face; run once per mesh.
//
// Follows CFV/FiniteVolume.cpp:22-648 (metrics), VariationalReconstruction.cpp
// :56-498 (ConstructBaseAndWeight) and :507-872 (ConstructRecCoeff).
#include "solver.cuh"
#include "basis_eval.cuh"

namespace dndsb
{
namespace
{
DNDSB_D void load_cell_coords(const MeshD &m, int64_t c, real *cs)
{
    for (int v = 0; v < m.nvert; v++)
    {
        int64_t nd = m.cell2node[c * m.nvert + v];
        for (int d = 0; d < 3; d++)
            cs[v * 3 + d] = m.coords[nd * 3 + d] + m.cellShift[(c * m.nvert + v) * 3 + d];
    }
}

DNDSB_D void load_face_coords(const MeshD &m, int64_t f, real *cs)
{
    for (int v = 0; v < m.nfv; v++)
    {
        int64_t nd = m.face2node[f * m.nfv + v];
        for (int d = 0; d < 3; d++)
            cs[v * 3 + d] = m.coords[nd * 3 + d] + m.faceShift[(f * m.nfv + v) * 3 + d];
    }
}

// FiniteVolume.cpp:22-330: volume (order-6 rule), barycentre, centre,
// Jacobian determinants and points of the intOrder rule, aligned half box
// FiniteVolume.cpp:288-335 cellMajorHBox with FiniteVolume.hpp:387-393 GetCellMaxLenScale: twice the
// largest vertex extent along the principal axes of the cell's inertia tensor (integrated at
// INT_ORDER_MAX).  Principal axes by cyclic Jacobi rotations; a fully isotropic tensor keeps the
// coordinate axes, as the reference's diagonal perturbation does.
DNDSB_D real cell_major_length(const MeshD &m, const real *cs, const real *bary, real vol)
{
    real A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    PtGeo pg;
    real p[3], w;
    int nMax = quad_n(m.cellType, kIntOrderMax);
    for (int q = 0; q < nMax; q++)
    {
        quad_point(m.cellType, kIntOrderMax, q, p, w);
        pt_geo(m.cellType, cs, p, pg);
        real J = cell_jdet(m.dim, pg);
        real x[3] = {pg.x[0] - bary[0], pg.x[1] - bary[1], pg.x[2] - bary[2]};
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                A[a][b] += x[a] * x[b] * J * w;
    }
    const int n = m.dim;
    real nrm = 0;
    for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++)
            A[a][b] /= vol, nrm += A[a][b] * A[a][b];
    real V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 50; sweep++)
    {
        real off = 0;
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                off += A[a][b] * A[a][b];
        if (off <= 1e-34 * nrm)
            break;
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
            {
                if (A[a][b] == 0)
                    continue;
                real th = (A[b][b] - A[a][a]) / (2 * A[a][b]);
                real t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1));
                real c = 1 / sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < 3; k++)
                {
                    real x = A[k][a], y = A[k][b];
                    A[k][a] = c * x - s * y, A[k][b] = s * x + c * y;
                }
                for (int k = 0; k < 3; k++)
                {
                    real x = A[a][k], y = A[b][k];
                    A[a][k] = c * x - s * y, A[b][k] = s * x + c * y;
                }
                for (int k = 0; k < 3; k++)
                {
                    real x = V[k][a], y = V[k][b];
                    V[k][a] = c * x - s * y, V[k][b] = s * x + c * y;
                }
            }
    }
    real h = 0;
    for (int k = 0; k < m.nvert; k++)
    {
        real x[3] = {cs[k * 3] - bary[0], cs[k * 3 + 1] - bary[1], cs[k * 3 + 2] - bary[2]};
        for (int a = 0; a < n; a++)
            h = dmax(h, fabs(V[0][a] * x[0] + V[1][a] * x[1] + V[2][a] * x[2]));
    }
    return 2 * h;
}

DNDSB_GLOBAL void k_cell_metrics(MeshD m, int intOrder, GeomD g)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real cs[24];
        load_cell_coords(m, c, cs);
        PtGeo pg;
        real v = 0, p[3], w;
        int nMax = quad_n(m.cellType, kIntOrderMax);
        for (int q = 0; q < nMax; q++)
        {
            quad_point(m.cellType, kIntOrderMax, q, p, w);
            pt_geo(m.cellType, cs, p, pg);
            v += cell_jdet(m.dim, pg) * w;
        }
        v += kVerySmall;
        g.vol[c] = v;
        real b[3] = {0, 0, 0};
        for (int q = 0; q < g.nGc; q++)
        {
            quad_point(m.cellType, intOrder, q, p, w);
            pt_geo(m.cellType, cs, p, pg);
            real J = cell_jdet(m.dim, pg);
            for (int d = 0; d < 3; d++)
            {
                b[d] += pg.x[d] * J * w;
                g.cellPP[(c * g.nGc + q) * 3 + d] = pg.x[d];
            }
            g.cellJDet[c * g.nGc + q] = J + kVerySmall;
        }
        for (int d = 0; d < 3; d++)
            g.cellBary[c * 3 + d] = b[d] / v;
        quad_point(m.cellType, 1, 0, p, w);
        pt_geo(m.cellType, cs, p, pg);
        for (int d = 0; d < 3; d++)
            g.cellCent[c * 3 + d] = pg.x[d];
        for (int d = 0; d < 3; d++)
        {
            real h = 0;
            for (int k = 0; k < m.nvert; k++)
                h = dmax(h, fabs(cs[k * 3 + d] - g.cellBary[c * 3 + d]));
            g.cellScale[c * 3 + d] = h;
        }
        if (m.dim == 2)
            g.cellScale[c * 3 + 2] = 1;
        g.hMax[c] = cell_major_length(m, cs, &g.cellBary[c * 3], v);
    }
}

// FiniteVolume.cpp:352-543: area, centre, Jacobian determinants, points and unit normals, mean normal
DNDSB_GLOBAL void k_face_metrics(MeshD m, int intOrder, GeomD g)
{
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        real cs[12];
        load_face_coords(m, f, cs);
        PtGeo pg;
        real a = 0, nm[3] = {0, 0, 0}, p[3], w, n[3];
        for (int q = 0; q < g.nGf; q++)
        {
            quad_point(m.faceType, intOrder, q, p, w);
            pt_geo(m.faceType, cs, p, pg);
            real J = face_jdet_normal(m.dim, pg, n);
            real nn = sqrt(dot3(n, n));
            a += J * w;
            g.faceJDet[f * g.nGf + q] = J + kVerySmall;
            for (int d = 0; d < 3; d++)
            {
                g.facePP[(f * g.nGf + q) * 3 + d] = pg.x[d];
                g.faceNorm[(f * g.nGf + q) * 3 + d] = n[d] / nn;
                nm[d] += n[d] / nn * J * w;
            }
        }
        g.faceArea[f] = a + kVerySmall;
        real nn = sqrt(dot3(nm, nm));
        for (int d = 0; d < 3; d++)
            g.faceMeanNorm[f * 3 + d] = nm[d] / nn;
        quad_point(m.faceType, 1, 0, p, w);
        pt_geo(m.faceType, cs, p, pg);
        for (int d = 0; d < 3; d++)
            g.faceCent[f * 3 + d] = pg.x[d];
    }
}

// FiniteVolume.cpp:590-648 ConstructCellSmoothScale
DNDSB_GLOBAL void k_smooth_init(MeshD m, GeomD g, real *scale, real *cur)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real s = 0;
        for (int k = 0; k < m.nf; k++)
            s += g.faceArea[m.cell2face[c * m.nf + k] >> 1];
        scale[c] = g.vol[c] / (s + kVerySmall);
        cur[c] = scale[c];
    }
}

DNDSB_GLOBAL void k_smooth_iter(MeshD m, const real *cur, real *nxt)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real nAdj = 0, sum = 0;
        for (int k = 0; k < m.nf; k++)
        {
            int o = m.cellNbr[c * m.nf + k];
            if (o >= 0)
                nAdj += 1, sum += cur[o];
        }
        sum += nAdj * cur[c];
        sum /= nAdj * 2;
        nxt[c] = dmin(cur[c], sum);
    }
}

DNDSB_GLOBAL void k_smooth_ratio(int64_t n, const real *cur, const real *scale, real *ratio)
{
    DNDSB_KERNEL_LOOP(c, n)
    {
        ratio[c] = cur[c] / scale[c];
    }
}

DNDSB_GLOBAL void k_quad_weights(int cellType, int faceType, int intOrder, int nGc, int nGf, real *cw, real *fw)
{
    DNDSB_KERNEL_LOOP(i, 64)
    {
        real p[3], w;
        if (i < nGc)
            quad_point(cellType, intOrder, (int)i, p, w), cw[i] = w;
        if (i < nGf)
            quad_point(faceType, intOrder, (int)i, p, w), fw[i] = w;
    }
}

// VariationalReconstruction.cpp:80-108: cell means of the monomials (order-6 rule)
template <int DIM, int NDOF>
DNDSB_GLOBAL void k_base_moment(MeshD m, GeomD g, int aniso, real *moment)
{
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real cs[24];
        load_cell_coords(m, c, cs);
        real acc[NDOF], T[NDOF], p[3], w;
        for (int k = 0; k < NDOF; k++)
            acc[k] = 0;
        PtGeo pg;
        int nMax = quad_n(m.cellType, kIntOrderMax);
        for (int q = 0; q < nMax; q++)
        {
            quad_point(m.cellType, kIntOrderMax, q, p, w);
            pt_geo(m.cellType, cs, p, pg);
            real J = cell_jdet(DIM, pg);
            cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], nullptr, aniso, pg.x, 1, T);
            for (int k = 0; k < NDOF; k++)
                acc[k] += T[k] * J * w;
        }
        for (int k = 0; k < NDOF; k++)
            moment[c * NDOF + k] = acc[k] / acc[0];
    }
}

// VariationalReconstruction.cpp:200-441: face weight wd*wg per order and the functional length scale
template <int DIM>
DNDSB_GLOBAL void k_face_weight(MeshD m, GeomD g, VRSettingsD s, const real *bcW, int nZone, real *faceWeight, real *faceL)
{
    DNDSB_KERNEL_LOOP(f, m.nFace)
    {
        int c0 = m.face2cell[f * 2], c1 = m.face2cell[f * 2 + 1];
        real dv[3];
        if (c1 >= 0)
            for (int d = 0; d < 3; d++)
                dv[d] = g.cellBary[c1 * 3 + d] - m.facePShift[f * 3 + d] - g.cellBary[c0 * 3 + d];
        else
        {
            real vCB[3];
            for (int d = 0; d < 3; d++)
                vCB[d] = g.faceCent[f * 3 + d] - g.cellBary[c0 * 3 + d];
            real vn = dot3(vCB, &g.faceMeanNorm[f * 3]);
            for (int d = 0; d < 3; d++)
                dv[d] = 2 * vn * g.faceMeanNorm[f * 3 + d];
        }
        real L;
        if (s.scaleType == 1) // BaryDiff: |faceBaryDiffV| over the geometric dimensions
        {
            real q = 0;
            for (int d = 0; d < DIM; d++)
                q += dv[d] * dv[d];
            L = sqrt(q);
        }
        else // MeanAACBB: rms of the sides' averaged aligned half boxes
        {
            real hb[3] = {0, 0, 0};
            int n = 0;
            for (int sd = 0; sd < 2; sd++)
            {
                int c = m.face2cell[f * 2 + sd];
                if (c < 0)
                    continue;
                for (int d = 0; d < 3; d++)
                    hb[d] += g.cellScale[c * 3 + d];
                n++;
            }
            real q = 0;
            for (int d = 0; d < DIM; d++)
                q += sqr(hb[d] / n);
            L = sqrt(q / DIM);
        }
        faceL[f] = L * s.scaleMultiplier;
        real dn = sqrt(dot3(dv, dv));
        real wg = 1;
        if (s.geomWeightScheme == 1)
            wg = s.geomWeightBias + pow(pow(g.faceArea[f], 1. / real(DIM - 1)) / dn, s.geomWeightPower * 0.5);
        else if (s.geomWeightScheme == 2)
            wg = s.geomWeightBias + pow(g.faceArea[f], s.geomWeightPower1 * 0.5) * pow(dn, s.geomWeightPower2 * 0.5);
        int P = s.maxOrder;
        real wd[4] = {0, 0, 0, 0};
        if (s.dirWeightScheme == 0)
        {
            const real inv_fact[4] = {1, 1, 0.5, 1.0 / 6.0};
            for (int p = 0; p <= P; p++)
                wd[p] = inv_fact[p];
        }
        else if (s.dirWeightScheme == 1)
        {
            if (P == 1)
                wd[0] = wd[1] = 1;
            else if (P == 2)
                wd[0] = 1, wd[1] = 0.4643, wd[2] = 0.1559;
            else
                wd[0] = 1, wd[1] = .5295, wd[2] = wd[3] = .2117;
        }
        else
            for (int p = 0; p <= P; p++)
                wd[p] = s.manualDirWeights[p];
        if (c1 < 0)
        {
            int z = m.faceZone[f];
            for (int p = 0; p <= P; p++)
                wd[p] *= (bcW && z < nZone ? bcW[z * 4 + p] : 1.0) * s.bcWeight;
        }
        for (int p = 0; p <= P; p++)
            faceWeight[f * (P + 1) + p] = wd[p] * wg;
    }
}

// VR functional of one face point (VariationalReconstruction.hpp:460-590 with
// AccumulateDiffOrderContributions :32-98): Conj += JW * sum over derivative
// orders of weight^2 * L^(2 order) * <D^k phi_i, D^k phi_j> (combinatorial weights)
template <int DIM, int NDOF>
DNDSB_D void functional_acc(const real *w2L /*per order*/, int maxOrd, const real *DI, const real *DJ, int nJ, real JW, real *Conj)
{
    constexpr int R = NDOF - 1;
    for (int o = maxOrd; o >= 0; o--)
    {
        int k0 = Basis<DIM>::order_start(o), k1 = Basis<DIM>::order_start(o + 1);
        real sc = w2L[o] * JW;
        for (int k = k0; k < k1; k++)
        {
            real ck = Basis<DIM>::ncomb(k) * sc;
            for (int i = 0; i < R; i++)
            {
                real a = DI[k * NDOF + 1 + i] * ck;
                if (a == 0)
                    continue;
                for (int j = 0; j < nJ; j++)
                    Conj[i * nJ + j] += a * DJ[k * NDOF + (nJ == 1 ? 0 : 1 + j)];
            }
        }
    }
}

template <int DIM, int P>
DNDSB_D void face_w2L(const VRD &vr, int64_t f, real *w2L)
{
    real L = vr.faceL[f];
    real L2 = L * L, Lp = 1;
    for (int o = 0; o <= P; o++)
    {
        real w = vr.faceWeight[f * (P + 1) + o];
        w2L[o] = w * w * (L == 0 ? 1.0 : Lp);
        Lp *= L2;
    }
}

// VariationalReconstruction.cpp:507-824: A, B_k, b_k, A^-1 and the products, one cell per thread
template <int DIM, int P>
DNDSB_GLOBAL void k_vr_coeff(MeshD m, GeomD g, VRD vr, int *err)
{
    constexpr int NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        real A[R * R], Ai[R * R], B[R * R], b[R];
        real TI[NDOF * NDOF], TJ[NDOF * NDOF], w2L[P + 1];
        const real one[1] = {1.0};
        bool aniso = vr.s.anisotropicLengths;
        for (int i = 0; i < R * R; i++)
            A[i] = 0;
        // pass 1: A = sum over all faces of the self functional
        for (int k = 0; k < m.nf; k++)
        {
            int fp = m.cell2face[c * m.nf + k];
            int64_t f = fp >> 1;
            int side = fp & 1;
            face_w2L<DIM, P>(vr, f, w2L);
            for (int q = 0; q < g.nGf; q++)
            {
                real p[3];
                for (int d = 0; d < 3; d++)
                    p[d] = g.facePP[(f * g.nGf + q) * 3 + d] + (side ? m.facePShift[f * 3 + d] : 0.0);
                cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], &vr.baseMoment[c * NDOF], aniso, p, NDOF, TI);
                functional_acc<DIM, NDOF>(w2L, P, TI, TI, R, g.faceJDet[f * g.nGf + q] * g.faceQw[q], A);
            }
        }
        for (int i = 0; i < R * R; i++)
            vr.matA[c * R * R + i] = A[i];
        if (!invert_gj<R>(A, Ai))
        {
            atomicOr(err, (int)DE_SINGULAR);
            continue;
        }
        real *blk = vr.AAInvB + c * (m.nf + 1) * R * R;
        for (int i = 0; i < R * R; i++)
            blk[i] = Ai[i];
        // pass 2: B_k and b_k per face, then A^-1 B_k and A^-1 b_k
        for (int k = 0; k < m.nf; k++)
        {
            int fp = m.cell2face[c * m.nf + k];
            int64_t f = fp >> 1;
            int side = fp & 1;
            int o = m.cellNbr[c * m.nf + k];
            face_w2L<DIM, P>(vr, f, w2L);
            for (int i = 0; i < R * R; i++)
                B[i] = 0;
            for (int i = 0; i < R; i++)
                b[i] = 0;
            for (int q = 0; q < g.nGf; q++)
            {
                real p[3], po[3];
                for (int d = 0; d < 3; d++)
                {
                    real x = g.facePP[(f * g.nGf + q) * 3 + d], sh = m.facePShift[f * 3 + d];
                    p[d] = x + (side ? sh : 0.0);
                    po[d] = x + (side ? 0.0 : sh);
                }
                real JW = g.faceJDet[f * g.nGf + q] * g.faceQw[q];
                cell_basis<DIM, NDOF>(&g.cellCent[c * 3], &g.cellScale[c * 3], &vr.baseMoment[c * NDOF], aniso, p, NDOF, TI);
                if (o >= 0)
                {
                    cell_basis<DIM, NDOF>(&g.cellCent[o * 3], &g.cellScale[o * 3], &vr.baseMoment[o * NDOF], aniso, po, NDOF, TJ);
                    functional_acc<DIM, NDOF>(w2L, P, TI, TJ, R, JW, B);
                }
                functional_acc<DIM, NDOF>(w2L, 0, TI, one, 1, JW, b);
            }
            real *Mk = blk + (1 + k) * R * R;
            real *bk = vr.AInvb + (c * m.nf + k) * R;
            for (int i = 0; i < R; i++)
            {
                for (int j = 0; j < R; j++)
                {
                    real acc = 0;
                    if (o >= 0)
                        for (int l = 0; l < R; l++)
                            acc += Ai[i * R + l] * B[l * R + j];
                    Mk[i * R + j] = acc;
                }
                real acc = 0;
                if (o >= 0)
                    for (int l = 0; l < R; l++)
                        acc += Ai[i * R + l] * b[l];
                bk[i] = acc;
            }
        }
    }
}

// packed sweep coefficients [cell][face k][j][i]: entry (i, j) of A^-1 B_k for j < R, (A^-1 b_k)_i for j = R
DNDSB_GLOBAL void k_pack_sweep(int64_t nCell, int nf, int R, const real *__restrict__ AAInvB, const real *__restrict__ AInvb, real *out,
                               float *out32)
{
    const int64_t per = (int64_t)nf * R * (R + 1);
    DNDSB_KERNEL_LOOP(e, nCell * per)
    {
        int64_t c = e / per;
        int r = (int)(e - c * per);
        // layout [cell][face k][j][i]: j < R is column j of A^-1 B_k, j = R is A^-1 b_k
        int k = r / (R * (R + 1));
        int rem = r - k * R * (R + 1);
        int j = rem / R, i = rem - j * R;
        real v = j < R ? AAInvB[((c * (nf + 1) + 1 + k) * R + i) * R + j] : AInvb[(c * nf + k) * R + i];
        out[e] = v;
        out32[e] = (float)v;
    }
}

DNDSB_GLOBAL void k_to_f32(int64_t n, const real *a, float *b)
{
    DNDSB_KERNEL_LOOP(i, n)
    {
        b[i] = (float)a[i];
    }
}

int alloc_real(real **p, int64_t n)
{
    return dev_alloc((void **)p, sizeof(real) * n) == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace

int geom_construct(const MeshD &m, const VRSettingsD &s, GeomD &g, cudaStream_t st)
{
    g.nGc = quad_n(m.cellType, s.intOrder);
    g.nGf = quad_n(m.faceType, s.intOrder);
    int rc = ST_OK;
    rc |= alloc_real(&g.vol, m.nCell);
    rc |= alloc_real(&g.cellBary, m.nCell * 3);
    rc |= alloc_real(&g.cellCent, m.nCell * 3);
    rc |= alloc_real(&g.cellScale, m.nCell * 3);
    rc |= alloc_real(&g.cellJDet, m.nCell * g.nGc);
    rc |= alloc_real(&g.cellPP, m.nCell * g.nGc * 3);
    rc |= alloc_real(&g.smoothRatio, m.nCell);
    rc |= alloc_real(&g.hMax, m.nCell);
    rc |= alloc_real(&g.faceArea, m.nFace);
    rc |= alloc_real(&g.faceCent, m.nFace * 3);
    rc |= alloc_real(&g.faceJDet, m.nFace * g.nGf);
    rc |= alloc_real(&g.facePP, m.nFace * g.nGf * 3);
    rc |= alloc_real(&g.faceNorm, m.nFace * g.nGf * 3);
    rc |= alloc_real(&g.faceMeanNorm, m.nFace * 3);
    rc |= alloc_real(&g.cellQw, 64);
    rc |= alloc_real(&g.faceQw, 64);
    if (rc)
        return ST_CUDA;
    DNDSB_LAUNCH(k_quad_weights, 64, 64, st, m.cellType, m.faceType, s.intOrder, g.nGc, g.nGf, g.cellQw, g.faceQw);
    DNDSB_LAUNCH(k_cell_metrics, m.nCell, 128, st, m, s.intOrder, g);
    DNDSB_LAUNCH(k_face_metrics, m.nFace, 128, st, m, s.intOrder, g);
    real *scale = nullptr, *a = nullptr, *b = nullptr;
    if (alloc_real(&scale, m.nCell) | alloc_real(&a, m.nCell) | alloc_real(&b, m.nCell))
        return ST_CUDA;
    DNDSB_LAUNCH(k_smooth_init, m.nCell, 256, st, m, g, scale, a);
    for (int it = 1; it <= 15; it++) // nIterCellSmoothScale default (FiniteVolumeSettings.hpp)
    {
        DNDSB_LAUNCH(k_smooth_iter, m.nCell, 256, st, m, a, b);
        real *t = a;
        a = b, b = t;
    }
    DNDSB_LAUNCH(k_smooth_ratio, m.nCell, 256, st, m.nCell, a, scale, g.smoothRatio);
    dev_sync(st);
    dev_free(scale), dev_free(a), dev_free(b);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int vr_construct_base_and_weight(const MeshD &m, const GeomD &g, VRD &vr, const real *bcDirWeightHost, int nZone, cudaStream_t st)
{
    int P = vr.s.maxOrder;
    if (P < 1 || P > 3 || (m.dim != 2 && m.dim != 3))
        return ST_UNSUPPORTED;
    vr.P = P;
    vr.NDOF = m.dim == 2 ? (P == 1 ? 3 : P == 2 ? 6 : 10) : (P == 1 ? 4 : P == 2 ? 10 : 20);
    vr.R = vr.NDOF - 1;
    if (alloc_real(&vr.baseMoment, m.nCell * vr.NDOF) | alloc_real(&vr.faceWeight, m.nFace * (P + 1)) | alloc_real(&vr.faceL, m.nFace))
        return ST_CUDA;
    real *bcW = nullptr;
    if (bcDirWeightHost && nZone > 0)
    {
        if (alloc_real(&bcW, nZone * 4))
            return ST_CUDA;
        h2d(bcW, bcDirWeightHost, sizeof(real) * nZone * 4, st);
    }
    int an = vr.s.anisotropicLengths;
#define DNDSB_BM(D, N) DNDSB_LAUNCH((k_base_moment<D, N>), m.nCell, 128, st, m, g, an, vr.baseMoment)
    if (m.dim == 2)
    {
        if (vr.NDOF == 3)
            DNDSB_BM(2, 3);
        else if (vr.NDOF == 6)
            DNDSB_BM(2, 6);
        else
            DNDSB_BM(2, 10);
        DNDSB_LAUNCH(k_face_weight<2>, m.nFace, 128, st, m, g, vr.s, bcW, nZone, vr.faceWeight, vr.faceL);
    }
    else
    {
        if (vr.NDOF == 4)
            DNDSB_BM(3, 4);
        else if (vr.NDOF == 10)
            DNDSB_BM(3, 10);
        else
            DNDSB_BM(3, 20);
        DNDSB_LAUNCH(k_face_weight<3>, m.nFace, 128, st, m, g, vr.s, bcW, nZone, vr.faceWeight, vr.faceL);
    }
#undef DNDSB_BM
    dev_sync(st);
    dev_free(bcW);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int vr_construct_rec_coeff(const MeshD &m, const GeomD &g, VRD &vr, int *errWord, cudaStream_t st)
{
    int R = vr.R;
    int64_t nA = m.nCell * (m.nf + 1) * R * R, nb = m.nCell * m.nf * R;
    if (alloc_real(&vr.AAInvB, nA) | alloc_real(&vr.AInvb, nb) | alloc_real(&vr.matA, m.nCell * R * R))
        return ST_CUDA;
    if (dev_alloc((void **)&vr.AAInvB32, sizeof(float) * nA) != cudaSuccess || dev_alloc((void **)&vr.AInvb32, sizeof(float) * nb) != cudaSuccess)
        return ST_CUDA;
    dev_zero(errWord, sizeof(int), st);
#define DNDSB_RC(D, PP) DNDSB_LAUNCH((k_vr_coeff<D, PP>), m.nCell, 64, st, m, g, vr, errWord)
    if (m.dim == 2)
    {
        if (vr.P == 1)
            DNDSB_RC(2, 1);
        else if (vr.P == 2)
            DNDSB_RC(2, 2);
        else
            DNDSB_RC(2, 3);
    }
    else
    {
        if (vr.P == 1)
            DNDSB_RC(3, 1);
        else if (vr.P == 2)
            DNDSB_RC(3, 2);
        else
            DNDSB_RC(3, 3);
    }
#undef DNDSB_RC
    DNDSB_LAUNCH(k_to_f32, nA, 256, st, nA, vr.AAInvB, vr.AAInvB32);
    DNDSB_LAUNCH(k_to_f32, nb, 256, st, nb, vr.AInvb, vr.AInvb32);
    {
        int64_t nS = m.nCell * m.nf * R * (R + 1);
        dev_free(vr.sweepCoef), dev_free(vr.sweepCoef32);
        vr.sweepCoef = nullptr, vr.sweepCoef32 = nullptr;
        if (alloc_real(&vr.sweepCoef, nS) || dev_alloc((void **)&vr.sweepCoef32, sizeof(float) * nS) != cudaSuccess)
            return ST_CUDA;
        DNDSB_LAUNCH(k_pack_sweep, nS, 256, st, m.nCell, m.nf, R, vr.AAInvB, vr.AInvb, vr.sweepCoef, vr.sweepCoef32);
    }
    int e = 0;
    d2h(&e, errWord, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess || last_error() != cudaSuccess)
        return ST_CUDA;
    return (e & DE_SINGULAR) ? ST_NONFINITE : ST_OK;
}
} // namespace dndsb
