// Derivatives of the residual path with respect to the mesh node coordinates: the per-cell
// recomputation in dual numbers shared by adjoint_geom.cu (3-D) and adjoint_geom2d.cu (2-D).
//
// The reference computes the geometry once per mesh (FiniteVolume.cpp:22-648), the VR basis
// moments, face weights and A^-1 B / A^-1 b once (VariationalReconstruction.cpp:56-872), and
// then the residual: the VR sweep (VariationalReconstruction_Reconstruction.hxx:19-176,485-615)
// and EvaluateRHS (EulerEvaluator_EvaluateRHS.hxx:55-818).  Every entry of a cell's residual
// depends on the coordinates of a small patch of nodes: the cell's own and those of its face
// neighbours (centres, barycentres, half boxes and basis moments of both sides of each face; the
// face points, normals, Jacobians and weights).  These kernels recompute that chain for one cell
// in dual numbers, in the order the setup kernels use:
//   * VJP: one thread per (cell, patch node) with the node's three coordinates seeded
//     (Dual<3>); the cell's residual derivatives contracted with the cotangent give the node's
//     share, and a gather in node order sums the shares (deterministic, no atomics);
//   * JVP: one thread per cell with a coordinate direction seeded on every node (Dual<1>).
// The cell means u, the reconstruction uRec and deltaLambdaCell are held fixed.  A^-1 is
// differentiated as d(A^-1) = -A^-1 dA A^-1 (A is symmetric positive definite, where the
// reference's pseudo-inverse is the inverse).  Inviscid 5-variable models.
#pragma once
#include "solver.cuh"
#include "basis_eval.cuh"
#include "bc.cuh"
#include "dual.cuh"

namespace dndsb
{
constexpr int kGeoMaxVert = 8;
constexpr int kGeoBlock = 64;

namespace
{
// VJP seed: the three coordinates of one node
struct SeedNode
{
    int32_t node;
    DNDSB_D void load(const real *X, int32_t nd, const real *sh, Dual<3> *out) const
    {
        for (int d = 0; d < 3; d++)
        {
            out[d] = Dual<3>(X[(int64_t)nd * 3 + d] + sh[d]);
            if (nd == node)
                out[d].d[d] = 1;
        }
    }
};

// JVP seed: one direction of all node coordinates
struct SeedDir
{
    const real *dX;
    DNDSB_D void load(const real *X, int32_t nd, const real *sh, Dual<1> *out) const
    {
        for (int d = 0; d < 3; d++)
        {
            out[d] = Dual<1>(X[(int64_t)nd * 3 + d] + sh[d]);
            out[d].d[0] = dX[(int64_t)nd * 3 + d];
        }
    }
};

template <typename T, int NDOF>
struct CellG
{
    T vol, bary[3], cent[3], scale[3], moment[NDOF];
    static constexpr int kFields = 10 + NDOF;
    DNDSB_D T *fields() { return &vol; }
};

// Cell geometry from the per-mesh cache: [field][lane], lane 0 the value, lane 1 + 3 v + d its derivative
// with respect to coordinate d of the cell's vertex v (the first vertex of a node carries all of it)
template <int NDOF>
DNDSB_D void lanes_load(const real *cg, const MeshD &m, int64_t c, const SeedNode &sd, CellG<Dual<3>, NDOF> &o)
{
    const int L = 1 + 3 * m.nvert;
    Dual<3> *f = o.fields();
    for (int i = 0; i < CellG<Dual<3>, NDOF>::kFields; i++)
        f[i] = Dual<3>(cg[i * L]);
    for (int v = 0; v < m.nvert; v++)
        if (m.cell2node[c * m.nvert + v] == sd.node)
            for (int i = 0; i < CellG<Dual<3>, NDOF>::kFields; i++)
                for (int d = 0; d < 3; d++)
                    f[i].d[d] += cg[i * L + 1 + 3 * v + d];
}

template <int NDOF>
DNDSB_D void lanes_load(const real *cg, const MeshD &m, int64_t c, const SeedDir &sd, CellG<Dual<1>, NDOF> &o)
{
    const int L = 1 + 3 * m.nvert;
    Dual<1> *f = o.fields();
    real dx[3 * kGeoMaxVert];
    for (int v = 0; v < m.nvert; v++)
        for (int d = 0; d < 3; d++)
            dx[v * 3 + d] = sd.dX[(int64_t)m.cell2node[c * m.nvert + v] * 3 + d];
    for (int i = 0; i < CellG<Dual<1>, NDOF>::kFields; i++)
    {
        real a = 0;
        for (int l = 0; l < 3 * m.nvert; l++)
            a += cg[i * L + 1 + l] * dx[l];
        f[i] = Dual<1>(cg[i * L]);
        f[i].d[0] = a;
    }
}

// geometry of cell c: from the cache when there is one, else recomputed
template <int DIM, int NDOF, typename T, typename Seed>
DNDSB_D void cell_geo_or_lanes(const real *lanes, const MeshD &m, int intOrder, int nGc, bool aniso, int64_t c, const Seed &sd,
                               CellG<T, NDOF> &o);

template <typename T>
struct FaceG
{
    T cs[12];
    T area, cent[3], meanNorm[3];
};

// cell metrics (FiniteVolume.cpp:22-330: volume by the order-6 rule, barycentre by the intOrder
// rule, centre, axis-aligned half box) and the basis moments (VariationalReconstruction.cpp
// :80-108), as k_cell_metrics and k_base_moment compute them
template <int DIM, int NDOF, typename T, typename Seed>
DNDSB_D void cell_geo(const MeshD &m, int intOrder, int nGc, bool aniso, int64_t c, const Seed &sd, CellG<T, NDOF> &o)
{
    T cs[3 * kGeoMaxVert];
    for (int v = 0; v < m.nvert; v++)
        sd.load(m.coords, m.cell2node[c * m.nvert + v], &m.cellShift[(c * m.nvert + v) * 3], &cs[v * 3]);
    PtGeoT<T> pg;
    real p[3], w;
    const int nMax = quad_n(m.cellType, kIntOrderMax);
    T v = 0.0;
    for (int q = 0; q < nMax; q++)
    {
        quad_point(m.cellType, kIntOrderMax, q, p, w);
        pt_geo(m.cellType, cs, p, pg);
        v += cell_jdet(m.dim, pg) * w;
    }
    v = v + kVerySmall;
    o.vol = v;
    T b[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < nGc; q++)
    {
        quad_point(m.cellType, intOrder, q, p, w);
        pt_geo(m.cellType, cs, p, pg);
        T J = cell_jdet(m.dim, pg);
        for (int d = 0; d < 3; d++)
            b[d] += pg.x[d] * J * w;
    }
    for (int d = 0; d < 3; d++)
        o.bary[d] = b[d] / v;
    quad_point(m.cellType, 1, 0, p, w);
    pt_geo(m.cellType, cs, p, pg);
    for (int d = 0; d < 3; d++)
        o.cent[d] = pg.x[d];
    for (int d = 0; d < 3; d++)
    {
        T h = 0.0;
        for (int k = 0; k < m.nvert; k++)
            h = dmax(h, T(fabs(cs[k * 3 + d] - o.bary[d])));
        o.scale[d] = h;
    }
    if (m.dim == 2)
        o.scale[2] = 1.0;
    T acc[NDOF], Tb[NDOF];
    for (int k = 0; k < NDOF; k++)
        acc[k] = 0.0;
    for (int q = 0; q < nMax; q++)
    {
        quad_point(m.cellType, kIntOrderMax, q, p, w);
        pt_geo(m.cellType, cs, p, pg);
        T J = cell_jdet(DIM, pg);
        cell_basis<DIM, NDOF>(o.cent, o.scale, nullptr, aniso, pg.x, 1, Tb);
        for (int k = 0; k < NDOF; k++)
            acc[k] += Tb[k] * J * w;
    }
    for (int k = 0; k < NDOF; k++)
        o.moment[k] = acc[k] / acc[0];
}

template <int DIM, int NDOF, typename T, typename Seed>
DNDSB_D void cell_geo_or_lanes(const real *lanes, const MeshD &m, int intOrder, int nGc, bool aniso, int64_t c, const Seed &sd,
                               CellG<T, NDOF> &o)
{
    if (lanes)
        lanes_load<NDOF>(lanes + c * (int64_t)CellG<T, NDOF>::kFields * (1 + 3 * m.nvert), m, c, sd, o);
    else
        cell_geo<DIM, NDOF>(m, intOrder, nGc, aniso, c, sd, o);
}

// face area, mean normal and centre (FiniteVolume.cpp:352-543, as k_face_metrics)
template <typename T, typename Seed>
DNDSB_D void face_geo(const MeshD &m, int intOrder, int nGf, int64_t f, const Seed &sd, FaceG<T> &o)
{
    for (int v = 0; v < m.nfv; v++)
        sd.load(m.coords, m.face2node[f * m.nfv + v], &m.faceShift[(f * m.nfv + v) * 3], &o.cs[v * 3]);
    PtGeoT<T> pg;
    real p[3], w;
    T a = 0.0, nm[3] = {0.0, 0.0, 0.0}, n[3];
    for (int q = 0; q < nGf; q++)
    {
        quad_point(m.faceType, intOrder, q, p, w);
        pt_geo(m.faceType, o.cs, p, pg);
        T J = face_jdet_normal(m.dim, pg, n);
        T nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        a += J * w;
        for (int d = 0; d < 3; d++)
            nm[d] += n[d] / nn * J * w;
    }
    o.area = a + kVerySmall;
    T nn = sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]);
    for (int d = 0; d < 3; d++)
        o.meanNorm[d] = nm[d] / nn;
    quad_point(m.faceType, 1, 0, p, w);
    pt_geo(m.faceType, o.cs, p, pg);
    for (int d = 0; d < 3; d++)
        o.cent[d] = pg.x[d];
}

// point q of the face rule: coordinates, unit normal and |J| times the weight
template <typename T>
DNDSB_D void face_point(const MeshD &m, int intOrder, const FaceG<T> &fg, int q, real qw, T pp[3], T nrm[3], T &JW)
{
    PtGeoT<T> pg;
    real p[3], w;
    quad_point(m.faceType, intOrder, q, p, w);
    pt_geo(m.faceType, fg.cs, p, pg);
    T n[3];
    T J = face_jdet_normal(m.dim, pg, n);
    T nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int d = 0; d < 3; d++)
        pp[d] = pg.x[d], nrm[d] = n[d] / nn;
    JW = (J + kVerySmall) * qw;
}

// VariationalReconstruction.cpp:200-441 as k_face_weight: the functional length and the geometric
// weight factor of the face.  The stored weights hold the constant direction and boundary factors
// times the geometric factor, so the weights in T are the stored ones scaled by wg / value(wg).
template <int DIM, int P, typename T>
DNDSB_D void face_weights(const MeshD &m, const VRD &vr, int64_t f, const FaceG<T> &fg, const T *bary0, const T *bary1, const T *scale0,
                          const T *scale1, T w2L[P + 1], T &w0)
{
    const VRSettingsD &s = vr.s;
    T dv[3];
    if (bary1)
        for (int d = 0; d < 3; d++)
            dv[d] = bary1[d] - m.facePShift[f * 3 + d] - bary0[d];
    else
    {
        T vCB[3];
        for (int d = 0; d < 3; d++)
            vCB[d] = fg.cent[d] - bary0[d];
        T vn = vCB[0] * fg.meanNorm[0] + vCB[1] * fg.meanNorm[1] + vCB[2] * fg.meanNorm[2];
        for (int d = 0; d < 3; d++)
            dv[d] = 2 * vn * fg.meanNorm[d];
    }
    T L;
    if (s.scaleType == 1)
    {
        T q = 0.0;
        for (int d = 0; d < DIM; d++)
            q += dv[d] * dv[d];
        L = sqrt(q);
    }
    else
    {
        T hb[3] = {0.0, 0.0, 0.0};
        int n = 1;
        for (int d = 0; d < 3; d++)
            hb[d] += scale0[d];
        if (scale1)
        {
            for (int d = 0; d < 3; d++)
                hb[d] += scale1[d];
            n++;
        }
        T q = 0.0;
        for (int d = 0; d < DIM; d++)
            q += (hb[d] / n) * (hb[d] / n);
        L = sqrt(q / DIM);
    }
    L = L * s.scaleMultiplier;
    T dn = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    T wg = 1.0;
    if (s.geomWeightScheme == 1)
        wg = s.geomWeightBias + pow(pow(fg.area, 1. / real(DIM - 1)) / dn, s.geomWeightPower * 0.5);
    else if (s.geomWeightScheme == 2)
        wg = s.geomWeightBias + pow(fg.area, s.geomWeightPower1 * 0.5) * pow(dn, s.geomWeightPower2 * 0.5);
    const real wv = value_of(wg);
    T scl = 1.0;
    if (wv != 0)
        scl = wg / wv;
    T L2 = L * L, Lp = 1.0;
    for (int o = 0; o <= P; o++)
    {
        T w = scl * vr.faceWeight[f * (P + 1) + o];
        w2L[o] = value_of(L) == 0 ? T(w * w) : T(w * w * Lp);
        Lp = Lp * L2;
    }
    w0 = scl * vr.faceWeight[f * (P + 1)];
}

// A^-1 in dual numbers: the value by Gauss-Jordan, the derivatives by d(A^-1) = -A^-1 dA A^-1
template <int R, int N>
DNDSB_D bool invert_t(const Dual<N> *A, Dual<N> *Ai)
{
    real a[R * R], ai[R * R], t[R * R];
    for (int i = 0; i < R * R; i++)
        a[i] = A[i].v;
    if (!invert_gj<R>(a, ai))
        return false;
    for (int i = 0; i < R * R; i++)
        Ai[i] = Dual<N>(ai[i]);
#pragma unroll 1
    for (int k = 0; k < N; k++)
    {
#pragma unroll 1
        for (int i = 0; i < R; i++)
            for (int j = 0; j < R; j++)
            {
                real s = 0;
                for (int l = 0; l < R; l++)
                    s += A[i * R + l].d[k] * ai[l * R + j];
                t[i * R + j] = s;
            }
#pragma unroll 1
        for (int i = 0; i < R; i++)
            for (int j = 0; j < R; j++)
            {
                real s = 0;
                for (int l = 0; l < R; l++)
                    s += ai[i * R + l] * t[l * R + j];
                Ai[i * R + j].d[k] = -s;
            }
    }
    return true;
}

// The residual entries of cell c in the scalar type T:
//   rhs = EvaluateRHS(u, uRec)_c (k_rhs_face / k_rhs_bc, inviscid; gathered as k_rhs_gather),
//   S   = sum_k (A^-1 B_k uRec_k + A^-1 b_k (u_k - u_c)) + A^-1 BCC (k_vr_coeff, k_vr_jacobi, k_vr_bc),
// with B_k uRec_k and b_k (u_k - u_c) accumulated point by point instead of stored.
template <int DIM, int P, typename T, typename Seed>
DNDSB_D void cell_local(const MeshD &m, const GeomD &g, const VRD &vr, const EulerSettingsD &s, const real *dLamCell, const real *u,
                        const real *uRec, int64_t c, const Seed &sd, bool wantRhs, bool wantRec, T *rhs, T *S, int &bad,
                        const real *lanes)
{
    constexpr int NV = 5, NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    const int intOrder = vr.s.intOrder;
    const bool aniso = vr.s.anisotropicLengths;
    CellG<T, NDOF> gc, go;
    cell_geo_or_lanes<DIM, NDOF>(lanes, m, intOrder, g.nGc, aniso, c, sd, gc);
    T A[R * R], Sacc[R * NV], flux[NV];
    for (int i = 0; i < R * R; i++)
        A[i] = 0.0;
    for (int i = 0; i < R * NV; i++)
        Sacc[i] = 0.0;
    for (int v = 0; v < NV; v++)
        flux[v] = 0.0;
    const real *uc = u + c * NV, *rc = uRec + c * R * NV;
    T ucT[NV];
    for (int v = 0; v < NV; v++)
        ucT[v] = uc[v];
    for (int k = 0; k < m.nf; k++)
    {
        const int fp = m.cell2face[c * m.nf + k];
        const int64_t f = fp >> 1;
        const int side = fp & 1;
        const int o = m.cellNbr[c * m.nf + k];
        FaceG<T> fg;
        face_geo(m, intOrder, g.nGf, f, sd, fg);
        if (o >= 0)
            cell_geo_or_lanes<DIM, NDOF>(lanes, m, intOrder, g.nGc, aniso, o, sd, go);
        const CellG<T, NDOF> &g0 = side ? go : gc, &g1 = side ? gc : go;
        T w2L[P + 1], w0;
        face_weights<DIM, P>(m, vr, f, fg, g0.bary, o >= 0 ? g1.bary : nullptr, g0.scale, o >= 0 ? g1.scale : nullptr, w2L, w0);
        const real *ro = o >= 0 ? uRec + (int64_t)o * R * NV : nullptr;
        real du[NV];
        for (int v = 0; v < NV; v++)
            du[v] = o >= 0 ? u[(int64_t)o * NV + v] - uc[v] : 0.0;
        // boundary faces: ghost of the cell mean at the mean normal (Roe means of EvaluateRHS.hxx:198-210)
        const int zone = m.faceZone[f];
        T ULmB[NV], URmB[NV];
        if (o < 0 && wantRhs)
        {
            for (int v = 0; v < NV; v++)
                ULmB[v] = uc[v];
            if (!bc_value<NV>(vr.bnd, zone, ULmB, fg.meanNorm, URmB))
                for (int v = 0; v < NV; v++)
                    URmB[v] = ULmB[v];
        }
        T fluxF[NV];
        for (int v = 0; v < NV; v++)
            fluxF[v] = 0.0;
        for (int q = 0; q < g.nGf; q++)
        {
            T pp[3], nrm[3], JW;
            face_point(m, intOrder, fg, q, g.faceQw[q], pp, nrm, JW);
            T pc[3], po[3];
            for (int d = 0; d < 3; d++)
            {
                const real sh = m.facePShift[f * 3 + d];
                pc[d] = pp[d] + (side ? sh : 0.0);
                po[d] = pp[d] + (side ? 0.0 : sh);
            }
            T TI[NDOF * NDOF];
            cell_basis<DIM, NDOF>(gc.cent, gc.scale, gc.moment, aniso, pc, wantRec ? NDOF : 1, TI);
            if (wantRec)
            {
                // VR functional (VariationalReconstruction.hpp:460-590): A += <D phi_i, D phi_j>
#pragma unroll 1
                for (int ob = P; ob >= 0; ob--)
                {
                    const T sc = w2L[ob] * JW;
                    for (int kk = Basis<DIM>::order_start(ob); kk < Basis<DIM>::order_start(ob + 1); kk++)
                    {
                        const T ck = Basis<DIM>::ncomb(kk) * sc;
                        for (int i = 0; i < R; i++)
                        {
                            const T a = TI[kk * NDOF + 1 + i] * ck;
                            for (int j = 0; j < R; j++)
                                A[i * R + j] += a * TI[kk * NDOF + 1 + j];
                        }
                    }
                }
                if (o >= 0)
                {
                    T TJ[NDOF * NDOF];
                    cell_basis<DIM, NDOF>(go.cent, go.scale, go.moment, aniso, po, NDOF, TJ);
#pragma unroll 1
                    for (int ob = P; ob >= 0; ob--)
                    {
                        const T sc = w2L[ob] * JW;
                        for (int kk = Basis<DIM>::order_start(ob); kk < Basis<DIM>::order_start(ob + 1); kk++)
                        {
                            const T ck = Basis<DIM>::ncomb(kk) * sc;
                            T gk[NV];
                            for (int v = 0; v < NV; v++)
                            {
                                gk[v] = 0.0;
                                for (int j = 0; j < R; j++)
                                    gk[v] += TJ[kk * NDOF + 1 + j] * ro[j * NV + v];
                            }
                            for (int i = 0; i < R; i++)
                            {
                                const T a = TI[kk * NDOF + 1 + i] * ck;
                                for (int v = 0; v < NV; v++)
                                    Sacc[i * NV + v] += a * gk[v];
                            }
                        }
                    }
                    // b_k (u_k - u_c): the order-0 functional against the constant 1
                    const T sc0 = w2L[0] * JW;
                    for (int i = 0; i < R; i++)
                    {
                        const T a = TI[1 + i] * sc0;
                        for (int v = 0; v < NV; v++)
                            Sacc[i * NV + v] += a * du[v];
                    }
                }
                else if (value_of(w0) != 0)
                {
                    // GetBoundaryRHS (_Reconstruction.hxx:19-176) as k_vr_bc
                    T UL[NV], ULf[NV], UB[NV];
                    for (int v = 0; v < NV; v++)
                    {
                        T a = uc[v];
                        for (int j = 0; j < R; j++)
                            a += TI[1 + j] * rc[j * NV + v];
                        UL[v] = a;
                    }
                    compress_rec<NV>(ucT, UL, ULf);
                    if (!bc_value_fix<NV>(vr.bnd, zone, ULf, nrm, UB))
                        for (int v = 0; v < NV; v++)
                            UB[v] = ULf[v];
                    const T JWb = JW * w0 * w0;
                    for (int i = 0; i < R; i++)
                        for (int v = 0; v < NV; v++)
                            Sacc[i * NV + v] += TI[1 + i] * (UB[v] - uc[v]) * JWb;
                }
            }
            if (wantRhs)
            {
                T F[NV], l0, l1, l4;
                if (o >= 0)
                {
                    // interior face (k_rhs_face): left is face2cell side 0
                    const int64_t c0 = side ? o : c, c1 = side ? c : o;
                    T TO[NDOF];
                    cell_basis<DIM, NDOF>(go.cent, go.scale, go.moment, aniso, po, 1, TO);
                    const T *T0 = side ? TO : TI, *T1 = side ? TI : TO;
                    const real *r0 = uRec + c0 * R * NV, *r1 = uRec + c1 * R * NV;
                    T UL[NV], UR[NV], ULm[NV], URm[NV];
                    for (int v = 0; v < NV; v++)
                    {
                        T a = u[c0 * NV + v], b = u[c1 * NV + v];
                        ULm[v] = a, URm[v] = b;
                        for (int j = 0; j < R; j++)
                        {
                            a += T0[1 + j] * r0[j * NV + v];
                            b += T1[1 + j] * r1[j * NV + v];
                        }
                        UL[v] = a, UR[v] = b;
                    }
                    const real dLambda = dmax(dLamCell[c0], dLamCell[c1]);
                    bad |= !riemann_flux(s.rsType, UL, UR, ULm, URm, nrm, s.gamma, dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4);
                }
                else
                {
                    // boundary face (k_rhs_bc, inviscid)
                    T UL[NV], UR[NV];
                    for (int v = 0; v < NV; v++)
                    {
                        T a = uc[v];
                        for (int j = 0; j < R; j++)
                            a += TI[1 + j] * rc[j * NV + v];
                        UL[v] = a;
                    }
                    if (!bc_value_fix<NV>(vr.bnd, zone, UL, nrm, UR))
                        for (int v = 0; v < NV; v++)
                            UR[v] = UL[v];
                    for (int v = 0; v < NV; v++)
                        F[v] = 0.0;
                    bad |= !riemann_flux(s.rsType, UL, UR, ULmB, URmB, nrm, s.gamma, dLamCell[c], s.rsFixScale, s.rsIncFScale, F, l0, l1, l4);
                }
                for (int v = 0; v < NV; v++)
                    fluxF[v] -= F[v] * JW;
            }
        }
        if (wantRhs)
        {
            const real sg = side ? -1.0 : 1.0;
            for (int v = 0; v < NV; v++)
                flux[v] += sg * fluxF[v];
        }
    }
    if (wantRhs)
    {
        T iv = 1.0 / gc.vol;
        for (int v = 0; v < NV; v++)
            rhs[v] = flux[v] * iv;
    }
    if (wantRec)
    {
        T Ai[R * R];
        if (!invert_t<R>(A, Ai))
        {
            bad = 1;
            return;
        }
#pragma unroll 1
        for (int i = 0; i < R; i++)
            for (int v = 0; v < NV; v++)
            {
                T acc = 0.0;
                for (int j = 0; j < R; j++)
                    acc += Ai[i * R + j] * Sacc[j * NV + v];
                S[i * NV + v] = acc;
            }
    }
}

// VJP share of one (cell, patch node): the derivatives of cell c's residual entries with respect to
// the node's coordinates, contracted with the cotangents w (EvaluateRHS) and relax * cot (sweep)
template <int DIM, int P>
DNDSB_GLOBAL void __launch_bounds__(kGeoBlock) k_coords_vjp(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ dLamCell,
                                                            const real *__restrict__ u, const real *__restrict__ uRec, const real *__restrict__ w,
                                                            const real *__restrict__ cot, real relax, const int32_t *__restrict__ patch,
                                                            int maxSlot, real *__restrict__ share, int *err, const real *__restrict__ lanes)
{
    constexpr int NV = 5, NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(e, m.nCell * maxSlot)
    {
        const int64_t c = e / maxSlot;
        const int32_t node = patch[e];
        real out[3] = {0, 0, 0};
        if (node >= 0)
        {
            SeedNode sd{node};
            Dual<3> rhs[NV], S[R * NV];
            int bad = 0;
            cell_local<DIM, P>(m, g, vr, s, dLamCell, u, uRec, c, sd, w != nullptr, cot != nullptr, rhs, S, bad, lanes);
            Dual<3> acc = 0.0;
            if (w)
                for (int v = 0; v < NV; v++)
                    acc += rhs[v] * w[c * NV + v];
            if (cot)
                for (int i = 0; i < R * NV; i++)
                    acc += S[i] * (relax * cot[c * R * NV + i]);
            for (int d = 0; d < 3; d++)
                out[d] = acc.d[d];
            if (bad)
                atomicOr(err, (int)DE_NONPHYSICAL);
        }
        for (int d = 0; d < 3; d++)
            share[e * 3 + d] = out[d];
    }
}

// JVP: directional derivatives of cell c's residual entries along the node displacement dX
template <int DIM, int P>
DNDSB_GLOBAL void __launch_bounds__(kGeoBlock) k_coords_jvp(MeshD m, GeomD g, VRD vr, EulerSettingsD s, const real *__restrict__ dLamCell,
                                                            const real *__restrict__ u, const real *__restrict__ uRec, const real *__restrict__ dX,
                                                            real relax, real *__restrict__ dRhs, real *__restrict__ dRec, int *err,
                                                            const real *__restrict__ lanes)
{
    constexpr int NV = 5, NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(c, m.nCell)
    {
        SeedDir sd{dX};
        Dual<1> rhs[NV], S[R * NV];
        int bad = 0;
        cell_local<DIM, P>(m, g, vr, s, dLamCell, u, uRec, c, sd, dRhs != nullptr, dRec != nullptr, rhs, S, bad, lanes);
        if (dRhs)
            for (int v = 0; v < NV; v++)
                dRhs[c * NV + v] = rhs[v].d[0];
        if (dRec)
            for (int i = 0; i < R * NV; i++)
                dRec[c * R * NV + i] = relax * S[i].d[0];
        if (bad)
            atomicOr(err, (int)DE_NONPHYSICAL);
    }
}
// the per-mesh cache of cell geometry lanes: one thread per (cell, vertex), that vertex's node seeded
template <int DIM, int P>
DNDSB_GLOBAL void __launch_bounds__(kGeoBlock) k_cell_lanes(MeshD m, GeomD g, VRD vr, real *__restrict__ lanes)
{
    constexpr int NDOF = ndof_of<DIM>(P), NF = CellG<real, NDOF>::kFields;
    const int L = 1 + 3 * m.nvert;
    DNDSB_KERNEL_LOOP(e, m.nCell * m.nvert)
    {
        const int64_t c = e / m.nvert;
        const int v = (int)(e - c * m.nvert);
        const int32_t node = m.cell2node[c * m.nvert + v];
        bool dup = false;
        for (int v2 = 0; v2 < v; v2++)
            dup = dup || m.cell2node[c * m.nvert + v2] == node;
        CellG<Dual<3>, NDOF> o;
        cell_geo<DIM, NDOF>(m, vr.s.intOrder, g.nGc, vr.s.anisotropicLengths, c, SeedNode{node}, o);
        real *cg = lanes + c * (int64_t)NF * L;
        const Dual<3> *f = o.fields();
        for (int i = 0; i < NF; i++)
        {
            if (v == 0)
                cg[i * L] = f[i].v;
            for (int d = 0; d < 3; d++)
                cg[i * L + 1 + 3 * v + d] = dup ? 0.0 : f[i].d[d];
        }
    }
}

// Share of one (boundary cell, cell vertex) in the derivative of the pressure force
// J = sum over the zone's faces and points of p(U) (n . dir) |J| w (k_pressure_force) with respect to
// the vertex coordinates: the cell's basis and its faces' geometry depend on its own nodes only.
// Written into the patch slot of that node in the cell's own patch (a node met twice in a cell, as
// periodic images, is seeded once).
template <int DIM, int P>
DNDSB_GLOBAL void __launch_bounds__(kGeoBlock) k_pressure_force_coords(MeshD m, GeomD g, VRD vr, real gamma, int zone, real d0, real d1, real d2,
                                                                       const real *__restrict__ u, const real *__restrict__ uRec,
                                                                       const int32_t *__restrict__ patch, int maxSlot, real *__restrict__ share)
{
    constexpr int NV = 5, NDOF = ndof_of<DIM>(P), R = NDOF - 1;
    DNDSB_KERNEL_LOOP(e, m.nBndCell * m.nvert)
    {
        const int64_t ii = e / m.nvert;
        const int v = (int)(e - ii * m.nvert);
        const int64_t c = m.bndCell[ii];
        const int32_t node = m.cell2node[c * m.nvert + v];
        bool dup = false;
        for (int v2 = 0; v2 < v; v2++)
            dup = dup || m.cell2node[c * m.nvert + v2] == node;
        int slot = 0;
        while (slot < maxSlot && patch[c * maxSlot + slot] != node)
            slot++;
        if (dup || slot == maxSlot)
            continue;
        SeedNode sd{node};
        const bool aniso = vr.s.anisotropicLengths;
        CellG<Dual<3>, NDOF> gc;
        bool any = false;
        Dual<3> J = 0.0;
        for (int k = 0; k < m.nf; k++)
        {
            if (m.cellNbr[c * m.nf + k] >= 0)
                continue;
            const int64_t f = m.cell2face[c * m.nf + k] >> 1;
            if (m.faceZone[f] != zone)
                continue;
            if (!any)
                cell_geo<DIM, NDOF>(m, vr.s.intOrder, g.nGc, aniso, c, sd, gc);
            any = true;
            FaceG<Dual<3>> fg;
            face_geo(m, vr.s.intOrder, g.nGf, f, sd, fg);
            for (int q = 0; q < g.nGf; q++)
            {
                Dual<3> pp[3], nrm[3], JW, T0[NDOF];
                face_point(m, vr.s.intOrder, fg, q, g.faceQw[q], pp, nrm, JW);
                cell_basis<DIM, NDOF>(gc.cent, gc.scale, gc.moment, aniso, pp, 1, T0);
                Dual<3> UL[NV];
                for (int w = 0; w < NV; w++)
                {
                    Dual<3> a = 0.0;
                    for (int j = 0; j < R; j++)
                        a += T0[1 + j] * uRec[(c * R + j) * NV + w];
                    UL[w] = u[c * NV + w] + a;
                }
                Dual<3> vel[3] = {UL[1] / UL[0], UL[2] / UL[0], UL[3] / UL[0]};
                Dual<3> pr = (gamma - 1) * (UL[4] - 0.5 * UL[0] * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]));
                Dual<3> wt = JW * (nrm[0] * d0 + nrm[1] * d1 + nrm[2] * d2);
                J += wt * pr;
            }
        }
        for (int d = 0; d < 3; d++)
            share[(c * maxSlot + slot) * 3 + d] = J.d[d];
    }
}
} // namespace

template <int DIM>
void pressure_force_coords_launch(const MeshD &m, const GeomD &g, const VRD &vr, real gamma, int zone, const real *dir, const real *u,
                                  const real *uRec, const CoordAdjWs &ws, cudaStream_t st)
{
    constexpr int PTop = DIM == 2 ? 3 : 2;
    const int64_t n = m.nBndCell * m.nvert;
    if (vr.P == 1)
        DNDSB_LAUNCH((k_pressure_force_coords<DIM, 1>), n, kGeoBlock, st, m, g, vr, gamma, zone, dir[0], dir[1], dir[2], u, uRec, ws.patch, ws.maxSlot, ws.share);
    else if (vr.P == 2)
        DNDSB_LAUNCH((k_pressure_force_coords<DIM, 2>), n, kGeoBlock, st, m, g, vr, gamma, zone, dir[0], dir[1], dir[2], u, uRec, ws.patch, ws.maxSlot, ws.share);
    else
        DNDSB_LAUNCH((k_pressure_force_coords<DIM, PTop>), n, kGeoBlock, st, m, g, vr, gamma, zone, dir[0], dir[1], dir[2], u, uRec, ws.patch,
                     ws.maxSlot, ws.share);
}

// launches for one dimension; P = 1, 2 (and 3 in 2-D)
template <int DIM>
void coords_vjp_launch(const MeshD &m, const GeomD &g, const VRD &vr, const EulerSettingsD &es, const real *dLamCell, const real *u,
                       const real *uRec, const real *w, const real *cot, const CoordAdjWs &ws, int *err, cudaStream_t st)
{
    constexpr int PTop = DIM == 2 ? 3 : 2;
    const int64_t n = m.nCell * ws.maxSlot;
    const real relax = vr.s.jacobiRelax;
    if (vr.P == 1)
        DNDSB_LAUNCH((k_coords_vjp<DIM, 1>), n, kGeoBlock, st, m, g, vr, es, dLamCell, u, uRec, w, cot, relax, ws.patch, ws.maxSlot, ws.share, err,
                     ws.lanes);
    else if (vr.P == 2)
        DNDSB_LAUNCH((k_coords_vjp<DIM, 2>), n, kGeoBlock, st, m, g, vr, es, dLamCell, u, uRec, w, cot, relax, ws.patch, ws.maxSlot, ws.share, err,
                     ws.lanes);
    else
        DNDSB_LAUNCH((k_coords_vjp<DIM, PTop>), n, kGeoBlock, st, m, g, vr, es, dLamCell, u, uRec, w, cot, relax, ws.patch, ws.maxSlot, ws.share,
                     err, ws.lanes);
}

template <int DIM>
void coords_jvp_launch(const MeshD &m, const GeomD &g, const VRD &vr, const EulerSettingsD &es, const real *dLamCell, const real *dX, const real *u,
                       const real *uRec, real *dRhs, real *dRec, int *err, const real *lanes, cudaStream_t st)
{
    constexpr int PTop = DIM == 2 ? 3 : 2;
    const real relax = vr.s.jacobiRelax;
    if (vr.P == 1)
        DNDSB_LAUNCH((k_coords_jvp<DIM, 1>), m.nCell, kGeoBlock, st, m, g, vr, es, dLamCell, u, uRec, dX, relax, dRhs, dRec, err, lanes);
    else if (vr.P == 2)
        DNDSB_LAUNCH((k_coords_jvp<DIM, 2>), m.nCell, kGeoBlock, st, m, g, vr, es, dLamCell, u, uRec, dX, relax, dRhs, dRec, err, lanes);
    else
        DNDSB_LAUNCH((k_coords_jvp<DIM, PTop>), m.nCell, kGeoBlock, st, m, g, vr, es, dLamCell, u, uRec, dX, relax, dRhs, dRec, err, lanes);
}

template <int DIM>
void coords_lanes_launch(const MeshD &m, const GeomD &g, const VRD &vr, real *lanes, cudaStream_t st)
{
    constexpr int PTop = DIM == 2 ? 3 : 2;
    const int64_t n = m.nCell * m.nvert;
    if (vr.P == 1)
        DNDSB_LAUNCH((k_cell_lanes<DIM, 1>), n, kGeoBlock, st, m, g, vr, lanes);
    else if (vr.P == 2)
        DNDSB_LAUNCH((k_cell_lanes<DIM, 2>), n, kGeoBlock, st, m, g, vr, lanes);
    else
        DNDSB_LAUNCH((k_cell_lanes<DIM, PTop>), n, kGeoBlock, st, m, g, vr, lanes);
}
} // namespace dndsb
