// Gauss-point-parallel VJP of the interior faces: plain Roe or HLLE+ and the compact viscous flux for 5
// variables, plain Roe with the SA model for 6 (the derivative counterpart of k_rhs_face_fast in fast.cu);
// instantiated by adjoint_fast.cu (5 variables) and adjoint_fast_sa.cu (6).
//
// The layout of k_rhs_face_fast: one thread per (face, Gauss point), 32 faces per block (the points of a
// face in different warps), the 64 adjacent cells staged in shared memory and the per-face data (Roe
// averages, GRP distance, dLambda, the cotangent jump w0/V0 - w1/V1) formed once per face.  Each thread
// reverses the face integrand at its point, -(F(U_L, U_R; r) - Fv(U_M, grad U_M)) |J| w with the compact
// gradient (EvaluateRHS.hxx:369-525): the cotangents of the two point states (Ub0, Ub1), of grad U_M (GMb)
// and of the Roe-average fields (hand-written reverse sweeps of roe_rev.cuh and visc_rev.cuh).  Their
// images in the cotangent rows of both cells' (u, uRec),
//     row_j,v = sum_q [phi_j(p_q) Ub_q,v + sum_d dphi_j/dx_d(p_q) GMb_q,d,v],
// are summed over the points in point order through shared memory, all rows in one round (or half of them
// per round where the shares would not fit).  The Roe-average cotangents are summed the same way and
// carried to the two cell means by a
// Dual<1> evaluation of the averages per mean component (one thread each).  The block's face records
// [32][2][(R+1) NV] are assembled in shared memory and stored row-contiguously.
#pragma once
#include "solver.cuh"
#include "fast_common.cuh"
#include "roe_rev.cuh"
#include "visc_rev.cuh"

namespace dndsb
{
namespace
{
using namespace fastc;
using D1 = Dual<1>;

// resident blocks per SM the register budget is sized for (two blocks of 9 warps at 9 points per face)
template <int NG>
constexpr int vjp_min_blocks() { return (9 / NG) > 0 ? (9 / NG) : 1; }

// x^e for a compile-time exponent
template <int E>
DNDSB_D real pw(real x)
{
    if constexpr (E == 0)
        return 1.0;
    else
        return x * pw<E - 1>(x);
}

// row j of a staged cell at the normalised point (x, y, z): phi_j and its gradient (VariationalReconstruction.hpp:378-442)
template <int DIM, int J>
DNDSB_D void basis_row(real x, real y, real z, const real *iL, real mom, real &phi, real &dx, real &dy, real &dz)
{
    constexpr int c = mcode(DIM, J), ex = c & 3, ey = (c >> 2) & 3, ez = (c >> 4) & 3;
    phi = pw<ex>(x) * pw<ey>(y) * pw<ez>(z) - mom;
    if constexpr (ex > 0)
        dx = ex * pw<(ex > 0 ? ex - 1 : 0)>(x) * pw<ey>(y) * pw<ez>(z) * iL[0];
    else
        dx = 0;
    if constexpr (ey > 0)
        dy = ey * pw<ex>(x) * pw<(ey > 0 ? ey - 1 : 0)>(y) * pw<ez>(z) * iL[1];
    else
        dy = 0;
    if constexpr (ez > 0)
        dz = ez * pw<ex>(x) * pw<ey>(y) * pw<(ez > 0 ? ez - 1 : 0)>(z) * iL[2];
    else
        dz = 0;
}

template <int DIM, int P, int NV, int NG, bool VISC>
struct VjpRows
{
    using Lt = Layout<DIM, P, NV>;
    static constexpr int R = Lt::R, W = (R + 1) * NV;
    // reconstruction rows per round: all of them when the 32 faces' shares fit in 120 KB of shared memory,
    // else half of them
    static constexpr int ROWS = NG * 32 * (R + 1) * 2 * NV * 8 <= 120 * 1024 ? R + 1 : (R + 2) / 2;
    static constexpr int CH = ROWS * 2 * NV > 15 ? ROWS * 2 * NV : 15; // values per point of one round

    // the point shares of row J (both sides) into slot J - J0 of the round's buffer
    template <int J, int J0>
    static DNDSB_D void shares(const real *xs, const real *cell0, const real *cell1, const real *Ub0, const real *Ub1, const real *GMb, real *sRed,
                               int q, int fl)
    {
        if constexpr (J <= R && J < J0 + ROWS)
        {
#pragma unroll
            for (int side = 0; side < 2; side++)
            {
                const real *Ub = side ? Ub1 : Ub0;
                real phi = 1, dx = 0, dy = 0, dz = 0;
                if constexpr (J > 0)
                {
                    const real *cell = side ? cell1 : cell0;
                    basis_row<DIM, J>(xs[side * 3], xs[side * 3 + 1], xs[side * 3 + 2], cell + Lt::OL, cell[Lt::OM + J], phi, dx, dy, dz);
                }
#pragma unroll
                for (int v = 0; v < NV; v++)
                {
                    real a = phi * Ub[v];
                    if constexpr (VISC && J > 0)
                    {
                        a += dx * GMb[v] + dy * GMb[NV + v];
                        if (DIM == 3)
                            a += dz * GMb[2 * NV + v];
                    }
                    sRed[((((J - J0) * 2 + side) * NV + v) * NG + q) * 32 + fl] = a;
                }
            }
            shares<J + 1, J0>(xs, cell0, cell1, Ub0, Ub1, GMb, sRed, q, fl);
        }
    }

    // rounds of ROWS rows: the shares into sRed, summed over the points in point order into the face records
    // sOut (row 0, the cell means, adds to the Roe-average part already there)
    template <int J0>
    static DNDSB_D void rounds(const real *xs, const real *cell0, const real *cell1, const real *Ub0, const real *Ub1, const real *GMb, real *sRed,
                               real *sOut, const int *sC, int64_t f0, int64_t nFace, int q, int fl, int tid, int nthr)
    {
        if constexpr (J0 <= R)
        {
            constexpr int nRow = R + 1 - J0 < ROWS ? R + 1 - J0 : ROWS;
            shares<J0, J0>(xs, cell0, cell1, Ub0, Ub1, GMb, sRed, q, fl);
            __syncthreads();
            for (int e = tid; e < 32 * nRow * 2 * NV; e += nthr)
            {
                const int fi = e & 31, k = e >> 5;
                if (f0 + fi < nFace && sC[32 + fi] >= 0)
                {
                    real acc = 0;
#pragma unroll
                    for (int qq = 0; qq < NG; qq++)
                        acc += sRed[(k * NG + qq) * 32 + fi];
                    const int row = J0 + k / (2 * NV), side = (k / NV) & 1, v = k % NV;
                    real &o = sOut[fi * 2 * W + side * W + row * NV + v];
                    o = row == 0 ? o + acc : acc;
                }
            }
            __syncthreads();
            rounds<J0 + ROWS>(xs, cell0, cell1, Ub0, Ub1, GMb, sRed, sOut, sC, f0, nFace, q, fl, tid, nthr);
        }
    }
};

template <int DIM, int P, int NV, int NG, bool VISC>
__global__ void __launch_bounds__(32 * NG, vjp_min_blocks<NG>())
    k_rhs_vjp_fast(MeshD m, GeomD g, const real *__restrict__ facePt, const real *__restrict__ cellPar, const real *__restrict__ moment,
                   EulerSettingsD s, int hllep, const real *__restrict__ w, const real *__restrict__ u, const real *__restrict__ uRec,
                   const real *__restrict__ dLamCell, real *__restrict__ faceAdj, int *err)
{
    using Lt = Layout<DIM, P, NV>;
    using Rows = VjpRows<DIM, P, NV, NG, VISC>;
    constexpr int CS = Lt::CS, R = Lt::R, NDOF = Lt::NDOF, W = Rows::W, CH = Rows::CH;
    extern __shared__ real sm[];
    real *sCell = sm;                                // [64][CS]: slots 0..31 side-0 cells, 32..63 side-1 cells
    FaceData *sFace = (FaceData *)(sCell + 64 * CS); // [32]
    real *sG = (real *)(sFace + 32);                 // [32][NV] the cotangent jump w0 / V0 - w1 / V1
    real *sT = sG + 32 * NV;                         // [15][32] the Roe-average cotangents summed per face
    real *sRed = sT + 15 * 32;                       // [CH][NG][32] the point shares of one round
    real *sOut = sRed + CH * NG * 32;                // [32][2 W] the block's face records
    __shared__ int sC[64];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int64_t f0 = (int64_t)blockIdx.x * 32;
    const real gamma = s.gamma;
    if (tid < 32)
    {
        int64_t f = f0 + tid;
        sC[tid] = f < m.nFace ? m.face2cell[f * 2] : -1;
        sC[32 + tid] = f < m.nFace ? m.face2cell[f * 2 + 1] : -1;
    }
    const int fl = tid & 31, q = tid >> 5;
    const int64_t f = f0 + fl;
    real p0[3] = {0, 0, 0}, n[3] = {0, 0, 0}, JW = 0;
    if (f < m.nFace)
    {
        const real *pt = facePt + ((int64_t)q * m.nFace + f) * 7;
        p0[0] = pt[0], p0[1] = pt[1], p0[2] = pt[2], n[0] = pt[3], n[1] = pt[4], n[2] = pt[5], JW = pt[6];
    }
    __syncthreads();
    for (int e = tid; e < 64 * CS; e += nthr)
    {
        int slot = e / CS, off = e - slot * CS;
        int c = sC[slot];
        real val = 0;
        if (c >= 0)
        {
            if (off < Lt::OC)
                val = off < Lt::OU ? uRec[(int64_t)c * (R * NV) + off] : u[(int64_t)c * NV + off - Lt::OU];
            else if (off < Lt::OM)
                val = cellPar[(int64_t)c * 6 + off - Lt::OC];
            else if (off < Lt::OM + NDOF)
                val = moment[(int64_t)c * NDOF + off - Lt::OM];
        }
        sCell[e] = val;
    }
    for (int e = tid; e < 32 * 2 * W; e += nthr)
        sOut[e] = 0;
    __syncthreads();
    if (tid < 64)
    {
        // warp 0: Roe averages of the cell means; warp 1: dLambda, face geometry and the cotangent jump
        int t = tid & 31;
        int64_t ff = f0 + t;
        int c0 = sC[t], c1 = sC[32 + t];
        FaceData *fd = sFace + t;
        if (ff < m.nFace && c1 >= 0)
        {
            if (tid < 32)
            {
                RoeAvg r;
                roe_average(sCell + t * CS + Lt::OU, sCell + (32 + t) * CS + Lt::OU, gamma, r);
                fd->r = r;
            }
            else
            {
                fd->dLambda = dmax(dLamCell[c0], dLamCell[c1]);
                for (int d = 0; d < 3; d++)
                {
                    real sh = m.facePShift[ff * 3 + d];
                    fd->db[d] = g.cellBary[(int64_t)c1 * 3 + d] - sh - g.cellBary[(int64_t)c0 * 3 + d];
                    fd->shift[d] = sh;
                }
                fd->gbase = dmin(g.vol[c0], g.vol[c1]) * 2.0 / g.faceArea[ff];
                const real iv0 = 1.0 / g.vol[c0], iv1 = 1.0 / g.vol[c1];
                for (int v = 0; v < NV; v++)
                    sG[t * NV + v] = w[(int64_t)c0 * NV + v] * iv0 - w[(int64_t)c1 * NV + v] * iv1;
            }
        }
    }
    __syncthreads();
    const bool act = f < m.nFace && sC[32 + fl] >= 0;
    real Ub0[NV], Ub1[NV], GMb[VISC ? 3 * NV : 1];
    roe_rev::RoeBar rb;
    roe_rev::roebar_zero(rb);
#pragma unroll
    for (int v = 0; v < NV; v++)
        Ub0[v] = Ub1[v] = 0;
#pragma unroll
    for (int i = 0; i < (VISC ? 3 * NV : 1); i++)
        GMb[i] = 0;
    const real *cell0 = sCell + fl * CS, *cell1 = sCell + (32 + fl) * CS;
    real xs[6] = {0, 0, 0, 0, 0, 0}; // the point normalised in each side's cell frame
    if (act)
    {
        const FaceData *fd = sFace + fl;
        const real p1[3] = {p0[0] + fd->shift[0], p0[1] + fd->shift[1], p0[2] + fd->shift[2]};
        for (int d = 0; d < DIM; d++)
        {
            xs[d] = (p0[d] - cell0[Lt::OC + d]) * cell0[Lt::OL + d];
            xs[3 + d] = (p1[d] - cell1[Lt::OC + d]) * cell1[Lt::OL + d];
        }
        real UL[NV], UR[NV], G[3 * NV];
        recon_point<DIM, P, NV, false>(cell0, p0, UL, G);
        recon_point<DIM, P, NV, true>(cell1, p1, UR, G);
        if (!(UL[0] > 0 && UR[0] > 0 && fd->r.asqr > 0))
            atomicOr(err, (int)DE_NONPHYSICAL);
        real Fbar[NV];
#pragma unroll
        for (int v = 0; v < NV; v++)
            Fbar[v] = -JW * sG[fl * NV + v];
        if (NV == 5 && hllep)
            roe_rev::hllep_rev(UL, UR, n, fd->r, gamma, fd->dLambda, s.rsFixScale, Fbar, Ub0, Ub1, rb);
        else
        {
            // plain Roe on the five flow variables; with the SA model the nuTilde flux
            // F5 = ((vnL UL5 + vnR UR5) - (UR5 - UL5) l123) / 2 (sa_convective_flux) adds to the cotangents of the
            // point states and of the fixed eigenvalue l123
            real incU[5], incFb[5], incUb[5], AtL[5], AtR[5], l123 = 0;
#pragma unroll
            for (int v = 0; v < 5; v++)
                incU[v] = UR[v] - UL[v], incFb[v] = -0.5 * Fbar[v];
            const real l123b = NV == 6 ? -0.5 * (UR[NV - 1] - UL[NV - 1]) * Fbar[NV - 1] : 0.0;
            roe_rev::roe0_diss_rev(incU, n, fd->r, gamma, fd->dLambda, s.rsFixScale, s.rsIncFScale, incFb, incUb, rb, l123b, &l123);
            flux_jac_du_t<5>(UL, n, Fbar, 0.0, gamma, AtL);
            flux_jac_du_t<5>(UR, n, Fbar, 0.0, gamma, AtR);
#pragma unroll
            for (int v = 0; v < 5; v++)
                Ub0[v] = 0.5 * AtL[v] - incUb[v], Ub1[v] = 0.5 * AtR[v] + incUb[v];
            if constexpr (NV == 6)
            {
                const real iL = 1.0 / UL[0], iR = 1.0 / UR[0];
                const real vnL = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) * iL, vnR = (UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2]) * iR;
                const real fb = 0.5 * Fbar[5];
                Ub0[5] = fb * (vnL + l123), Ub1[5] = fb * (vnR - l123);
                const real vnLb = fb * UL[5], vnRb = fb * UR[5];
#pragma unroll
                for (int d = 0; d < 3; d++)
                    Ub0[1 + d] += vnLb * n[d] * iL, Ub1[1 + d] += vnRb * n[d] * iR;
                Ub0[0] -= vnLb * vnL * iL, Ub1[0] -= vnRb * vnR * iR;
            }
        }
        if constexpr (VISC)
        {
            // the compact gradient (EvaluateRHS.hxx:363-386): G holds GL + GR
            real distGRP = fd->gbase;
            distGRP = dmax(dmin(fabs(fd->db[0] * n[0] + fd->db[1] * n[1] + fd->db[2] * n[2]), distGRP * 2), distGRP * 0.25);
            const real iD = 1.0 / distGRP;
            real UMr[NV], Fvbar[NV], bar[4 * NV];
#pragma unroll
            for (int v = 0; v < NV; v++)
                UMr[v] = 0.5 * (UL[v] + UR[v]), Fvbar[v] = JW * sG[fl * NV + v];
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int v = 0; v < NV; v++)
                    G[d * NV + v] = G[d * NV + v] * 0.5 + iD * (n[d] * (UR[v] - UL[v]));
            visc_rev::visc_point_bar<NV>(s, UMr, G, n, Fvbar, bar);
#pragma unroll
            for (int v = 0; v < NV; v++)
            {
                const real nGb = n[0] * bar[NV + v] + n[1] * bar[2 * NV + v] + n[2] * bar[3 * NV + v];
                Ub0[v] += 0.5 * bar[v] - iD * nGb;
                Ub1[v] += 0.5 * bar[v] + iD * nGb;
            }
#pragma unroll
            for (int i = 0; i < 3 * NV; i++)
                GMb[i] = 0.5 * bar[NV + i];
        }
    }
    // the Roe-average cotangents: 15 fields summed over the points of each face
    {
        const real rf[15] = {rb.v[0], rb.v[1], rb.v[2], rb.vL[0], rb.vL[1], rb.vL[2], rb.vR[0], rb.vR[1], rb.vR[2],
                             rb.aL, rb.aR, rb.vsqr, rb.H, rb.asqr, rb.a};
#pragma unroll
        for (int k = 0; k < 15; k++)
            sRed[(k * NG + q) * 32 + fl] = rf[k];
        __syncthreads();
        for (int e = tid; e < 32 * 15; e += nthr)
        {
            const int fi = e & 31, k = e >> 5;
            real acc = 0;
#pragma unroll
            for (int qq = 0; qq < NG; qq++)
                acc += sRed[(k * NG + qq) * 32 + fi];
            sT[k * 32 + fi] = acc;
        }
        __syncthreads();
    }
    // ... carried to the cell means: thread e -> face e % 32, mean component e / 32 (side (e / 32) / NV)
    for (int e = tid; e < 32 * 2 * NV; e += nthr)
    {
        const int fi = e & 31, i = e >> 5;
        if (f0 + fi < m.nFace && sC[32 + fi] >= 0)
        {
            const real *m0 = sCell + fi * CS + Lt::OU, *m1 = sCell + (32 + fi) * CS + Lt::OU;
            RoeAvgT<D1> rD;
            D1 a[NV], b[NV];
#pragma unroll
            for (int v = 0; v < NV; v++)
                a[v] = D1::var(m0[v], i == v ? 0 : -1), b[v] = D1::var(m1[v], i == NV + v ? 0 : -1);
            roe_average(a, b, gamma, rD);
            const real *t = sT + fi;
            real x = t[9 * 32] * rD.aL.d[0] + t[10 * 32] * rD.aR.d[0] + t[11 * 32] * rD.vsqr.d[0] + t[12 * 32] * rD.H.d[0] +
                     t[13 * 32] * rD.asqr.d[0] + t[14 * 32] * rD.a.d[0];
#pragma unroll
            for (int d = 0; d < 3; d++)
                x += t[d * 32] * rD.v[d].d[0] + t[(3 + d) * 32] * rD.vL[d].d[0] + t[(6 + d) * 32] * rD.vR[d].d[0];
            sOut[fi * 2 * W + (i / NV) * W + i % NV] = x;
        }
    }
    __syncthreads();
    // the rows: the cell means (row 0) and the reconstruction rows 1..R
    Rows::template rounds<0>(xs, cell0, cell1, Ub0, Ub1, GMb, sRed, sOut, sC, f0, m.nFace, q, fl, tid, nthr);
    // interior faces' records (boundary faces keep what the boundary kernel stored)
    for (int e = tid; e < 32 * 2 * W; e += nthr)
    {
        const int fi = e / (2 * W);
        if (f0 + fi < m.nFace && sC[32 + fi] >= 0)
            faceAdj[f0 * 2 * W + e] = sOut[e];
    }
}

template <int DIM, int P, int NV, int NG>
int launch_vjp_fast(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, bool hllep, bool visc, const real *w, const real *u,
                    const real *uRec, real *faceAdj, cudaStream_t st)
{
    using Lt = Layout<DIM, P, NV>;
    constexpr int W = (Lt::R + 1) * NV, CH = VjpRows<DIM, P, NV, NG, true>::CH;
    constexpr size_t smem = sizeof(real) * (64 * Lt::CS + 32 * NV + 15 * 32 + CH * NG * 32 + 32 * 2 * W) + sizeof(FaceData) * 32;
    static_assert(smem <= 227 * 1024, "shared memory of k_rhs_vjp_fast above the 227 KB a block may hold");
    auto kern = visc ? k_rhs_vjp_fast<DIM, P, NV, NG, true> : k_rhs_vjp_fast<DIM, P, NV, NG, false>;
    static unsigned long long attrSet[2] = {0, 0}; // per variant, one bit per device: dynamic shared memory limit raised
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !((attrSet[visc] >> dev) & 1ULL))
    {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return ST_CUDA;
        attrSet[visc] |= 1ULL << dev;
    }
    const unsigned nb = (unsigned)((m.nFace + 31) / 32);
    kern<<<nb, 32 * NG, smem, st>>>(m, g, ev.facePt, ev.cellPar, vr.baseMoment, ev.s, hllep ? 1 : 0, w, u, uRec, ev.deltaLambdaCell, faceAdj,
                                    ev.errWord);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

template <int DIM, int P, int NV>
int dispatch_vjp_ng(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, bool hllep, bool visc, const real *w, const real *u,
                    const real *uRec, real *faceAdj, cudaStream_t st)
{
    const int nG = g.nGf;
    if constexpr (DIM == 3)
    {
        if (nG == 9)
            return launch_vjp_fast<DIM, P, NV, 9>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
        if (nG == 4)
            return launch_vjp_fast<DIM, P, NV, 4>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
        if (nG == 7)
            return launch_vjp_fast<DIM, P, NV, 7>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
        if (nG == 3)
            return launch_vjp_fast<DIM, P, NV, 3>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
        if (nG == 6)
            return launch_vjp_fast<DIM, P, NV, 6>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
    }
    else
    {
        if (nG == 3)
            return launch_vjp_fast<DIM, P, NV, 3>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
        if (nG == 2)
            return launch_vjp_fast<DIM, P, NV, 2>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
    }
    return ST_UNSUPPORTED;
}
} // namespace
} // namespace dndsb
