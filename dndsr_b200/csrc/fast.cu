// Tuned kernels of the two dominant operators.
//
// RHS face flux: one thread per (face, Gauss point), 32 faces per block.  The
// reconstruction data of the 64 cells adjacent to the block's faces (uRec,
// cell mean, centre, length scales, moments) are staged once in shared
// memory; per-face Roe averages (shared by every Gauss point of a face,
// Gas.hpp:229-259) are computed once; the Gauss-point contributions are
// summed in a fixed order, so results are deterministic.  The basis and its
// first derivatives are generated from compile-time exponent tables, so the
// sparse derivative rows cost only their non-zero terms.
//
// VR Jacobi sweep: R threads per cell (one output row each), 32 cells per
// block.  Each thread streams its rows of the A^-1 B_k blocks once (coalesced
// across the cell's threads) while the neighbour reconstructions are staged
// in shared memory face by face.
#include "solver.cuh"
#include "basis_eval.cuh"
#include "sa.cuh"
#include "fast_common.cuh"

namespace dndsb
{
namespace
{
using namespace fastc;

// resident blocks per SM the register budget is sized for (about 27 warps per SM: at 9 points per
// face, 3 blocks of 288 threads with 72 registers each and some spilling beat 2 blocks with 96 by
// 18 % on the TGV workload at 64^3)
#ifndef DNDSB_RHS_WARPS_PER_SM
#define DNDSB_RHS_WARPS_PER_SM 27
#endif
template <int NG>
constexpr int min_blocks() { return (DNDSB_RHS_WARPS_PER_SM / NG) > 0 ? (DNDSB_RHS_WARPS_PER_SM / NG) : 1; }

// MODE 0: the whole integrand; 1: the inviscid flux only, from point values without their gradients (the
// evaluators that ignore viscosity).  Splitting a viscous evaluation into an inviscid and a viscous launch
// measured 1.63 ms against 0.94 ms for one MODE 0 launch on the TGV workload (the staging and the point
// values done twice), so viscous evaluations stay in one launch.
// LAM: also record the face integrals of the Riemann eigenvalues divided by the area into lam [3][nFace]
// (EvaluateRHS.hxx:527-545, for useRoeJacobian); a separate instantiation, so the default one is unchanged
template <int DIM, int P, int NV, int NG, int MODE, bool LAM>
__global__ void __launch_bounds__(32 * NG, min_blocks<NG>())
    k_rhs_face_fast(MeshD m, GeomD g, const real *__restrict__ facePt, const real *__restrict__ cellPar, const real *__restrict__ moment,
                    EulerSettingsD s, const real *__restrict__ u, const real *__restrict__ uRec, const real *__restrict__ dLamCell,
                    real *__restrict__ faceFlux, int *err, real *__restrict__ lam)
{
    using Lt = Layout<DIM, P, NV>;
    constexpr int CS = Lt::CS, R = Lt::R, NDOF = Lt::NDOF;
    extern __shared__ real sm[];
    real *sCell = sm;                                 // [64][CS]: slots 0..31 side-0 cells, 32..63 side-1 cells
    FaceData *sFace = (FaceData *)(sCell + 64 * CS);  // [32]
    real *sFlux = (real *)(sFace + 32);               // [NG][32][NV]
    __shared__ int sC[64];
    const int tid = threadIdx.x;
    const int64_t f0 = (int64_t)blockIdx.x * 32;
    const real gamma = s.gamma, cp = s.Rgas * gamma / (gamma - 1);
    if (tid < 32)
    {
        int64_t f = f0 + tid;
        sC[tid] = f < m.nFace ? m.face2cell[f * 2] : -1;
        sC[32 + tid] = f < m.nFace ? m.face2cell[f * 2 + 1] : -1;
    }
    // this thread's Gauss point (issued before the staging barriers so the loads overlap them)
    const int fl = tid & 31, q = tid >> 5;
    const int64_t f = f0 + fl;
    real p0[3] = {0, 0, 0}, n[3] = {0, 0, 0}, JW = 0;
    if (f < m.nFace)
    {
        const real *pt = facePt + ((int64_t)q * m.nFace + f) * 7;
        p0[0] = pt[0], p0[1] = pt[1], p0[2] = pt[2], n[0] = pt[3], n[1] = pt[4], n[2] = pt[5], JW = pt[6];
    }
    __syncthreads();
    for (int e = tid; e < 64 * CS; e += blockDim.x)
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
            // off == OM + NDOF is the padding slot of an odd stride: nothing to read
        }
        sCell[e] = val;
    }
    __syncthreads();
    if (tid < 64)
    {
        // warp 0: Roe averages of the cell means; warp 1: dLambda and face geometry
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
            }
        }
    }
    __syncthreads();
    real out[NV], lw[3] = {0, 0, 0};
#pragma unroll
    for (int v = 0; v < NV; v++)
        out[v] = 0;
    if (f < m.nFace && sC[32 + fl] >= 0)
    {
        const FaceData *fd = sFace + fl;
        real p1[3] = {p0[0] + fd->shift[0], p0[1] + fd->shift[1], p0[2] + fd->shift[2]};
        // G holds GL + GR: the viscous gradient only needs their sum (EvaluateRHS.hxx:369-386)
        real UL[NV], UR[NV], G[MODE == 1 ? 1 : 3 * NV];
        if constexpr (MODE == 1)
        {
            recon_value<DIM, P, NV>(sCell + fl * CS, p0, UL);
            recon_value<DIM, P, NV>(sCell + (32 + fl) * CS, p1, UR);
        }
        else
        {
            recon_point<DIM, P, NV, false>(sCell + fl * CS, p0, UL, G);
            recon_point<DIM, P, NV, true>(sCell + (32 + fl) * CS, p1, UR, G);
        }
        real Fv[NV];
#pragma unroll
        for (int v = 0; v < NV; v++)
            Fv[v] = 0;
        if constexpr (MODE != 1)
            if (!s.ignoreVis)
        {
            real distGRP = fd->gbase;
            distGRP = dmax(dmin(fabs(fd->db[0] * n[0] + fd->db[1] * n[1] + fd->db[2] * n[2]), distGRP * 2), distGRP * 0.25);
            real iD = 1.0 / distGRP;
            real UM[NV], GP[3 * NV];
#pragma unroll
            for (int v = 0; v < NV; v++)
                UM[v] = 0.5 * (UL[v] + UR[v]);
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int v = 0; v < NV; v++)
                    G[d * NV + v] = G[d * NV + v] * 0.5 + iD * (n[d] * (UR[v] - UL[v]));
            real irho = 1.0 / UM[0]; // the one reciprocal density of the viscous flux
            grad_cons2prim_ir<NV>(UM, irho, G, GP, gamma);
            if (NV == 5)
            {
                real pM = (gamma - 1) * (UM[4] - 0.5 * (UM[1] * UM[1] + UM[2] * UM[2] + UM[3] * UM[3]) * irho);
                real Tm = pM * irho * s.kT;
                real mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, UM[0], Tm);
                viscous_flux_ir<NV>(UM, irho, GP, n, false, gamma, mu, cp * mu * s.iPr, s.kT, Fv);
            }
            else // SA: eddy viscosity in the momentum/energy fluxes and the nuTilde diffusion flux
                point_viscous_flux<NV>(s, UM, GP, n, false, Fv);
        }
        real F[NV], l0, l1, l4, nm[3];
        bool ok = true;
#pragma unroll
        for (int v = 0; v < NV; v++)
            F[v] = 0;
        {
            if (s.rsMeanValueEig) // batched mean-value eigenvalues along the face's mean normal
                nm[0] = g.faceMeanNorm[f * 3], nm[1] = g.faceMeanNorm[f * 3 + 1], nm[2] = g.faceMeanNorm[f * 3 + 2];
            ok = riemann_flux_pre(s.rsType, UL, UR, fd->r, n, gamma, fd->dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4,
                                  s.rsMeanValueEig ? (const real *)nm : nullptr);
            if (NV == 6)
                F[NV - 1] = sa_convective_flux(UL, UR, n, l1);
        }
#pragma unroll
        for (int v = 0; v < NV; v++)
            out[v] = -(F[v] - Fv[v]) * JW;
        if constexpr (LAM)
            lw[0] = l0 * JW, lw[1] = l1 * JW, lw[2] = l4 * JW;
        bool fin = true;
#pragma unroll
        for (int v = 0; v < NV; v++)
            fin = fin && isfinite(out[v]);
        if (!ok || !fin)
            atomicOr(err, !ok ? (int)DE_NONPHYSICAL : (int)DE_NONFINITE);
    }
#pragma unroll
    for (int v = 0; v < NV; v++)
        sFlux[(q * 32 + fl) * NV + v] = out[v];
    __syncthreads();
    // coalesced write of the 32 faces x NV block; the sum over Gauss points runs in q order
    for (int e = tid; e < 32 * NV; e += blockDim.x)
    {
        int fi = e / NV, v = e - fi * NV;
        int64_t ff = f0 + fi;
        if (ff < m.nFace)
        {
            real acc = 0;
#pragma unroll
            for (int qq = 0; qq < NG; qq++)
                acc += sFlux[(qq * 32 + fi) * NV + v];
            faceFlux[ff * NV + v] = acc;
        }
    }
    if constexpr (LAM)
    {
        __syncthreads(); // sFlux is reused for the eigenvalues
#pragma unroll
        for (int i = 0; i < 3; i++)
            sFlux[(q * 32 + fl) * NV + i] = lw[i];
        __syncthreads();
        for (int e = tid; e < 32 * 3; e += blockDim.x)
        {
            int fi = e / 3, i = e - fi * 3;
            int64_t ff = f0 + fi;
            if (ff < m.nFace && sC[32 + fi] >= 0) // boundary faces are recorded by the boundary kernel
            {
                real acc = 0;
#pragma unroll
                for (int qq = 0; qq < NG; qq++)
                    acc += sFlux[(qq * 32 + fi) * NV + i];
                lam[i * m.nFace + ff] = acc / g.faceArea[ff];
            }
        }
    }
}

// facePt [NG][nFace][7] = point, unit normal, |J| w   and cellPar [nCell][6] = centre, 1/L
DNDSB_GLOBAL void k_face_points(int64_t nFace, int nG, const real *__restrict__ pp, const real *__restrict__ nrm, const real *__restrict__ jd,
                                const real *__restrict__ qw, real *out)
{
    DNDSB_KERNEL_LOOP(i, nFace * nG)
    {
        int64_t f = i / nG;
        int q = (int)(i - f * nG);
        real *o = out + ((int64_t)q * nFace + f) * 7;
        for (int d = 0; d < 3; d++)
            o[d] = pp[i * 3 + d], o[3 + d] = nrm[i * 3 + d];
        o[6] = jd[i] * qw[q];
    }
}

template <int DIM>
DNDSB_GLOBAL void k_cell_par(int64_t nCell, int aniso, const real *__restrict__ cent, const real *__restrict__ hbox, real *out)
{
    DNDSB_KERNEL_LOOP(c, nCell)
    {
        real L[3];
        cell_lengths<DIM>(hbox + c * 3, aniso, L);
        for (int d = 0; d < 3; d++)
            out[c * 6 + d] = cent[c * 3 + d], out[c * 6 + 3 + d] = 1.0 / L[d];
    }
}

// VR Jacobi sweep, R threads per cell (VariationalReconstruction_Reconstruction.hxx:485-615).
// Coefficients come from the packed, transposed stream coefT[cell][face][j][i] (j < R: A^-1 B
// entry (i, j); j = R: A^-1 b entry i), so for each j the R threads of a cell read R consecutive
// values (one or two L1 lines per cell instead of a strided row each).  The neighbour's uRec
// block and mean are read as broadcasts: the R threads of a cell share each line through L1.
// No barriers; the next face's coefficients are loaded while the current face is applied.
template <int R, int NV, typename TC>
__global__ void __launch_bounds__(32 * R, 2) k_vr_jacobi_fast(int64_t nCell, int nf, const int32_t *__restrict__ nbr, const TC *__restrict__ coefT,
                                                           const real *__restrict__ uRec, real *__restrict__ uRecNew, const real *__restrict__ u,
                                                           real relax, int recordInc, int uRecIsZero)
{
    const int tid = threadIdx.x;
    const int cl = tid / R, i = tid - cl * R;
    const int64_t c = (int64_t)blockIdx.x * 32 + cl;
    if (c >= nCell)
        return;
    real acc[NV], ui[NV];
#pragma unroll
    for (int v = 0; v < NV; v++)
    {
        real x = uRec[(c * R + i) * NV + v];
        acc[v] = recordInc ? (uRecIsZero ? 0.0 : x) : x * (1 - relax);
        ui[v] = u[c * NV + v];
    }
    const real sgn = recordInc ? -1.0 : relax;
    const bool useRec = !(recordInc && uRecIsZero);
    const TC *cb = coefT + c * nf * (R + 1) * R + i; // entry (face k, j) at cb[(k (R+1) + j) R]
    TC Mcur[R + 1], Mnext[R + 1];
#pragma unroll
    for (int j = 0; j <= R; j++)
        Mcur[j] = (useRec || j == R) ? cb[j * R] : TC(0);
    for (int k = 0; k < nf; k++)
    {
        if (k + 1 < nf)
        {
#pragma unroll
            for (int j = 0; j <= R; j++)
                Mnext[j] = (useRec || j == R) ? cb[((k + 1) * (R + 1) + j) * R] : TC(0);
        }
        int o = nbr[c * nf + k];
        if (o >= 0)
        {
            real t[NV];
            const real *rr = uRec + (int64_t)o * R * NV;
            const real *uo = u + (int64_t)o * NV;
            const real bi = (real)Mcur[R];
#pragma unroll
            for (int v = 0; v < NV; v++)
                t[v] = bi * (uo[v] - ui[v]);
            if (useRec)
            {
#pragma unroll
                for (int j = 0; j < R; j++)
                {
                    const real mij = (real)Mcur[j];
#pragma unroll
                    for (int v = 0; v < NV; v++)
                        t[v] += mij * rr[j * NV + v];
                }
            }
#pragma unroll
            for (int v = 0; v < NV; v++)
                acc[v] += sgn * t[v];
        }
#pragma unroll
        for (int j = 0; j <= R; j++)
            Mcur[j] = Mnext[j];
    }
#pragma unroll
    for (int v = 0; v < NV; v++)
        uRecNew[(c * R + i) * NV + v] = acc[v];
}

template <int DIM, int P, int NV, int NG>
int launch_rhs_fast(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *u, const real *uRec, real *ff, cudaStream_t st)
{
    using Lt = Layout<DIM, P, NV>;
    size_t smem = sizeof(real) * (64 * Lt::CS + NG * 32 * NV) + sizeof(FaceData) * 32;
    static unsigned long long attrSet = 0; // one bit per device: dynamic shared memory limit raised
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !((attrSet >> dev) & 1ULL))
    {
        if (cudaFuncSetAttribute(k_rhs_face_fast<DIM, P, NV, NG, 0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_rhs_face_fast<DIM, P, NV, NG, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_rhs_face_fast<DIM, P, NV, NG, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_rhs_face_fast<DIM, P, NV, NG, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return ST_CUDA;
        attrSet |= 1ULL << dev;
    }
    unsigned nb = (unsigned)((m.nFace + 31) / 32);
    real *lam = ev.jacMode == 2 ? ev.lambdaFace0 : nullptr;
#define DNDSB_RFF(MODE, LAM)                                                                                                                  \
    k_rhs_face_fast<DIM, P, NV, NG, MODE, LAM><<<nb, 32 * NG, smem, st>>>(m, g, ev.facePt, ev.cellPar, vr.baseMoment, ev.s, u, uRec,            \
                                                                          ev.deltaLambdaCell, ff, ev.errWord, lam)
    if (ev.s.ignoreVis)
    {
        if (lam)
            DNDSB_RFF(1, true);
        else
            DNDSB_RFF(1, false);
    }
    else
    {
        if (lam)
            DNDSB_RFF(0, true);
        else
            DNDSB_RFF(0, false);
    }
#undef DNDSB_RFF
    return ST_OK;
}

template <int DIM, int P>
int dispatch_ng(int nG, const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *u, const real *uRec, real *ff,
                cudaStream_t st)
{
    if (DIM == 3)
    {
        if (nG == 9)
            return launch_rhs_fast<DIM, P, 5, 9>(m, g, vr, ev, u, uRec, ff, st);
        if (nG == 4)
            return launch_rhs_fast<DIM, P, 5, 4>(m, g, vr, ev, u, uRec, ff, st);
        if (nG == 7)
            return launch_rhs_fast<DIM, P, 5, 7>(m, g, vr, ev, u, uRec, ff, st);
        if (nG == 3)
            return launch_rhs_fast<DIM, P, 5, 3>(m, g, vr, ev, u, uRec, ff, st);
        if (nG == 6)
            return launch_rhs_fast<DIM, P, 5, 6>(m, g, vr, ev, u, uRec, ff, st);
    }
    else
    {
        if (nG == 3)
            return launch_rhs_fast<DIM, P, 5, 3>(m, g, vr, ev, u, uRec, ff, st);
        if (nG == 2)
            return launch_rhs_fast<DIM, P, 5, 2>(m, g, vr, ev, u, uRec, ff, st);
    }
    return ST_UNSUPPORTED;
}
} // namespace

int fast_geometry(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, cudaStream_t st)
{
    if (dev_alloc((void **)&ev.facePt, sizeof(real) * m.nFace * g.nGf * 7) != cudaSuccess ||
        dev_alloc((void **)&ev.cellPar, sizeof(real) * m.nCell * 6) != cudaSuccess)
        return ST_CUDA;
    DNDSB_LAUNCH(k_face_points, m.nFace * g.nGf, 256, st, m.nFace, g.nGf, g.facePP, g.faceNorm, g.faceJDet, g.faceQw, ev.facePt);
    if (m.dim == 2)
        DNDSB_LAUNCH(k_cell_par<2>, m.nCell, 256, st, m.nCell, vr.s.anisotropicLengths, g.cellCent, g.cellScale, ev.cellPar);
    else
        DNDSB_LAUNCH(k_cell_par<3>, m.nCell, 256, st, m.nCell, vr.s.anisotropicLengths, g.cellCent, g.cellScale, ev.cellPar);
    return dev_sync(st) == cudaSuccess && last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

// returns ST_UNSUPPORTED when no tuned instantiation exists (the caller then uses the generic kernel)
int rhs_face_fast(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *u, const real *uRec, real *ff, cudaStream_t st)
{
    if (!ev.facePt || (ev.s.nVars != 5 && ev.s.nVars != 6))
        return ST_UNSUPPORTED;
    if (ev.s.nVars == 6)
    {
        // the SA model: hexahedral meshes at degree 1 (quadrilateral faces, 4 or 9 points)
        if (m.dim != 3 || vr.P != 1)
            return ST_UNSUPPORTED;
        if (g.nGf == 4)
            return launch_rhs_fast<3, 1, 6, 4>(m, g, vr, ev, u, uRec, ff, st);
        if (g.nGf == 9)
            return launch_rhs_fast<3, 1, 6, 9>(m, g, vr, ev, u, uRec, ff, st);
        return ST_UNSUPPORTED;
    }
    if (m.dim == 2)
    {
        if (vr.P == 1)
            return dispatch_ng<2, 1>(g.nGf, m, g, vr, ev, u, uRec, ff, st);
        if (vr.P == 2)
            return dispatch_ng<2, 2>(g.nGf, m, g, vr, ev, u, uRec, ff, st);
        return dispatch_ng<2, 3>(g.nGf, m, g, vr, ev, u, uRec, ff, st);
    }
    if (vr.P == 1)
        return dispatch_ng<3, 1>(g.nGf, m, g, vr, ev, u, uRec, ff, st);
    if (vr.P == 2)
        return dispatch_ng<3, 2>(g.nGf, m, g, vr, ev, u, uRec, ff, st);
    return dispatch_ng<3, 3>(g.nGf, m, g, vr, ev, u, uRec, ff, st);
}

int vr_iter_fast(const MeshD &m, const VRD &vr, int nv, const real *uRec, real *uRecNew, const real *u, int recordInc, int uRecIsZero,
                 int useFP32, cudaStream_t st)
{
    if ((nv != 5 && nv != 6) || !vr.sweepCoef)
        return ST_UNSUPPORTED;
    if (nv == 6)
    {
        // the SA model at degree 1 in 3-D (R = 3)
        if (vr.R != 3)
            return ST_UNSUPPORTED;
        unsigned nb6 = (unsigned)((m.nCell + 31) / 32);
        if (useFP32)
            k_vr_jacobi_fast<3, 6, float><<<nb6, 32 * 3, 0, st>>>(m.nCell, m.nf, m.cellNbr, vr.sweepCoef32, uRec, uRecNew, u, vr.s.jacobiRelax,
                                                                 recordInc, uRecIsZero);
        else
            k_vr_jacobi_fast<3, 6, real><<<nb6, 32 * 3, 0, st>>>(m.nCell, m.nf, m.cellNbr, vr.sweepCoef, uRec, uRecNew, u, vr.s.jacobiRelax,
                                                                recordInc, uRecIsZero);
        return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
    }
    unsigned nb = (unsigned)((m.nCell + 31) / 32);
    real relax = vr.s.jacobiRelax;
#define DNDSB_VRF(RR)                                                                                                                       \
    do                                                                                                                                      \
    {                                                                                                                                       \
        if (useFP32)                                                                                                                        \
            k_vr_jacobi_fast<RR, 5, float><<<nb, 32 * RR, 0, st>>>(m.nCell, m.nf, m.cellNbr, vr.sweepCoef32, uRec, uRecNew, u, relax,      \
                                                                   recordInc, uRecIsZero);                                                  \
        else                                                                                                                                \
            k_vr_jacobi_fast<RR, 5, real><<<nb, 32 * RR, 0, st>>>(m.nCell, m.nf, m.cellNbr, vr.sweepCoef, uRec, uRecNew, u, relax,         \
                                                                  recordInc, uRecIsZero);                                                   \
    } while (0)
    switch (vr.R)
    {
    case 2:
        DNDSB_VRF(2);
        break;
    case 3:
        DNDSB_VRF(3);
        break;
    case 5:
        DNDSB_VRF(5);
        break;
    case 9:
        DNDSB_VRF(9);
        break;
    default:
        return ST_UNSUPPORTED;
    }
#undef DNDSB_VRF
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
