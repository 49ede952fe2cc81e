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

namespace dndsb
{
namespace
{
// packed exponents (ex + 4 ey + 16 ez) of the monomials, BaseFunction.hpp:55-107
DNDSB_HD constexpr int mcode(int dim, int k)
{
    constexpr int c3[20] = {0, 1, 4, 16, 2, 8, 32, 5, 20, 17, 3, 12, 48, 6, 9, 24, 36, 33, 18, 21};
    constexpr int c2[10] = {0, 1, 4, 2, 5, 8, 3, 6, 9, 12};
    return dim == 3 ? c3[k] : c2[k];
}

template <int DIM, int P, int NV>
struct Layout
{
    static constexpr int NDOF = ndof_of<DIM>(P);
    static constexpr int R = NDOF - 1;
    // per staged cell: uRec [R][NV], u [NV], centre [3], 1/L [3], moments [NDOF]
    static constexpr int OU = R * NV, OC = OU + NV, OL = OC + 3, OM = OL + 3;
    static constexpr int CS = (OM + NDOF) | 1; // odd stride: lanes of a warp (different faces) hit different banks
};

// per-face data shared by the Gauss points of a face (27 doubles: an odd stride in shared memory)
struct FaceData
{
    RoeAvg r;       // Roe averages of the two cell means
    real dLambda;   // max deltaLambdaCell of the two cells
    real db[3];     // barycentre difference, side 1 seen from side 0
    real gbase;     // 2 min(V0, V1) / A
    real shift[3];  // periodic translation into side 1's frame
    real pad;       // keeps the stride odd
};
static_assert(sizeof(FaceData) == 27 * sizeof(real), "FaceData layout");

// u + phi . uRec and the gradient D1 phi . uRec of one cell at point p (VariationalReconstruction.hpp:378-442 rows 0..dim)
template <int DIM, int P, int NV, bool ACC>
DNDSB_D void recon_point(const real *cell, const real *p, real *U, real *G)
{
    using Lt = Layout<DIM, P, NV>;
    const real *rec = cell, *uu = cell + Lt::OU, *cent = cell + Lt::OC, *iL = cell + Lt::OL, *mom = cell + Lt::OM;
    real x = (p[0] - cent[0]) * iL[0], y = (p[1] - cent[1]) * iL[1], z = DIM == 3 ? (p[2] - cent[2]) * iL[2] : 0.0;
    real px[4] = {1, x, x * x, x * x * x}, py[4] = {1, y, y * y, y * y * y}, pz[4] = {1, z, z * z, z * z * z};
#pragma unroll
    for (int v = 0; v < NV; v++)
    {
        U[v] = uu[v];
        if (!ACC)
            G[v] = G[NV + v] = G[2 * NV + v] = 0;
    }
#pragma unroll
    for (int k = 1; k < Lt::NDOF; k++)
    {
        const int c = mcode(DIM, k);
        const int ex = c & 3, ey = (c >> 2) & 3, ez = (c >> 4) & 3;
        real phi = px[ex] * py[ey] * pz[ez] - mom[k];
        real dx = ex ? ex * px[ex ? ex - 1 : 0] * py[ey] * pz[ez] * iL[0] : 0.0;
        real dy = ey ? ey * px[ex] * py[ey ? ey - 1 : 0] * pz[ez] * iL[1] : 0.0;
        real dz = ez ? ez * px[ex] * py[ey] * pz[ez ? ez - 1 : 0] * iL[2] : 0.0;
        const real *r = rec + (k - 1) * NV;
#pragma unroll
        for (int v = 0; v < NV; v++)
        {
            real rv = r[v];
            U[v] += phi * rv;
            if (ex)
                G[v] += dx * rv;
            if (ey)
                G[NV + v] += dy * rv;
            if (DIM == 3 && ez)
                G[2 * NV + v] += dz * rv;
        }
    }
}

// resident blocks per SM the register budget is sized for (about 18 warps per SM)
#ifndef DNDSB_RHS_WARPS_PER_SM
#define DNDSB_RHS_WARPS_PER_SM 18
#endif
template <int NG>
constexpr int min_blocks() { return (DNDSB_RHS_WARPS_PER_SM / NG) > 0 ? (DNDSB_RHS_WARPS_PER_SM / NG) : 1; }

template <int DIM, int P, int NV, int NG>
__global__ void __launch_bounds__(32 * NG, min_blocks<NG>())
    k_rhs_face_fast(MeshD m, GeomD g, const real *__restrict__ facePt, const real *__restrict__ cellPar, const real *__restrict__ moment,
                    EulerSettingsD s, const real *__restrict__ u, const real *__restrict__ uRec, const real *__restrict__ dLamCell,
                    real *__restrict__ faceFlux, int *err)
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
    real out[NV];
#pragma unroll
    for (int v = 0; v < NV; v++)
        out[v] = 0;
    if (f < m.nFace && sC[32 + fl] >= 0)
    {
        const FaceData *fd = sFace + fl;
        real p1[3] = {p0[0] + fd->shift[0], p0[1] + fd->shift[1], p0[2] + fd->shift[2]};
        // G holds GL + GR: the viscous gradient only needs their sum (EvaluateRHS.hxx:369-386)
        real UL[NV], UR[NV], G[3 * NV];
        recon_point<DIM, P, NV, false>(sCell + fl * CS, p0, UL, G);
        recon_point<DIM, P, NV, true>(sCell + (32 + fl) * CS, p1, UR, G);
        real Fv[5] = {0, 0, 0, 0, 0};
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
            grad_cons2prim<NV>(UM, G, GP, gamma);
            real irho = 1.0 / UM[0];
            real pM = (gamma - 1) * (UM[4] - 0.5 * (UM[1] * UM[1] + UM[2] * UM[2] + UM[3] * UM[3]) * irho);
            real Tm = pM / ((gamma - 1) / gamma * cp * UM[0]);
            real mu = mu_eff(s.muModel, s.muGas, s.TRef, s.CSutherland, UM[0], Tm);
            viscous_flux<NV>(UM, GP, n, false, gamma, mu, cp * mu / s.prGas, cp, Fv);
        }
        real F[5], l0, l1, l4;
        bool ok = riemann_flux_pre(s.rsType, UL, UR, fd->r, n, gamma, fd->dLambda, s.rsFixScale, s.rsIncFScale, F, l0, l1, l4);
#pragma unroll
        for (int v = 0; v < 5; v++)
            out[v] = -(F[v] - Fv[v]) * JW;
        bool fin = true;
#pragma unroll
        for (int v = 0; v < 5; v++)
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
// No barriers: the neighbour rows are read through L1 (the R threads of a cell
// share each row), and the next face's coefficient row is loaded while the
// current one is applied, so every thread keeps a full row of HBM loads in flight.
template <int R, int NV, typename TC>
__global__ void __launch_bounds__(32 * R) k_vr_jacobi_fast(int64_t nCell, int nf, const int32_t *__restrict__ nbr, const TC *__restrict__ AAInvB,
                                                           const TC *__restrict__ AInvb, const real *__restrict__ uRec, real *__restrict__ uRecNew,
                                                           const real *__restrict__ u, real relax, int recordInc, int uRecIsZero)
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
    const TC *Mbase = AAInvB + ((c * (nf + 1) + 1) * R + i) * R; // row i of block 1 + k is Mbase + k R^2
    TC Mcur[R], Mnext[R];
#pragma unroll
    for (int j = 0; j < R; j++)
        Mcur[j] = useRec ? Mbase[j] : TC(0);
    for (int k = 0; k < nf; k++)
    {
        if (k + 1 < nf)
        {
#pragma unroll
            for (int j = 0; j < R; j++)
                Mnext[j] = useRec ? Mbase[(k + 1) * R * R + j] : TC(0);
        }
        int o = nbr[c * nf + k];
        if (o >= 0)
        {
            real bi = (real)AInvb[(c * nf + k) * R + i];
            const real *rr = uRec + (int64_t)o * R * NV;
            const real *uo = u + (int64_t)o * NV;
            real t[NV];
#pragma unroll
            for (int v = 0; v < NV; v++)
                t[v] = bi * (uo[v] - ui[v]);
            if (useRec)
            {
#pragma unroll
                for (int j = 0; j < R; j++)
                {
                    real mij = (real)Mcur[j];
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
        for (int j = 0; j < R; j++)
            Mcur[j] = Mnext[j];
    }
#pragma unroll
    for (int v = 0; v < NV; v++)
        uRecNew[(c * R + i) * NV + v] = acc[v];
}

// VR Jacobi sweep with the coefficient stream staged by bulk async copies (the Blackwell TMA
// engine, untiled form): each block owns G consecutive cells at a time; one thread issues a single
// cp.async.bulk of their packed [G][nf][R][R+1] coefficients into shared memory and an mbarrier
// counts the bytes in; meanwhile every thread loads its own row of uRec and u.  R threads per
// cell then apply the rows from shared memory (neighbour reconstructions through L1/L2).  Several
// resident blocks per SM keep several copies in flight.  The wait on the mbarrier is bounded:
// when it runs out the block records an error and returns after a second bounded wait.
DNDSB_D uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

DNDSB_D bool mbar_wait(uint32_t mb, uint32_t phase, int limit)
{
    for (int it = 0; it < limit; it++)
    {
        uint32_t ok;
        asm volatile("{\n .reg .pred P1;\n mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n selp.b32 %0, 1, 0, P1;\n}\n"
                     : "=r"(ok)
                     : "r"(mb), "r"(phase)
                     : "memory");
        if (ok)
            return true;
    }
    return false;
}

template <int R, int NV, typename TC, int G>
__global__ void __launch_bounds__(G * R) k_vr_jacobi_bulk(int64_t nCell, int nf, const int32_t *__restrict__ nbr, const TC *__restrict__ coef,
                                                          const real *__restrict__ uRec, real *__restrict__ uRecNew, const real *__restrict__ u,
                                                          real relax, int recordInc, int uRecIsZero, int *err)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) unsigned long long mbar;
    const TC *sc = (const TC *)smraw;
    const int tid = threadIdx.x, cl = tid / R, i = tid - cl * R;
    const int per = nf * R * (R + 1);
    const uint32_t bytesPerCell = (uint32_t)(per * sizeof(TC));
    const uint32_t mb = smem_addr(&mbar), sdst = smem_addr(smraw);
    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mb), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const real sgn = recordInc ? -1.0 : relax;
    const bool useRec = !(recordInc && uRecIsZero);
    uint32_t phase = 0;
    for (int64_t grp = blockIdx.x; grp * G < nCell; grp += gridDim.x)
    {
        const int64_t c0 = grp * G;
        const int n = (int)(nCell - c0 < G ? nCell - c0 : G);
        if (tid == 0)
        {
            const uint32_t bytes = (uint32_t)n * bytesPerCell;
            const TC *src = coef + c0 * per;
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mb), "r"(bytes) : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(sdst), "l"(src),
                         "r"(bytes), "r"(mb)
                         : "memory");
        }
        const int64_t c = c0 + cl;
        const bool act = cl < n;
        real acc[NV], ui[NV];
        int on[8];
        if (act)
        {
#pragma unroll
            for (int v = 0; v < NV; v++)
            {
                real x = uRec[(c * R + i) * NV + v];
                acc[v] = recordInc ? (uRecIsZero ? 0.0 : x) : x * (1 - relax);
                ui[v] = u[c * NV + v];
            }
            for (int k = 0; k < nf; k++)
                on[k] = nbr[c * nf + k];
        }
        // every thread waits (bounded), then the block decides together whether the copy landed
        bool landed = mbar_wait(mb, phase, 1 << 22);
        if (!__syncthreads_and(landed))
        {
            if (tid == 0)
                atomicOr(err, 1);
            mbar_wait(mb, phase, 1 << 22); // let a late copy finish before the block's shared memory is released
            return;
        }
        phase ^= 1;
        if (act)
        {
            for (int k = 0; k < nf; k++)
            {
                int o = on[k];
                if (o < 0)
                    continue;
                const TC *row = sc + (cl * nf + k) * R * (R + 1) + i * (R + 1);
                real bi = (real)row[R];
                const real *rr = uRec + (int64_t)o * R * NV;
                const real *uo = u + (int64_t)o * NV;
                real t[NV];
#pragma unroll
                for (int v = 0; v < NV; v++)
                    t[v] = bi * (uo[v] - ui[v]);
                if (useRec)
                {
#pragma unroll
                    for (int j = 0; j < R; j++)
                    {
                        real mij = (real)row[j];
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
            for (int v = 0; v < NV; v++)
                uRecNew[(c * R + i) * NV + v] = acc[v];
        }
        __syncthreads(); // every row read before the next copy lands
    }
}

template <int R, typename TC>
constexpr int bulk_group() { return R <= 3 ? 64 : R <= 5 ? 32 : R <= 9 ? 16 : 8; }

template <int R, typename TC>
int launch_vr_bulk(const MeshD &m, const VRD &vr, const TC *coef, const real *uRec, real *uRecNew, const real *u, int recordInc, int uRecIsZero,
                   cudaStream_t st)
{
    constexpr int G = bulk_group<R, TC>();
    const size_t cellBytes = (size_t)m.nf * R * (R + 1) * sizeof(TC);
    if (cellBytes % 16 != 0 || m.nf > 8 || !coef || !vr.sweepErr)
        return ST_UNSUPPORTED;
    const size_t smem = cellBytes * G;
    if (smem > 200 * 1024)
        return ST_UNSUPPORTED;
    static unsigned long long attrSet = 0; // one bit per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !((attrSet >> dev) & 1ULL))
    {
        if (cudaFuncSetAttribute(k_vr_jacobi_bulk<R, 5, TC, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return ST_CUDA;
        attrSet |= 1ULL << dev;
    }
    int64_t groups = (m.nCell + G - 1) / G;
    int perSM = (int)((220 * 1024) / (smem + 1024));
    perSM = perSM < 1 ? 1 : perSM > 8 ? 8 : perSM;
    int64_t grid = 148LL * perSM;
    if (grid > groups)
        grid = groups;
    k_vr_jacobi_bulk<R, 5, TC, G><<<(unsigned)grid, G * R, smem, st>>>(m.nCell, m.nf, m.cellNbr, coef, uRec, uRecNew, u, vr.s.jacobiRelax,
                                                                       recordInc, uRecIsZero, vr.sweepErr);
    return ST_OK;
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
        if (cudaFuncSetAttribute(k_rhs_face_fast<DIM, P, NV, NG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return ST_CUDA;
        attrSet |= 1ULL << dev;
    }
    unsigned nb = (unsigned)((m.nFace + 31) / 32);
    k_rhs_face_fast<DIM, P, NV, NG><<<nb, 32 * NG, smem, st>>>(m, g, ev.facePt, ev.cellPar, vr.baseMoment, ev.s, u, uRec, ev.deltaLambdaCell, ff,
                                                              ev.errWord);
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
    if (!ev.facePt || ev.s.nVars != 5)
        return ST_UNSUPPORTED;
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
    if (nv != 5 || m.nf > 6)
        return ST_UNSUPPORTED;
    unsigned nb = (unsigned)((m.nCell + 31) / 32);
    real relax = vr.s.jacobiRelax;
#define DNDSB_VRF(RR)                                                                                                                       \
    do                                                                                                                                      \
    {                                                                                                                                       \
        int brc = useFP32 ? launch_vr_bulk<RR, float>(m, vr, vr.sweepCoef32, uRec, uRecNew, u, recordInc, uRecIsZero, st)               \
                          : launch_vr_bulk<RR, real>(m, vr, vr.sweepCoef, uRec, uRecNew, u, recordInc, uRecIsZero, st);                   \
        if (brc == ST_CUDA)                                                                                                                 \
            return ST_CUDA;                                                                                                                 \
        if (brc == ST_OK)                                                                                                                   \
            break;                                                                                                                          \
        if (useFP32)                                                                                                                        \
            k_vr_jacobi_fast<RR, 5, float><<<nb, 32 * RR, 0, st>>>(m.nCell, m.nf, m.cellNbr, vr.AAInvB32, vr.AInvb32, uRec, uRecNew, u, relax, \
                                                                   recordInc, uRecIsZero);                                                  \
        else                                                                                                                                \
            k_vr_jacobi_fast<RR, 5, real><<<nb, 32 * RR, 0, st>>>(m.nCell, m.nf, m.cellNbr, vr.AAInvB, vr.AInvb, uRec, uRecNew, u, relax,    \
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
    case 19:
        DNDSB_VRF(19);
        break;
    default:
        return ST_UNSUPPORTED;
    }
#undef DNDSB_VRF
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
