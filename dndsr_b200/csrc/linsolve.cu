// Native implicit linear solve: LU-SGS sweeps and left-preconditioned
// restarted GMRES in FP64 or FP32, with every scalar kept on the device.
//
// Replaces EulerSolver::solveLinear / doPrecondition
// (src/Euler/EulerSolver.hxx:1407-1579, 1605-1658) together with
// LUSGSMatrixInit (src/Euler/EulerEvaluator.hxx:37-159, scalar Jacobian),
// UpdateSGS (:550-693), LUSGSMatrixVec (:175-274) and
// GMRES_LeftPreconditioned::solve (src/Solver/Linear.hpp:46-133).
//
// Layout.  Inside the solve every cell vector is stored in colour-position
// order (position p holds cell colorCells[p]), so one colour class is one
// contiguous range and "neighbour already updated in this sweep" is a range
// test on the neighbour's position.  Per (position, face slot) the operator
// keeps {w*n, w*lambda} with w = alpha * A_f / (2 V_c) as one 4-vector and the
// neighbour's position; per position the scalar diagonal.  The state u is
// converted once per solve into the solve precision T.
//
// Precision.  T = double reproduces the FP64 operators; T = float is the
// FP32 preconditioner of the mixed-precision defect correction (the caller's
// residual and state update stay FP64).  Dot products accumulate in FP64 in
// both cases.  Reductions use a fixed partition and fixed trees, so results
// are bitwise reproducible.
//
// jacobiCode 2: the preconditioner is the reference's local LU (LUSGSMatrixToJacobianLU +
// LUSGSMatrixSolveJacobianLU, EulerEvaluator.hxx:290-359, 838-927; doPrecondition EulerSolver.hxx:1642-1657) with
// iluCode 0: a block ILU(0) of the operator factored colour by colour (ilu.cuh) once per solve, applied as two
// defect-correction steps x += (LU)^-1 (b - A x).  With the scalar Jacobian the operator is kept in block form
// (the scalar diagonal and the scalar flux increments as blocks) for it.
//
// Block mode (useScalarJacobian false, optionally useRoeJacobian): the operator is kept as dense blocks,
// per position the diagonal block and its inverse, per (position, face slot) the off-diagonal block
// (alpha/2)(A_f/V_c) dF/dU_o (the reference's fluxJacobian0_Right_Times_du_AsMatrix, the same blocks its
// local LU assembles, EulerEvaluator.hxx:290-359), built in FP64 and stored in T.
//
// GMRES scalars (Hessenberg, norms, least-squares solution, breakdown index)
// never leave the device: the whole solve is a fixed kernel sequence and is
// captured once into a CUDA graph that later solves replay.
#include "solver.cuh"
#include "roejac.cuh"
#include "ilu.cuh"

namespace dndsb
{
namespace
{
template <typename T>
struct Vec4;
template <>
struct Vec4<float>
{
    using type = float4;
};
template <>
struct Vec4<double>
{
    using type = double4;
};

// ---------------------------------------------------------------------------
// operator build: LUSGSMatrixInit (EulerEvaluator.hxx:37-159) + packing
// ---------------------------------------------------------------------------
// JD: diagonals per cell (1, or NV with the SA source Jacobian)
template <typename T, int NV>
constexpr int jd_of() { return NV == 6 ? NV : 1; }

template <typename T, int NV>
DNDSB_GLOBAL void k_sgsop_build(MeshD m, GeomD g, const real *__restrict__ lamFace, const real *__restrict__ dTau, real dt, real alphaDiag,
                                const real *__restrict__ u, const real *__restrict__ jSource, const int32_t *__restrict__ cellPos,
                                int32_t *nbrPos, typename Vec4<T>::type *op, T *jd, T *uT)
{
    DNDSB_KERNEL_LOOP(p, m.nCell)
    {
        int64_t c = m.colorCells[p];
        real iv = 1.0 / g.vol[c];
        real cf = 0.5 * alphaDiag / g.vol[c];
        real fp = 1.0 / dTau[c] + 1.0 / dt;
        for (int k = 0; k < m.nf; k++)
        {
            int pk = m.cell2face[c * m.nf + k];
            int64_t f = pk >> 1;
            real sg = (pk & 1) ? -1.0 : 1.0;
            fp += (0.5 * alphaDiag) * g.faceArea[f] * lamFace[f] * iv;
            real w = cf * g.faceArea[f];
            typename Vec4<T>::type o4;
            o4.x = (T)(w * g.faceMeanNorm[f * 3] * sg);
            o4.y = (T)(w * g.faceMeanNorm[f * 3 + 1] * sg);
            o4.z = (T)(w * g.faceMeanNorm[f * 3 + 2] * sg);
            o4.w = (T)(w * lamFace[f]);
            op[p * m.nf + k] = o4;
            int o = m.cellNbr[c * m.nf + k];
            nbrPos[p * m.nf + k] = o < 0 ? -1 : cellPos[o];
        }
        constexpr int JD = jd_of<T, NV>();
        for (int v = 0; v < JD; v++)
            jd[p * JD + v] = (T)(fp + (JD > 1 ? alphaDiag * jSource[c * NV + v] : 0.0));
        for (int v = 0; v < NV; v++)
            uT[p * NV + v] = (T)u[c * NV + v];
    }
}

// natural order FP64 -> position order T, and back
template <typename T, int NV>
DNDSB_GLOBAL void k_gather_T(int64_t n, const int32_t *__restrict__ pos2cell, const real *__restrict__ x, T *y)
{
    DNDSB_KERNEL_LOOP(p, n)
    {
        int64_t c = pos2cell[p];
        for (int v = 0; v < NV; v++)
            y[p * NV + v] = (T)x[c * NV + v];
    }
}

template <typename T, int NV>
DNDSB_GLOBAL void k_scatter_T(int64_t n, const int32_t *__restrict__ pos2cell, const T *__restrict__ y, real *x)
{
    DNDSB_KERNEL_LOOP(p, n)
    {
        int64_t c = pos2cell[p];
        for (int v = 0; v < NV; v++)
            x[c * NV + v] = (real)y[p * NV + v];
    }
}

template <typename T>
DNDSB_GLOBAL void k_zero_T(int64_t n, T *x)
{
    DNDSB_KERNEL_LOOP(i, n)
    x[i] = (T)0;
}

template <typename T>
DNDSB_GLOBAL void k_copy_T(int64_t n, const T *__restrict__ a, T *b)
{
    DNDSB_KERNEL_LOOP(i, n)
    b[i] = a[i];
}

template <typename T>
DNDSB_GLOBAL void k_sub_T(int64_t n, const T *__restrict__ a, const T *__restrict__ b, T *c) // c = a - b
{
    DNDSB_KERNEL_LOOP(i, n)
    c[i] = a[i] - b[i];
}

template <typename T>
DNDSB_GLOBAL void k_add_T(int64_t n, const T *__restrict__ a, T *b) // b += a
{
    DNDSB_KERNEL_LOOP(i, n)
    b[i] += a[i];
}

// scaled flux-increment Jacobian times dU (EulerEvaluator.hpp:1100-1158 with
// Gas.hpp:462-513), minus w*lambda*dU; o4 = {w n, w lambda}
template <typename T, int NV>
DNDSB_D void jac_du_scaled(const T *U, const T *dU, const typename Vec4<T>::type &o4, T gamma, T *dF)
{
    T ir = T(1) / U[0];
    T v0 = U[1] * ir, v1 = U[2] * ir, v2 = U[3] * ir;
    T p = (gamma - T(1)) * (U[4] - U[0] * T(0.5) * (v0 * v0 + v1 * v1 + v2 * v2));
    T dv0 = (dU[1] - U[1] * ir * dU[0]) * ir;
    T dv1 = (dU[2] - U[2] * ir * dU[0]) * ir;
    T dv2 = (dU[3] - U[3] * ir * dU[0]) * ir;
    T dp = (gamma - T(1)) * (dU[4] - T(0.5) * (dU[1] * v0 + dU[2] * v1 + dU[3] * v2 + U[1] * dv0 + U[2] * dv1 + U[3] * dv2));
    T vn = v0 * o4.x + v1 * o4.y + v2 * o4.z;
    T dvn = dv0 * o4.x + dv1 * o4.y + dv2 * o4.z;
    dF[0] = dU[1] * o4.x + dU[2] * o4.y + dU[3] * o4.z;
    dF[1] = dU[1] * vn + U[1] * dvn + o4.x * dp;
    dF[2] = dU[2] * vn + U[2] * dvn + o4.y * dp;
    dF[3] = dU[3] * vn + U[3] * dvn + o4.z * dp;
    dF[4] = (dU[4] + dp) * vn + (U[4] + p) * dvn;
    for (int j = 5; j < NV; j++)
        dF[j] = dU[j] * vn + U[j] * dvn;
    for (int j = 0; j < NV; j++)
        dF[j] -= o4.w * dU[j];
}

// one colour class of a forward / backward sweep (UpdateSGS, EulerEvaluator.hxx:550-693)
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_sgs_pos(int64_t pBeg, int64_t pEnd, const int32_t *__restrict__ nbrPos, const typename Vec4<T>::type *__restrict__ op,
                            const T *__restrict__ jd, const T *__restrict__ uT, const T *__restrict__ rhs, const T *__restrict__ xOld,
                            T *xNew, T gamma, int forward, int gsUpdate, int uIncIsZero)
{
    DNDSB_KERNEL_LOOP(ii, pEnd - pBeg)
    {
        int64_t p = pBeg + ii;
        T buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = rhs[p * NV + v];
#pragma unroll
        for (int k = 0; k < NF; k++)
        {
            int q = nbrPos[p * NF + k];
            if (q < 0 || q == p)
                continue;
            bool useNew = gsUpdate && (forward ? q < pBeg : q >= pEnd);
            if (uIncIsZero && !useNew)
                continue;
            typename Vec4<T>::type o4 = op[p * NF + k];
            const T *dU = (useNew ? xNew : xOld) + (int64_t)q * NV;
            T dF[NV];
            jac_du_scaled<T, NV>(uT + (int64_t)q * NV, dU, o4, gamma, dF);
            for (int v = 0; v < NV; v++)
                buf[v] -= dF[v];
        }
        constexpr int JD = jd_of<T, NV>();
        for (int v = 0; v < NV; v++)
            xNew[p * NV + v] = buf[v] * (T(1) / jd[p * JD + (JD > 1 ? v : 0)]);
    }
}

// LUSGSMatrixVec (EulerEvaluator.hxx:175-274)
// xs (may be null): a scale of x (the normalising factor of an unnormalised basis column): Ax = A (xs x)
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_matvec_pos(int64_t n, const int32_t *__restrict__ nbrPos, const typename Vec4<T>::type *__restrict__ op,
                               const T *__restrict__ jd, const T *__restrict__ uT, const T *__restrict__ x, T *Ax, T gamma,
                               const real *__restrict__ xs)
{
    const T sx = xs ? (T)*xs : T(1);
    DNDSB_KERNEL_LOOP(p, n)
    {
        T buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = 0;
#pragma unroll
        for (int k = 0; k < NF; k++)
        {
            int q = nbrPos[p * NF + k];
            if (q < 0)
                continue;
            typename Vec4<T>::type o4 = op[p * NF + k];
            T dF[NV];
            jac_du_scaled<T, NV>(uT + (int64_t)q * NV, x + (int64_t)q * NV, o4, gamma, dF);
            for (int v = 0; v < NV; v++)
                buf[v] -= dF[v];
        }
        constexpr int JD = jd_of<T, NV>();
        for (int v = 0; v < NV; v++)
            Ax[p * NV + v] = sx * (jd[p * JD + (JD > 1 ? v : 0)] * x[p * NV + v] - buf[v]);
    }
}

// block operator build.  Storage is tiled by 32 positions (ilu::BlockLay, s = 5): element k NV NV + e of a position's
// row of opB is element e of slot k's off-diagonal block (zero on boundaries); elements e and NV NV + e of jdB are
// the diagonal block and its inverse.  A warp reads one element of its 32 positions as one 256-byte line
// (FP64).  Per face slot the Roe dissipation
// matrix M of the face (Roe average of the two cells, the eigenvalues seen from this cell) is formed once: the
// diagonal block gains w (M + lambdaVis I) (and on a boundary face w (A(u_g) - M - lambdaVis I) dGhost/du), the
// off-diagonal block is w (A(u_o) - M - lambdaVis I); without the Roe term w (A(u_o) - lambdaFace I) and the
// scalar diagonal.  The same blocks as roej::cell_block and the neighbour increments, summed in the same order.
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_sgsop_build_blk(MeshD m, GeomD g, BoundaryD bnd, EvalD ev, int roe, const real *__restrict__ dTau, real dt, real alphaDiag,
                                    const real *__restrict__ u, const int32_t *__restrict__ cellPos, int32_t *nbrPos, T *opB, T *jdB, int *err)
{
    using namespace roej;
    constexpr int NN = NV * NV;
    const ilu::BlockLay oL{NF * NN, 5}, dL{2 * NN, 5};
    const real gamma = ev.s.gamma;
    DNDSB_KERNEL_LOOP(p, m.nCell)
    {
        int64_t c = m.colorCells[p];
        const real *uc = u + c * NV;
        real B[NN];
        for (int i = 0; i < NN; i++)
            B[i] = 0;
        real fp = 1.0 / dTau[c] + 1.0 / dt;
        const real iv = 1.0 / g.vol[c];
#pragma unroll 1
        for (int k = 0; k < NF; k++)
        {
            int o = m.cellNbr[c * NF + k];
            nbrPos[p * NF + k] = o < 0 ? -1 : cellPos[o];
            int pk = m.cell2face[c * NF + k];
            int64_t f = pk >> 1;
            int side = pk & 1;
            fp += (0.5 * alphaDiag) * g.faceArea[f] * ev.lambdaFace[f] * iv;
            real sg = side ? -1.0 : 1.0;
            real nn[3] = {g.faceMeanNorm[f * 3] * sg, g.faceMeanNorm[f * 3 + 1] * sg, g.faceMeanNorm[f * 3 + 2] * sg};
            real w = (0.5 * alphaDiag) * g.faceArea[f] * iv;
            real O[NN]; // the off-diagonal block (before w), zero on boundaries
            for (int i = 0; i < NN; i++)
                O[i] = 0;
            real uj[NV];
            if (o >= 0)
            {
                for (int v = 0; v < NV; v++)
                    uj[v] = u[(int64_t)o * NV + v];
                for (int i = 0; i < NV; i++) // A(u_o) by columns
                {
                    real e[NV], col[NV];
                    for (int v = 0; v < NV; v++)
                        e[v] = v == i ? 1.0 : 0.0;
                    flux_inc<NV>(uj, nn, e, gamma, col);
                    for (int v = 0; v < NV; v++)
                        O[v * NV + i] = col[v];
                }
            }
            if (!roe)
            {
                if (o >= 0)
                    for (int i = 0; i < NV; i++)
                        O[i * NV + i] -= ev.lambdaFace[f];
            }
            else
            {
                int zone = m.faceZone[f];
                if (o < 0 && !bc_value<NV>(bnd, zone, uc, nn, uj))
                    for (int v = 0; v < NV; v++)
                        uj[v] = uc[v];
                FaceLam L = face_lam(ev, f, side);
                RoeAvg r;
                roe_average(uc, uj, gamma, r);
                real M[NN];
                for (int i = 0; i < NV; i++)
                {
                    real e[NV], col[NV];
                    for (int v = 0; v < NV; v++)
                        e[v] = v == i ? 1.0 : 0.0, col[v] = 0;
                    roe_fdiff_add<NV>(e, nn, r, gamma, L.l0, L.l123, L.l4, col);
                    for (int v = 0; v < NV; v++)
                        M[v * NV + i] = col[v] + (v == i ? L.vis : 0.0);
                }
                for (int i = 0; i < NN; i++)
                    B[i] += w * M[i];
                if (o >= 0)
                    for (int i = 0; i < NN; i++)
                        O[i] -= M[i];
                else
                {
                    // (A(u_g) - M) JBC with the linearised ghost JBC (column-major)
                    int bt = (zone >= 0 && zone < bnd.nZone) ? bnd.type[zone] : 0;
                    real JBC[NN];
                    bc_linear<NV>(bt, nn, JBC);
                    for (int i = 0; i < NV; i++)
                    {
                        real dcol[NV], col[NV];
                        bool zero = true;
                        for (int v = 0; v < NV; v++)
                            dcol[v] = JBC[i * NV + v], zero = zero && dcol[v] == 0;
                        if (zero)
                            continue;
                        flux_inc<NV>(uj, nn, dcol, gamma, col);
                        for (int v = 0; v < NV; v++)
                        {
                            real md = 0;
                            for (int l = 0; l < NV; l++)
                                md += M[v * NV + l] * dcol[l];
                            B[v * NV + i] += w * (col[v] - md);
                        }
                    }
                }
            }
            for (int i = 0; i < NN; i++)
                opB[oL.at(p, k * NN + i)] = (T)(w * O[i]);
        }
        for (int i = 0; i < NV; i++)
        {
            if (roe)
                B[i * NV + i] += 1.0 / dTau[c] + 1.0 / dt;
            else
                B[i * NV + i] = fp;
            if (NV >= 6 && ev.jSource)
                B[i * NV + i] += alphaDiag * ev.jSource[c * NV + i];
        }
        real Bi[NN];
        if (!block_inv<NV>(B, Bi))
        {
            atomicOr(err, (int)DE_SINGULAR);
            for (int i = 0; i < NN; i++)
                Bi[i] = 0;
        }
        for (int i = 0; i < NN; i++)
            jdB[dL.at(p, i)] = (T)B[i], jdB[dL.at(p, NN + i)] = (T)Bi[i];
    }
}

// one colour class of a sweep with the block operator: x_p = D_p^-1 (rhs_p - sum_k O_pk x_q)
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_sgs_pos_blk(int64_t n, int64_t pBeg, int64_t pEnd, const int32_t *__restrict__ nbrPos, const T *__restrict__ opB,
                                const T *__restrict__ jdB, const T *__restrict__ rhs, const T *__restrict__ xOld, T *xNew, int forward, int gsUpdate,
                                int uIncIsZero)
{
    constexpr int NN = NV * NV;
    const ilu::BlockLay oL{NF * NN, 5}, dL{2 * NN, 5};
    DNDSB_KERNEL_LOOP(ii, pEnd - pBeg)
    {
        int64_t p = pBeg + ii;
        T buf[NV];
        for (int v = 0; v < NV; v++)
            buf[v] = rhs[p * NV + v];
#pragma unroll
        for (int k = 0; k < NF; k++)
        {
            int q = nbrPos[p * NF + k];
            if (q < 0 || q == p)
                continue;
            bool useNew = gsUpdate && (forward ? q < pBeg : q >= pEnd);
            if (uIncIsZero && !useNew)
                continue;
            const T *dU = (useNew ? xNew : xOld) + (int64_t)q * NV;
            T xq[NV];
            for (int l = 0; l < NV; l++)
                xq[l] = dU[l];
            for (int r = 0; r < NV; r++)
            {
                T acc = 0;
                for (int l = 0; l < NV; l++)
                    acc += opB[oL.at(p, k * NN + r * NV + l)] * xq[l];
                buf[r] -= acc;
            }
        }
        for (int r = 0; r < NV; r++)
        {
            T acc = 0;
            for (int l = 0; l < NV; l++)
                acc += jdB[dL.at(p, NN + r * NV + l)] * buf[l];
            xNew[p * NV + r] = acc;
        }
    }
}

template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_matvec_pos_blk(int64_t n, const int32_t *__restrict__ nbrPos, const T *__restrict__ opB, const T *__restrict__ jdB,
                                   const T *__restrict__ x, T *Ax, const real *__restrict__ xs)
{
    constexpr int NN = NV * NV;
    const ilu::BlockLay oL{NF * NN, 5}, dL{2 * NN, 5};
    const T sx = xs ? (T)*xs : T(1);
    DNDSB_KERNEL_LOOP(p, n)
    {
        T xp[NV], y[NV];
        for (int l = 0; l < NV; l++)
            xp[l] = x[p * NV + l];
        for (int r = 0; r < NV; r++)
        {
            T acc = 0;
            for (int l = 0; l < NV; l++)
                acc += jdB[dL.at(p, r * NV + l)] * xp[l];
            y[r] = acc;
        }
#pragma unroll
        for (int k = 0; k < NF; k++)
        {
            int q = nbrPos[p * NF + k];
            if (q < 0)
                continue;
            T xq[NV];
            for (int l = 0; l < NV; l++)
                xq[l] = x[(int64_t)q * NV + l];
            for (int r = 0; r < NV; r++)
            {
                T acc = 0;
                for (int l = 0; l < NV; l++)
                    acc += opB[oL.at(p, k * NN + r * NV + l)] * xq[l];
                y[r] += acc;
            }
        }
        for (int v = 0; v < NV; v++)
            Ax[p * NV + v] = sx * y[v];
    }
}

// GMRES bookkeeping kernels on device scalars.  sc layout: [0] scale = |M b|,
// [1] beta, [2] number of valid Arnoldi columns, [8 ...] least-squares y.
constexpr int kScY = 8;

// v = -(w - MLb) / beta  with beta = |w - MLb| already in sc[1]; x = 0 start uses w = 0
template <typename T>
DNDSB_GLOBAL void k_gmres_v0(int64_t n, const T *__restrict__ w, const T *__restrict__ MLb, T *v0, const real *sc, int wIsZero)
{
    real beta = sc[1];
    real s = beta > kVerySmall ? -1.0 / beta : 0.0;
    DNDSB_KERNEL_LOOP(i, n)
    {
        real d = (wIsZero ? 0.0 : (real)w[i]) - (real)MLb[i];
        v0[i] = (T)(d * s);
    }
}

// least squares  min |beta e1 - H y|  by Givens rotations on the Hessenberg
// (HardEigen::EigenLeastSquareSolve on the (j+1) x j leading block), over the valid columns and at most
// ncolMax of them; res (may be null): the norm of the least-squares residual, |beta e1 - H y|
DNDSB_GLOBAL void k_gmres_lsq(int k, const real *H, real *sc, int ncolMax, real *res)
{
    if (blockIdx.x != 0 || threadIdx.x != 0)
        return;
    int nv = (int)sc[2];
    if (nv > k)
        nv = k;
    if (nv > ncolMax)
        nv = ncolMax;
    real R[33 * 32];
    real gv[33];
    for (int i = 0; i <= nv; i++)
        gv[i] = i == 0 ? sc[1] : 0.0;
    for (int jj = 0; jj < nv; jj++)
        for (int i = 0; i <= nv; i++)
            R[i * 32 + jj] = i <= jj + 1 ? H[jj * (k + 1) + i] : 0.0;
    for (int jj = 0; jj < nv; jj++)
    {
        real a = R[jj * 32 + jj], b = R[(jj + 1) * 32 + jj];
        real r = sqrt(a * a + b * b);
        real c = r > 0 ? a / r : 1.0, s = r > 0 ? b / r : 0.0;
        for (int l = jj; l < nv; l++)
        {
            real x0 = R[jj * 32 + l], x1 = R[(jj + 1) * 32 + l];
            R[jj * 32 + l] = c * x0 + s * x1;
            R[(jj + 1) * 32 + l] = -s * x0 + c * x1;
        }
        real g0 = gv[jj], g1 = gv[jj + 1];
        gv[jj] = c * g0 + s * g1;
        gv[jj + 1] = -s * g0 + c * g1;
    }
    real rmax = 0;
    for (int jj = 0; jj < nv; jj++)
        rmax = dmax(rmax, fabs(R[jj * 32 + jj]));
    for (int jj = nv - 1; jj >= 0; jj--)
    {
        real acc = gv[jj];
        for (int l = jj + 1; l < nv; l++)
            acc -= R[jj * 32 + l] * sc[kScY + l];
        real d = R[jj * 32 + jj];
        sc[kScY + jj] = fabs(d) > 1e-14 * rmax ? acc / d : 0.0;
    }
    for (int jj = nv; jj < k; jj++)
        sc[kScY + jj] = 0;
    if (res)
        *res = fabs(gv[nv]);
}

// x += sum_i y_i v_i over the valid columns (v_i = colScale_i times the stored column)
template <typename T>
DNDSB_GLOBAL void k_gmres_update(int64_t n, int64_t ld, int k, const T *__restrict__ V, const real *__restrict__ sc,
                                 const real *__restrict__ colScale, T *x)
{
    int nv = (int)sc[2];
    if (nv > k)
        nv = k;
    DNDSB_KERNEL_LOOP(i, n)
    {
        real acc = (real)x[i];
        for (int jj = 0; jj < nv; jj++)
            acc += sc[kScY + jj] * colScale[jj] * (real)V[jj * ld + i];
        x[i] = (T)acc;
    }
}

// a new Arnoldi cycle: k valid columns so far, the first column stored normalised
DNDSB_GLOBAL void k_gmres_reset(real *sc, int k, real *colScale)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        sc[2] = k, colScale[0] = 1.0;
}

// scalars of a caller-driven Arnoldi cycle: weights of the plain dot, k columns valid, column 0 stored normalised
DNDSB_GLOBAL void k_krylov_begin(real *s2, unsigned *cnt, real *gsc, int k, real *colScale)
{
    if (blockIdx.x == 0 && threadIdx.x < 8)
        s2[threadIdx.x] = 1.0;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *cnt = 0, gsc[2] = k, colScale[0] = 1.0;
}

DNDSB_GLOBAL void k_krylov_scale(real *gsc)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        gsc[0] = gsc[1];
}

DNDSB_GLOBAL void k_copy_scalar(const real *a, real *b)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *b = *a;
}
} // namespace

// workspace owned by an evaluator handle
struct LinWs
{
    int prec = -1, k = 0, nv = 0, nf = 0, jacMode = 0;
    int64_t nCell = 0;
    int32_t *cellPos = nullptr, *nbrPos = nullptr;
    void *op = nullptr, *jd = nullptr, *uT = nullptr, *rhsT = nullptr, *x = nullptr, *tmp = nullptr, *tmp2 = nullptr, *MLb = nullptr,
         *V = nullptr;
    real *H = nullptr, *sc = nullptr, *s2 = nullptr, *red = nullptr;
    void *opB = nullptr, *jdB = nullptr; // block mode: off-diagonal blocks [nCell][nf][nv][nv], diagonal blocks + inverses [nCell][2][nv][nv]
    void *luB = nullptr, *luD = nullptr, *tmp3 = nullptr; // jacobiCode 2: ILU(0) slot blocks, inverted pivots, scratch
    int32_t *luNbr = nullptr, *luNLow = nullptr;          // the factors' compact slot order: neighbour positions, lower count
    real *colScale = nullptr; // [33] normalising factors of the stored (unnormalised) Krylov columns
    unsigned *cnt = nullptr;  // ticket counter of the one-launch reductions (zero between launches)
    cudaStream_t cs = nullptr;
    cudaEvent_t evIn = nullptr, evOut = nullptr;
    cudaGraphExec_t graph = nullptr;
    LinSettings key{};
    bool keyValid = false;
};

void linws_free(LinWs *w)
{
    if (!w)
        return;
    for (void *p : {(void *)w->cellPos, (void *)w->nbrPos, w->op, w->jd, w->opB, w->jdB, w->luB, w->luD, w->tmp3, (void *)w->luNbr,
                    (void *)w->luNLow, w->uT, w->rhsT, w->x, w->tmp, w->tmp2, w->MLb, w->V, (void *)w->H,
                    (void *)w->sc, (void *)w->s2, (void *)w->red, (void *)w->colScale, (void *)w->cnt})
        dev_free(p);
    graph_free(w->graph);
    stream_free(w->cs);
    event_free(w->evIn);
    event_free(w->evOut);
    delete w;
}

namespace
{
bool same_key(const LinSettings &a, const LinSettings &b)
{
    if (a.gmresCode != b.gmresCode || a.jacobiCode != b.jacobiCode || a.sgsIter != b.sgsIter || a.nGmresSpace != b.nGmresSpace ||
        a.nGmresIter != b.nGmresIter || a.precision != b.precision)
        return false;
    return true;
}

int ws_prepare(const MeshD &m, LinWs *&w, const LinSettings &ls, int nv, int jacMode)
{
    int k = ls.gmresCode ? ls.nGmresSpace : 0;
    size_t es = ls.precision ? sizeof(float) : sizeof(double);
    if (w && w->prec == ls.precision && w->k >= k && w->nv == nv && w->nCell == m.nCell && (w->jacMode != 0) == (jacMode != 0) &&
        (ls.jacobiCode != 2 || w->luB))
    {
        w->jacMode = jacMode; // block with or without the Roe term: same storage, rebuilt by every solve
        return ST_OK;
    }
    linws_free(w);
    w = new LinWs();
    w->prec = ls.precision, w->k = k, w->nv = nv, w->nf = m.nf, w->nCell = m.nCell, w->jacMode = jacMode;
    int64_t n = m.nCell * nv;
    bool ok = dev_alloc((void **)&w->cellPos, sizeof(int32_t) * m.nCell) == cudaSuccess &&
              dev_alloc((void **)&w->nbrPos, sizeof(int32_t) * m.nCell * m.nf) == cudaSuccess &&
              dev_alloc(&w->op, 4 * es * m.nCell * m.nf) == cudaSuccess && dev_alloc(&w->jd, es * m.nCell * (nv == 6 ? 6 : 1)) == cudaSuccess &&
              dev_alloc(&w->uT, es * n) == cudaSuccess && dev_alloc(&w->rhsT, es * n) == cudaSuccess &&
              dev_alloc(&w->x, es * n) == cudaSuccess && dev_alloc(&w->tmp, es * n) == cudaSuccess &&
              dev_alloc(&w->tmp2, es * n) == cudaSuccess && dev_alloc(&w->MLb, es * n) == cudaSuccess &&
              dev_alloc(&w->V, es * krylov_ld(n) * (k + 1)) == cudaSuccess &&
              dev_alloc((void **)&w->H, sizeof(real) * (k + 1) * (k > 0 ? k : 1)) == cudaSuccess &&
              dev_alloc((void **)&w->sc, sizeof(real) * (kScY + 40)) == cudaSuccess &&
              dev_alloc((void **)&w->s2, sizeof(real) * 8) == cudaSuccess &&
              dev_alloc((void **)&w->red, sizeof(real) * kRedBufLenK) == cudaSuccess &&
              dev_alloc((void **)&w->colScale, sizeof(real) * 33) == cudaSuccess && dev_alloc((void **)&w->cnt, sizeof(unsigned)) == cudaSuccess;
    const int64_t nPad = ilu::padded_rows(m.nCell, 5); // the block arrays are tiled by 32 positions
    if (ok && jacMode)
        ok = dev_alloc(&w->opB, es * nv * nv * nPad * m.nf) == cudaSuccess && dev_alloc(&w->jdB, es * 2 * nv * nv * nPad) == cudaSuccess;
    if (ok && jacMode && ls.jacobiCode == 2)
        ok = dev_alloc(&w->luB, es * nv * nv * nPad * m.nf) == cudaSuccess && dev_alloc(&w->luD, es * nv * nv * nPad) == cudaSuccess &&
             dev_alloc(&w->tmp3, es * n) == cudaSuccess && dev_alloc((void **)&w->luNbr, sizeof(int32_t) * m.nCell * m.nf) == cudaSuccess &&
             dev_alloc((void **)&w->luNLow, sizeof(int32_t) * m.nCell) == cudaSuccess;
    ok = ok && dev_zero(w->V, es * krylov_ld(n) * (k + 1), nullptr) == cudaSuccess; // the column pads stay zero
    ok = ok && dev_zero(w->cnt, sizeof(unsigned), nullptr) == cudaSuccess && dev_zero(w->colScale, sizeof(real) * 33, nullptr) == cudaSuccess;
    if (!ok || stream_create(&w->cs) != cudaSuccess || event_create(&w->evIn) != cudaSuccess || event_create(&w->evOut) != cudaSuccess)
    {
        linws_free(w);
        w = nullptr;
        return ST_CUDA;
    }
    // position of every cell in the colour order
    std::vector<int32_t> pos2cell(m.nCell), pos(m.nCell);
    d2h(pos2cell.data(), m.colorCells, sizeof(int32_t) * m.nCell, nullptr);
    if (dev_sync(nullptr) != cudaSuccess)
        return ST_CUDA;
    for (int64_t p = 0; p < m.nCell; p++)
        pos[pos2cell[p]] = (int32_t)p;
    h2d(w->cellPos, pos.data(), sizeof(int32_t) * m.nCell, nullptr);
    return dev_sync(nullptr) == cudaSuccess ? ST_OK : ST_CUDA;
}

template <typename T, int NV, int NF>
struct Solve
{
    const MeshD &m;
    LinWs &w;
    const LinSettings &ls;
    T gamma;
    cudaStream_t st;
    int64_t n() const { return m.nCell * NV; }
    using T4 = typename Vec4<T>::type;
    int64_t ld() const { return krylov_ld(n()); }
    T *V(int i) const { return (T *)w.V + (int64_t)i * ld(); }

    // one colour sweep over all classes; result in xNew
    void sweep(const T *rhs, const T *xOld, T *xNew, bool forward, bool gs, bool zeroIn) const
    {
        if (w.jacMode)
        {
            auto kb = k_sgs_pos_blk<T, NV, NF>;
            if (!gs)
            {
                DNDSB_LAUNCH(kb, m.nCell, 128, st, m.nCell, 0, m.nCell, w.nbrPos, (const T *)w.opB, (const T *)w.jdB, rhs, xOld, xNew, (int)forward,
                             0, (int)zeroIn);
                return;
            }
            for (int ci = 0; ci < m.nColor; ci++)
            {
                int col = forward ? ci : m.nColor - 1 - ci;
                int64_t b = m.colorStart[col], e = m.colorStart[col + 1];
                DNDSB_LAUNCH(kb, e - b, 128, st, m.nCell, b, e, w.nbrPos, (const T *)w.opB, (const T *)w.jdB, rhs, xOld, xNew, (int)forward, 1,
                             (int)zeroIn);
            }
            return;
        }
        if (!gs)
        {
            auto kern = k_sgs_pos<T, NV, NF>;
            DNDSB_LAUNCH(kern, m.nCell, 128, st, 0, m.nCell, w.nbrPos, (const T4 *)w.op, (const T *)w.jd,
                         (const T *)w.uT, rhs, xOld, xNew, gamma, (int)forward, 0, (int)zeroIn);
            return;
        }
        auto kern = k_sgs_pos<T, NV, NF>;
        for (int ci = 0; ci < m.nColor; ci++)
        {
            int col = forward ? ci : m.nColor - 1 - ci;
            int64_t b = m.colorStart[col], e = m.colorStart[col + 1];
            DNDSB_LAUNCH(kern, e - b, 128, st, b, e, w.nbrPos, (const T4 *)w.op, (const T *)w.jd, (const T *)w.uT, rhs,
                         xOld, xNew, gamma, (int)forward, 1, (int)zeroIn);
        }
    }

    // doPrecondition with jacobiCode 2 (EulerSolver.hxx:1642-1657): two LUSGSMatrixSolveJacobianLU steps,
    // x += (LU)^-1 (rhs - A x) (x = (LU)^-1 rhs from a zero input)
    void ilu_pair(const T *rhs, T *x, bool zeroIn) const
    {
        int64_t nn = n();
        T *r = (T *)w.tmp2, *ax = (T *)w.tmp3;
        for (int it = 0; it < 2; it++)
        {
            bool zero = zeroIn && it == 0;
            T *y = zero ? x : r;
            if (!zero)
            {
                FA(x, ax);
                DNDSB_LAUNCH(k_sub_T<T>, nn, 256, st, nn, rhs, (const T *)ax, r);
            }
            auto kl = ilu::k_ilu_lower_c<T, NV, NF>;
            auto ku = ilu::k_ilu_upper_c<T, NV, NF>;
            const ilu::BlockLay lay{NF * NV * NV, 5}, dlay{NV * NV, 5};
            for (int ci = 0; ci < m.nColor; ci++)
                DNDSB_LAUNCH(kl, m.colorStart[ci + 1] - m.colorStart[ci], 128, st, m.colorStart[ci], m.colorStart[ci + 1], (const int32_t *)w.luNbr,
                             (const int32_t *)w.luNLow, (const T *)w.luB, lay, zero ? rhs : (const T *)r, y);
            for (int ci = m.nColor - 1; ci >= 0; ci--)
                DNDSB_LAUNCH(ku, m.colorStart[ci + 1] - m.colorStart[ci], 128, st, m.colorStart[ci], m.colorStart[ci + 1], (const int32_t *)w.luNbr,
                             (const int32_t *)w.luNLow, (const T *)w.luB, lay, (const T *)w.luD, dlay, y);
            if (!zero)
                DNDSB_LAUNCH(k_add_T<T>, nn, 256, st, nn, (const T *)r, x);
        }
    }

    // doPrecondition (EulerSolver.hxx:1605-1635): forward then backward sweep; x in, x out (ping-pong through tmp2)
    void sgs_pair(const T *rhs, T *x, bool zeroIn) const
    {
        if (ls.jacobiCode == 2)
        {
            ilu_pair(rhs, x, zeroIn);
            return;
        }
        bool gs = ls.jacobiCode == 1;
        sweep(rhs, x, (T *)w.tmp2, true, gs, zeroIn);
        sweep(rhs, (T *)w.tmp2, x, false, gs, false);
    }

    // the GMRES preconditioner: MLx = (1 + sgsIter) SGS pairs from zero
    void FML(const T *b, T *MLx) const
    {
        for (int i = 0; i <= ls.sgsIter; i++)
            sgs_pair(b, MLx, i == 0);
    }

    // xs: the normalising factor of x when x is a stored Krylov column (nullptr: 1)
    void FA(const T *x, T *Ax, const real *xs = nullptr) const
    {
        if (w.jacMode)
        {
            auto kb = k_matvec_pos_blk<T, NV, NF>;
            DNDSB_LAUNCH(kb, m.nCell, 128, st, m.nCell, w.nbrPos, (const T *)w.opB, (const T *)w.jdB, x, Ax, xs);
            return;
        }
        auto kern = k_matvec_pos<T, NV, NF>;
        DNDSB_LAUNCH(kern, m.nCell, 128, st, m.nCell, w.nbrPos, (const T4 *)w.op, (const T *)w.jd, (const T *)w.uT, x,
                     Ax, gamma, xs);
    }

    void body() const
    {
        T *x = (T *)w.x;
        const T *b = (const T *)w.rhsT;
        int64_t nn = n();
        DNDSB_LAUNCH(k_zero_T<T>, nn, 256, st, nn, x);
        bool xZero = true;
        if (ls.gmresCode == 0 || ls.gmresCode == 2)
        {
            // solveLinear gmresCode 0/2 (EulerSolver.hxx:1462-1517): (1 + sgsIter) SGS pairs
            for (int i = 0; i <= ls.sgsIter; i++)
                sgs_pair(b, x, i == 0);
            xZero = false;
        }
        if (ls.gmresCode == 0)
            return;
        // GMRES_LeftPreconditioned::solve (Linear.hpp:46-133)
        int k = ls.nGmresSpace;
        T *MLb = (T *)w.MLb, *tmp = (T *)w.tmp;
        FML(b, MLb);
        krylov_norm(prec(), nn, NV, MLb, w.s2, w.red, w.sc + 0, w.cnt, st); // scale
        for (int r = 0; r < ls.nGmresIter; r++)
        {
            // V0 = M (A x) - M b; beta = |V0|; V0 = -V0 / beta
            if (xZero)
            {
                DNDSB_LAUNCH(k_copy_scalar, 1, 32, st, w.sc + 0, w.sc + 1);
                DNDSB_LAUNCH(k_gmres_v0<T>, nn, 256, st, nn, (const T *)nullptr, MLb, V(0), w.sc, 1);
            }
            else
            {
                FA(x, tmp);
                FML(tmp, V(0));
                krylov_diff_norm(prec(), nn, NV, V(0), MLb, w.s2, w.red, w.sc + 1, w.cnt, st);
                DNDSB_LAUNCH(k_gmres_v0<T>, nn, 256, st, nn, V(0), MLb, V(0), w.sc, 0);
            }
            DNDSB_LAUNCH(k_gmres_reset, 1, 32, st, w.sc, k, w.colScale);
            for (int j = 0; j < k; j++)
            {
                // the basis columns stay unnormalised: v_j = colScale[j] V(j), the factor applied by each reader
                FA(V(j), tmp, w.colScale + j);
                FML(tmp, V(j + 1));
                real *hcol = w.H + (int64_t)j * (k + 1);
                // classical Gram-Schmidt: h = V^T w, w -= V h, h[j+1] = |w|, colScale[j+1] = 1 / h[j+1]
                krylov_mdot(prec(), nn, ld(), NV, j + 1, w.V, V(j + 1), w.s2, w.red, hcol, w.colScale, w.cnt, st);
                krylov_maxpy_norm(prec(), nn, ld(), NV, j + 1, w.V, hcol, w.colScale, V(j + 1), w.s2, w.red, hcol + j + 1, w.cnt, w.sc, j,
                                  w.colScale + j + 1, st);
            }
            DNDSB_LAUNCH(k_gmres_lsq, 1, 32, st, k, w.H, w.sc, k, (real *)nullptr);
            DNDSB_LAUNCH(k_gmres_update<T>, nn, 256, st, nn, ld(), k, (const T *)w.V, w.sc, w.colScale, x);
            xZero = false;
        }
    }
    static int prec() { return sizeof(T) == 4 ? 1 : 0; }
};

template <typename T, int NV, int NF>
int run(const MeshD &m, const GeomD &g, const BoundaryD &bnd, EvalD &ev, LinWs &w, const LinSettings &ls, real alphaDiag, const real *dTau,
        real dt, const real *u, const real *rhs, real *xInc, cudaStream_t st)
{
    using T4 = typename Vec4<T>::type;
    // the caller's stream -> the solver's stream
    event_record(w.evIn, st);
    stream_wait(w.cs, w.evIn);
    cudaStream_t cs = w.cs;
    h2d(w.s2, ls.scale2, sizeof(real) * 8, cs);
    auto kbuild = k_sgsop_build<T, NV>;
    auto kgather = k_gather_T<T, NV>;
    auto kscatter = k_scatter_T<T, NV>;
    if (NV == 6 && !ev.jSource)
        return ST_BADARG;
    if (w.jacMode)
    {
        if (w.jacMode == 2 && (!ev.lambdaFace0 || (m.nBndFace > 0 && !bnd.type)))
            return ST_BADARG;
        auto kb = k_sgsop_build_blk<T, NV, NF>;
        DNDSB_LAUNCH(kb, m.nCell, 128, cs, m, g, bnd, ev, (int)(w.jacMode == 2), dTau, dt, alphaDiag, u, w.cellPos, w.nbrPos, (T *)w.opB,
                     (T *)w.jdB, ev.errWord);
        if (ls.jacobiCode == 2) // LUSGSMatrixToJacobianLU + InPlaceDecompose, colour by colour
        {
            auto kf = ilu::k_ilu_factor<T, NV, NF>;
            const ilu::BlockLay lay{NF * NV * NV, 5}, dlay{NV * NV, 5}, jlay{2 * NV * NV, 5};
            for (int ci = 0; ci < m.nColor; ci++)
                DNDSB_LAUNCH(kf, m.colorStart[ci + 1] - m.colorStart[ci], 64, cs, m.colorStart[ci], m.colorStart[ci + 1], (const int32_t *)nullptr,
                             w.nbrPos, (const int32_t *)nullptr, (const T *)w.opB, (const T *)w.jdB, lay, dlay, jlay, (T *)w.luB, (T *)w.luD,
                             ev.errWord, w.luNbr, w.luNLow);
        }
    }
    else
        DNDSB_LAUNCH(kbuild, m.nCell, 128, cs, m, g, ev.lambdaFace, dTau, dt, alphaDiag, u, ev.jSource, w.cellPos, w.nbrPos, (T4 *)w.op,
                     (T *)w.jd, (T *)w.uT);
    DNDSB_LAUNCH(kgather, m.nCell, 256, cs, m.nCell, m.colorCells, rhs, (T *)w.rhsT);
    Solve<T, NV, NF> S{m, w, ls, (T)ev.s.gamma, cs};
    if (ls.useGraph)
    {
        if (!(w.graph && w.keyValid && same_key(w.key, ls)))
        {
            graph_free(w.graph);
            w.graph = nullptr;
            w.keyValid = false;
            if (graph_begin(cs) == cudaSuccess)
            {
                S.body();
                if (graph_end(cs, &w.graph) != cudaSuccess)
                    w.graph = nullptr;
            }
            last_error();
        }
        if (w.graph)
        {
            w.key = ls, w.keyValid = true;
            if (graph_launch(w.graph, cs) != cudaSuccess)
                return ST_CUDA;
        }
        else
            S.body();
    }
    else
    {
        w.key = ls, w.keyValid = true;
        S.body();
    }
    DNDSB_LAUNCH(kscatter, m.nCell, 256, cs, m.nCell, m.colorCells, (const T *)w.x, xInc);
    event_record(w.evOut, cs);
    stream_wait(st, w.evOut);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

template <typename T, int NV>
int run_nf(const MeshD &m, const GeomD &g, const BoundaryD &bnd, EvalD &ev, LinWs &w, const LinSettings &ls, real alphaDiag, const real *dTau,
           real dt, const real *u, const real *rhs, real *xInc, cudaStream_t st)
{
    switch (m.nf)
    {
    case 3:
        return run<T, NV, 3>(m, g, bnd, ev, w, ls, alphaDiag, dTau, dt, u, rhs, xInc, st);
    case 4:
        return run<T, NV, 4>(m, g, bnd, ev, w, ls, alphaDiag, dTau, dt, u, rhs, xInc, st);
    case 6:
        return run<T, NV, 6>(m, g, bnd, ev, w, ls, alphaDiag, dTau, dt, u, rhs, xInc, st);
    }
    return ST_UNSUPPORTED;
}
} // namespace

int linear_solve(const MeshD &m, const GeomD &g, const BoundaryD &bnd, EvalD &ev, LinWs *&ws, const LinSettings &ls, real alphaDiag,
                 const real *dTau, real dt, const real *u, const real *rhs, real *xInc, cudaStream_t st)
{
    if (ls.gmresCode < 0 || ls.gmresCode > 2 || ls.jacobiCode < 0 || ls.jacobiCode > 2 || ls.sgsIter < 0 || ls.nGmresIter < 0 ||
        (ls.gmresCode && (ls.nGmresSpace < 1 || ls.nGmresSpace > 32)) || ls.precision < 0 || ls.precision > 1)
        return ST_BADARG;
    int nv = ev.s.nVars;
    // the local LU works on blocks: with the scalar Jacobian its diagonal blocks are the scalar diagonal and the
    // neighbour blocks the scalar form of the flux increment (LUSGSMatrixToJacobianLU takes JDiag.getValue), which is
    // the block operator without the Roe term
    const int mode = ev.jacMode ? ev.jacMode : (ls.jacobiCode == 2 ? 1 : 0);
    int rc = ws_prepare(m, ws, ls, nv, mode);
    if (rc != ST_OK)
        return rc;
    if (nv == 5)
        return ls.precision ? run_nf<float, 5>(m, g, bnd, ev, *ws, ls, alphaDiag, dTau, dt, u, rhs, xInc, st)
                            : run_nf<double, 5>(m, g, bnd, ev, *ws, ls, alphaDiag, dTau, dt, u, rhs, xInc, st);
    if (nv == 6)
        return ls.precision ? run_nf<float, 6>(m, g, bnd, ev, *ws, ls, alphaDiag, dTau, dt, u, rhs, xInc, st)
                            : run_nf<double, 6>(m, g, bnd, ev, *ws, ls, alphaDiag, dTau, dt, u, rhs, xInc, st);
    return ST_UNSUPPORTED;
}

// ---- caller-driven Arnoldi process: the same reductions for an operator applied outside the library ----
// work: [red: kRedBufLenK doubles][s2: 8 doubles][cnt]
size_t krylov_work_bytes() { return sizeof(real) * (kRedBufLenK + 8) + 64; }

namespace
{
struct KWork
{
    real *red, *s2;
    unsigned *cnt;
    explicit KWork(void *w) : red((real *)w), s2((real *)w + kRedBufLenK), cnt((unsigned *)((real *)w + kRedBufLenK + 8)) {}
};

template <typename T>
void kstart(int64_t n, int k, const void *r, void *V, real *gsc, real *colScale, void *work, cudaStream_t st)
{
    KWork kw(work);
    const int prec = sizeof(T) == 4 ? 1 : 0;
    DNDSB_LAUNCH(k_krylov_begin, 1, 32, st, kw.s2, kw.cnt, gsc, k, colScale);
    krylov_norm(prec, n, 5, r, kw.s2, kw.red, gsc + 1, kw.cnt, st);
    DNDSB_LAUNCH(k_krylov_scale, 1, 32, st, gsc);
    DNDSB_LAUNCH(k_gmres_v0<T>, n, 256, st, n, (const T *)nullptr, (const T *)r, (T *)V, gsc, 1);
}

template <typename T>
void kupdate(int64_t n, int k, const void *V, const real *gsc, const real *colScale, void *x, cudaStream_t st)
{
    DNDSB_LAUNCH(k_gmres_update<T>, n, 256, st, n, krylov_ld(n), k, (const T *)V, gsc, colScale, (T *)x);
}
} // namespace

int krylov_start(int prec, int64_t n, int k, const void *r, void *V, real *gsc, real *colScale, void *work, cudaStream_t st)
{
    if (n <= 0 || k < 1 || k > 32 || prec < 0 || prec > 1)
        return ST_BADARG;
    if (prec)
        kstart<float>(n, k, r, V, gsc, colScale, work, st);
    else
        kstart<double>(n, k, r, V, gsc, colScale, work, st);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int krylov_arnoldi(int prec, int64_t n, int j, int k, void *V, real *H, real *colScale, real *gsc, real *res, void *work, cudaStream_t st)
{
    if (n <= 0 || k < 1 || k > 32 || j < 0 || j >= k || prec < 0 || prec > 1)
        return ST_BADARG;
    KWork kw(work);
    const int64_t ld = krylov_ld(n);
    real *hcol = H + (int64_t)j * (k + 1);
    void *w = (char *)V + (int64_t)(j + 1) * ld * (prec ? 4 : 8);
    krylov_mdot(prec, n, ld, 5, j + 1, V, w, kw.s2, kw.red, hcol, colScale, kw.cnt, st);
    krylov_maxpy_norm(prec, n, ld, 5, j + 1, V, hcol, colScale, w, kw.s2, kw.red, hcol + j + 1, kw.cnt, gsc, j, colScale + j + 1, st);
    DNDSB_LAUNCH(k_gmres_lsq, 1, 32, st, k, H, gsc, j + 1, res);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int krylov_update(int prec, int64_t n, int k, const void *V, const real *gsc, const real *colScale, void *x, cudaStream_t st)
{
    if (n <= 0 || k < 1 || k > 32 || prec < 0 || prec > 1)
        return ST_BADARG;
    if (prec)
        kupdate<float>(n, k, V, gsc, colScale, x, st);
    else
        kupdate<double>(n, k, V, gsc, colScale, x, st);
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
