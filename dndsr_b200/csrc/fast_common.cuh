// Shared pieces of the Gauss-point-parallel face kernels (fast.cu, adjoint_fast.cu): the monomial exponent
// table, the shared-memory layout of a staged cell, the per-face data and the point reconstruction.
#pragma once
#include "solver.cuh"
#include "basis_eval.cuh"

namespace dndsb
{
namespace fastc
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

// per-face data shared by the Gauss points of a face (29 doubles: an odd stride in shared memory)
struct FaceData
{
    RoeAvg r;       // Roe averages of the two cell means
    real dLambda;   // max deltaLambdaCell of the two cells
    real db[3];     // barycentre difference, side 1 seen from side 0
    real gbase;     // 2 min(V0, V1) / A
    real shift[3];  // periodic translation into side 1's frame
    real pad;       // keeps the stride odd
};
static_assert(sizeof(FaceData) == 29 * sizeof(real), "FaceData layout");

// u + phi . uRec and the gradient D1 phi . uRec of one cell at point p (VariationalReconstruction.hpp:378-442 rows 0..dim)
// u + phi . uRec of one cell at point p, without the gradient
template <int DIM, int P, int NV>
DNDSB_D void recon_value(const real *cell, const real *p, real *U)
{
    using Lt = Layout<DIM, P, NV>;
    const real *rec = cell, *uu = cell + Lt::OU, *cent = cell + Lt::OC, *iL = cell + Lt::OL, *mom = cell + Lt::OM;
    real x = (p[0] - cent[0]) * iL[0], y = (p[1] - cent[1]) * iL[1], z = DIM == 3 ? (p[2] - cent[2]) * iL[2] : 0.0;
    real px[4] = {1, x, x * x, x * x * x}, py[4] = {1, y, y * y, y * y * y}, pz[4] = {1, z, z * z, z * z * z};
#pragma unroll
    for (int v = 0; v < NV; v++)
        U[v] = uu[v];
#pragma unroll
    for (int k = 1; k < Lt::NDOF; k++)
    {
        const int c = mcode(DIM, k);
        const real phi = px[c & 3] * py[(c >> 2) & 3] * pz[(c >> 4) & 3] - mom[k];
        const real *r = rec + (k - 1) * NV;
#pragma unroll
        for (int v = 0; v < NV; v++)
            U[v] += phi * r[v];
    }
}

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
} // namespace fastc
} // namespace dndsb
