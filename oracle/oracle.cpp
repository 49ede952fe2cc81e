// CPU oracle for the DNDSR implicit residual path -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++17 + OpenMP, the reference algorithms the
// GPU library implements, so that tests/, __graft_entry__.smoke() and the
// bench's CPU-baseline leg can check and time them.  Nothing in the product
// (dndsr_b200/) links, loads or calls this code.
//
// Parity pin: the reference cannot be compiled here (it needs Eigen, Boost,
// CGAL, HDF5, CGNS, Metis and MPI), so this restatement is pinned to the
// reference's own golden vectors that need no mesh file:
//   * Riemann fluxes  test/cpp/Euler/test_RiemannSolvers.cpp:242-294
//   * flux consistency/symmetry cases of the same file
//   * VR exactness / convergence properties (test_Reconstruction.cpp:454-506)
// Each function below cites the reference file:line it follows (paths are
// relative to the reference project root).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#ifdef ORC_OPCOUNT
#include "opcount.hpp"
#endif

namespace orc
{
#ifdef ORC_OPCOUNT
using real = orc_cnt::R; // the op-counting build (oracle/opcount.hpp)
#else
using real = double;
#endif
// unqualified math calls: the std overloads for double, the counting ones (found by argument-dependent
// lookup) in the op-counting build
using std::abs;
using std::cos;
using std::exp;
using std::floor;
using std::log;
using std::max;
using std::min;
using std::pow;
using std::round;
using std::sin;
using std::sqrt;
using std::tanh;
constexpr real verySmallReal = 1e-200; // DNDS/Defines.hpp:199
constexpr real smallReal = 1e-10;      // DNDS/Defines.hpp:201
constexpr real veryLargeReal = 3e200;  // DNDS/Defines.hpp:195
constexpr real pi = 3.14159265358979323846;
constexpr int INT_ORDER_MAX = 6; // Geom/Quadratures/QuadratureBase.hpp:70

enum Elem
{
    LINE2 = 0,
    TRI3 = 1,
    QUAD4 = 2,
    TET4 = 3,
    HEX8 = 4
};

static inline real sqr(real x) { return x * x; }
static inline real signTol(real a, real tol) { return a > tol ? 1 : (a < -tol ? -1 : 0); } // Defines.hpp:543
static inline real signP(real a) { return a >= 0 ? 1 : -1; }                              // Defines.hpp:549

// ---------------------------------------------------------------------------
// Quadrature: Geom/QuadratureHub.hpp:39-140 (scheme choice), Quadratures/*.hpp
// (tabulated points as the reference prints them).
// ---------------------------------------------------------------------------
static const real GL1[2][1] = {{0}, {2}};
static const real GL2[2][2] = {{-0.577350269189626, 0.577350269189626}, {1, 1}};
static const real GL3[2][3] = {{-0.774596669241483, 0, 0.774596669241483},
                               {0.555555555555555, 0.888888888888889, 0.555555555555555}};
static const real GL4[2][4] = {{-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053},
                               {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454}};

static const real Tri1[3][1] = {{1. / 3.}, {1. / 3.}, {1. / 2.}};
static const real Tri3[3][3] = {{2. / 3., 1. / 6., 1. / 6.}, {1. / 6., 2. / 3., 1. / 6.}, {1. / 6., 1. / 6., 1. / 6.}};
static const real Tri6[3][6] = {{0.09157621350977102, 0.8168475729804585, 0.09157621350977052, 0.445948490915965, 0.10810301816807, 0.445948490915965},
                                {0.09157621350977102, 0.09157621350977052, 0.8168475729804585, 0.445948490915965, 0.445948490915965, 0.10810301816807},
                                {0.054975871827661, 0.054975871827661, 0.054975871827661, 0.1116907948390057, 0.1116907948390057, 0.1116907948390057}};
static const real Tri7[3][7] = {{0.3333333333333335, 0.470142064105115, 0.05971587178977, 0.470142064105115, 0.1012865073234565, 0.7974269853530875, 0.1012865073234565},
                                {0.3333333333333335, 0.470142064105115, 0.470142064105115, 0.05971587178977, 0.1012865073234565, 0.1012865073234565, 0.7974269853530875},
                                {0.1125, 0.066197076394253, 0.066197076394253, 0.066197076394253, 0.0629695902724135, 0.0629695902724135, 0.0629695902724135}};
static const real Tri12[3][12] = {{0.2492867451709105, 0.501426509658179, 0.2492867451709105, 0.063089014491502, 0.8738219710169954, 0.063089014491502,
                                   0.3103524510337845, 0.05314504984481699, 0.6365024991213986, 0.05314504984481699, 0.6365024991213986, 0.3103524510337845},
                                  {0.2492867451709105, 0.2492867451709105, 0.501426509658179, 0.063089014491502, 0.063089014491502, 0.8738219710169954,
                                   0.05314504984481699, 0.3103524510337845, 0.05314504984481699, 0.6365024991213986, 0.3103524510337845, 0.6365024991213986},
                                  {0.05839313786318975, 0.05839313786318975, 0.05839313786318975, 0.0254224531851035, 0.0254224531851035, 0.0254224531851035,
                                   0.04142553780918675, 0.04142553780918675, 0.04142553780918675, 0.04142553780918675, 0.04142553780918675, 0.04142553780918675}};
static const real Tet1[4][1] = {{0.25}, {0.25}, {0.25}, {0.1666666666666667}};
static const real Tet4[4][4] = {{0.1381966011250105, 0.1381966011250105, 0.5854101966249685, 0.1381966011250105},
                                {0.1381966011250105, 0.5854101966249684, 0.1381966011250105, 0.1381966011250105},
                                {0.5854101966249684, 0.1381966011250105, 0.1381966011250105, 0.1381966011250105},
                                {0.04166666666666666, 0.04166666666666666, 0.04166666666666666, 0.04166666666666666}};
static const real Tet8[4][8] = {{0.1069940147705369, 0.1069940147705369, 0.6790179556883893, 0.1069940147705369, 0.3280585716625127, 0.3280585716625127, 0.01582428501246191, 0.3280585716625127},
                                {0.1069940147705369, 0.6790179556883893, 0.1069940147705369, 0.1069940147705369, 0.3280585716625127, 0.01582428501246191, 0.3280585716625127, 0.3280585716625127},
                                {0.6790179556883893, 0.1069940147705369, 0.1069940147705369, 0.1069940147705369, 0.01582428501246191, 0.3280585716625127, 0.3280585716625127, 0.3280585716625127},
                                {0.01859314997209119, 0.01859314997209119, 0.01859314997209119, 0.01859314997209119, 0.02307351669457548, 0.02307351669457548, 0.02307351669457548, 0.02307351669457548}};
static const real Tet14[4][14] = {{0.09273525031089125, 0.09273525031089125, 0.7217942490673263, 0.09273525031089125, 0.3108859192633008, 0.3108859192633008, 0.06734224221009777,
                                   0.3108859192633008, 0.04550370412564952, 0.4544962958743505, 0.04550370412564952, 0.04550370412564952, 0.4544962958743505, 0.4544962958743505},
                                  {0.09273525031089125, 0.7217942490673263, 0.09273525031089125, 0.09273525031089125, 0.3108859192633008, 0.06734224221009777, 0.3108859192633008,
                                   0.3108859192633008, 0.4544962958743505, 0.04550370412564952, 0.04550370412564952, 0.4544962958743505, 0.04550370412564952, 0.4544962958743505},
                                  {0.7217942490673263, 0.09273525031089125, 0.09273525031089125, 0.09273525031089125, 0.06734224221009777, 0.3108859192633008, 0.3108859192633008,
                                   0.3108859192633008, 0.4544962958743505, 0.4544962958743505, 0.4544962958743505, 0.04550370412564952, 0.04550370412564952, 0.04550370412564952},
                                  {0.01224884051939367, 0.01224884051939367, 0.01224884051939367, 0.01224884051939367, 0.01878132095300264, 0.01878132095300264, 0.01878132095300264,
                                   0.01878132095300264, 0.0070910034628469, 0.0070910034628469, 0.0070910034628469, 0.0070910034628469, 0.0070910034628469, 0.0070910034628469}};
static const real Tet24[4][24] = {{0.2146028712591523, 0.2146028712591523, 0.3561913862225431, 0.2146028712591523, 0.3223378901422754, 0.3223378901422754, 0.0329863295731736, 0.3223378901422754,
                                   0.04067395853461131, 0.04067395853461131, 0.8779781243961661, 0.04067395853461131, 0.6030056647916491, 0.6030056647916491, 0.06366100187501755, 0.2696723314583158,
                                   0.06366100187501755, 0.06366100187501755, 0.2696723314583158, 0.06366100187501755, 0.06366100187501755, 0.06366100187501755, 0.2696723314583158, 0.6030056647916491},
                                  {0.2146028712591523, 0.3561913862225431, 0.2146028712591523, 0.2146028712591523, 0.3223378901422754, 0.0329863295731736, 0.3223378901422754, 0.3223378901422754,
                                   0.04067395853461131, 0.8779781243961661, 0.04067395853461131, 0.04067395853461131, 0.06366100187501755, 0.06366100187501755, 0.06366100187501755, 0.6030056647916491,
                                   0.2696723314583158, 0.6030056647916491, 0.06366100187501755, 0.2696723314583158, 0.06366100187501755, 0.6030056647916491, 0.06366100187501755, 0.2696723314583158},
                                  {0.3561913862225431, 0.2146028712591523, 0.2146028712591523, 0.2146028712591523, 0.0329863295731736, 0.3223378901422754, 0.3223378901422754, 0.3223378901422754,
                                   0.8779781243961661, 0.04067395853461131, 0.04067395853461131, 0.04067395853461131, 0.2696723314583158, 0.06366100187501755, 0.6030056647916491, 0.06366100187501755,
                                   0.6030056647916491, 0.06366100187501755, 0.6030056647916491, 0.06366100187501755, 0.2696723314583158, 0.2696723314583158, 0.06366100187501755, 0.06366100187501755},
                                  {0.006653791709694545, 0.006653791709694545, 0.006653791709694545, 0.006653791709694545, 0.009226196923942479, 0.009226196923942479, 0.009226196923942479,
                                   0.009226196923942479, 0.001679535175886773, 0.001679535175886773, 0.001679535175886773, 0.001679535175886773, 0.008035714285714285, 0.008035714285714285,
                                   0.008035714285714285, 0.008035714285714285, 0.008035714285714285, 0.008035714285714285, 0.008035714285714285, 0.008035714285714285, 0.008035714285714285,
                                   0.008035714285714285, 0.008035714285714285, 0.008035714285714285}};

static int glSize(int order)
{
    if (order <= 1)
        return 1;
    if (order <= 3)
        return 2;
    if (order <= 5)
        return 3;
    return 4;
}

static const real *glData(int n, int row)
{
    switch (n)
    {
    case 1:
        return GL1[row];
    case 2:
        return GL2[row];
    case 3:
        return GL3[row];
    default:
        return GL4[row];
    }
}

// QuadratureHub.hpp:39-140
static int quadNPoints(int elem, int order)
{
    switch (elem)
    {
    case LINE2:
        return glSize(order);
    case QUAD4:
        return glSize(order) * glSize(order);
    case HEX8:
        return glSize(order) * glSize(order) * glSize(order);
    case TRI3:
        return order <= 1 ? 1 : order == 2 ? 3 : order <= 4 ? 6 : order == 5 ? 7 : 12;
    case TET4:
        return order <= 1 ? 1 : order == 2 ? 4 : order == 3 ? 8 : order <= 5 ? 14 : 24;
    }
    return 0;
}

// QuadratureHub.hpp:188-380
static void quadPoint(int elem, int order, int iG, real p[3], real &w)
{
    p[0] = p[1] = p[2] = 0;
    if (elem == LINE2 || elem == QUAD4 || elem == HEX8)
    {
        int n = glSize(order);
        const real *x = glData(n, 0), *wt = glData(n, 1);
        if (elem == LINE2)
        {
            p[0] = x[iG];
            w = wt[iG];
        }
        else if (elem == QUAD4)
        {
            int i = iG % n, j = iG / n;
            p[0] = x[i], p[1] = x[j];
            w = wt[i] * wt[j];
        }
        else
        {
            int i = iG % n, j = (iG / n) % n, k = iG / (n * n);
            p[0] = x[i], p[1] = x[j], p[2] = x[k];
            w = wt[i] * wt[j] * wt[k];
        }
        return;
    }
    int np = quadNPoints(elem, order);
    if (elem == TRI3)
    {
        const real *t = nullptr;
        switch (np)
        {
        case 1:
            p[0] = Tri1[0][iG], p[1] = Tri1[1][iG], w = Tri1[2][iG];
            return;
        case 3:
            p[0] = Tri3[0][iG], p[1] = Tri3[1][iG], w = Tri3[2][iG];
            return;
        case 6:
            p[0] = Tri6[0][iG], p[1] = Tri6[1][iG], w = Tri6[2][iG];
            return;
        case 7:
            p[0] = Tri7[0][iG], p[1] = Tri7[1][iG], w = Tri7[2][iG];
            return;
        default:
            p[0] = Tri12[0][iG], p[1] = Tri12[1][iG], w = Tri12[2][iG];
            (void)t;
            return;
        }
    }
    switch (np)
    {
    case 1:
        p[0] = Tet1[0][iG], p[1] = Tet1[1][iG], p[2] = Tet1[2][iG], w = Tet1[3][iG];
        return;
    case 4:
        p[0] = Tet4[0][iG], p[1] = Tet4[1][iG], p[2] = Tet4[2][iG], w = Tet4[3][iG];
        return;
    case 8:
        p[0] = Tet8[0][iG], p[1] = Tet8[1][iG], p[2] = Tet8[2][iG], w = Tet8[3][iG];
        return;
    case 14:
        p[0] = Tet14[0][iG], p[1] = Tet14[1][iG], p[2] = Tet14[2][iG], w = Tet14[3][iG];
        return;
    default:
        p[0] = Tet24[0][iG], p[1] = Tet24[1][iG], p[2] = Tet24[2][iG], w = Tet24[3][iG];
        return;
    }
}

static int elemNNode(int elem)
{
    static const int n[] = {2, 3, 4, 4, 8};
    return n[elem];
}

// Shape functions N and dN/dxi (Geom/Elements/{Line2,Tri3,Quad4,Tet4,Hex8}.hpp)
static void shapeD01(int elem, const real p[3], real N[8], real dN[3][8])
{
    real xi = p[0], et = p[1], zt = p[2];
    for (int d = 0; d < 3; d++)
        for (int i = 0; i < 8; i++)
            dN[d][i] = 0;
    switch (elem)
    {
    case LINE2:
        N[0] = 0.5 - 0.5 * xi, N[1] = 0.5 * xi + 0.5;
        dN[0][0] = -0.5, dN[0][1] = 0.5;
        break;
    case TRI3:
        N[0] = 1 - xi - et, N[1] = xi, N[2] = et;
        dN[0][0] = -1, dN[0][1] = 1;
        dN[1][0] = -1, dN[1][2] = 1;
        break;
    case QUAD4:
    {
        real t1 = 0.25 * et - 0.25, t3 = 0.25 * et + 0.25;
        N[0] = (xi - 1) * t1, N[1] = -t1 * (xi + 1), N[2] = (xi + 1) * t3, N[3] = -(xi - 1) * t3;
        real a = 0.25 * xi - 0.25, b = 0.25 * xi + 0.25;
        dN[0][0] = t1, dN[0][1] = -t1, dN[0][2] = t3, dN[0][3] = -t3;
        dN[1][0] = a, dN[1][1] = -b, dN[1][2] = b, dN[1][3] = -a;
        break;
    }
    case TET4:
        N[0] = 1 - xi - et - zt, N[1] = xi, N[2] = et, N[3] = zt;
        dN[0][0] = -1, dN[0][1] = 1;
        dN[1][0] = -1, dN[1][2] = 1;
        dN[2][0] = -1, dN[2][3] = 1;
        break;
    case HEX8:
    {
        static const int s[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1}};
        for (int i = 0; i < 8; i++)
        {
            real a = 1 + s[i][0] * xi, b = 1 + s[i][1] * et, c = 1 + s[i][2] * zt;
            N[i] = 0.125 * a * b * c;
            dN[0][i] = 0.125 * s[i][0] * b * c;
            dN[1][i] = 0.125 * a * s[i][1] * c;
            dN[2][i] = 0.125 * a * b * s[i][2];
        }
        break;
    }
    }
}

struct PointGeo
{
    real x[3];
    real J[3][3]; // J[r][c] = d x_r / d xi_c
};

static PointGeo pointGeo(int elem, const real *coords /*nn x 3*/, const real p[3])
{
    real N[8], dN[3][8];
    shapeD01(elem, p, N, dN);
    PointGeo g{};
    int nn = elemNNode(elem);
    for (int r = 0; r < 3; r++)
    {
        g.x[r] = 0;
        for (int i = 0; i < nn; i++)
            g.x[r] += coords[i * 3 + r] * N[i];
        for (int c = 0; c < 3; c++)
        {
            g.J[r][c] = 0;
            for (int i = 0; i < nn; i++)
                g.J[r][c] += coords[i * 3 + r] * dN[c][i];
        }
    }
    return g;
}

static void cross(const real a[3], const real b[3], real c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static real norm3(const real a[3]) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
static real dot3(const real a[3], const real b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Geom/Quadrature.hpp:480-490
static real cellJacDet(int dim, const PointGeo &g)
{
    if (dim == 2)
    {
        real a[3] = {g.J[0][0], g.J[1][0], g.J[2][0]}, b[3] = {g.J[0][1], g.J[1][1], g.J[2][1]}, c[3];
        cross(a, b, c);
        return norm3(c);
    }
    const auto &J = g.J;
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

// Geom/Quadrature.hpp:500-511 and Geom/Geometric.hpp:113-128
static real faceJDetNorm(int dim, const PointGeo &g, real n[3])
{
    real a[3] = {g.J[0][0], g.J[1][0], g.J[2][0]};
    if (dim == 2)
    {
        n[0] = a[1], n[1] = -a[0], n[2] = 0;
        return norm3(a);
    }
    real b[3] = {g.J[0][1], g.J[1][1], g.J[2][1]};
    cross(a, b, n);
    return norm3(n);
}

// ---------------------------------------------------------------------------
// Polynomial basis: Geom/BaseFunction.hpp:55-79 (3D order list), :96-107 (2D),
// :239-279 (factorials/comb counts), :285-700 (FPolynomialFill2D/3D)
// ---------------------------------------------------------------------------
static const int dOrder3[20][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1},
                                   {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {1, 2, 0}, {0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {2, 0, 1}, {1, 1, 1}};
static const int dOrder2[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {3, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 3, 0}};
static const int dFact[4][4] = {{1, 0, 0, 0}, {1, 1, 0, 0}, {1, 2, 2, 0}, {1, 3, 6, 6}};
static const int nComb2[10] = {1, 1, 1, 1, 2, 1, 1, 3, 3, 1};
static const int nComb3[20] = {1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 3, 3, 3, 3, 3, 3, 6};
static const int factorials[10] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880};

static real iPow(int p, real x)
{
    switch (p)
    {
    case 0:
        return 1.;
    case 1:
        return x;
    case 2:
        return x * x;
    case 3:
        return x * x * x;
    }
    return 1e300;
}

static int nDofOf(int dim, int order)
{
    static const int n2[] = {1, 3, 6, 10}, n3[] = {1, 4, 10, 20};
    return dim == 2 ? n2[order] : n3[order];
}

// fills T[rows][cols] (row-major, cols = NDOF)
static void polyFill(int dim, real *T, real x, real y, real z, real lx, real ly, real lz, int rows, int cols)
{
    for (int idiff = 0; idiff < rows; idiff++)
        for (int ib = 0; ib < cols; ib++)
        {
            const int *pb = dim == 2 ? dOrder2[ib] : dOrder3[ib];
            const int *pd = dim == 2 ? dOrder2[idiff] : dOrder3[idiff];
            int c = dFact[pb[0]][pd[0]] * dFact[pb[1]][pd[1]] * dFact[pb[2]][pd[2]];
            real v = c ? c * iPow(pb[0] - pd[0], x) * iPow(pb[1] - pd[1], y) * iPow(pb[2] - pd[2], z) : 0.;
            real l = iPow(pd[0], lx) * iPow(pd[1], ly) * iPow(pd[2], dim == 2 ? 1.0 : lz);
            T[idiff * cols + ib] = v / l;
        }
}

// ---------------------------------------------------------------------------
// Gas thermodynamics and Riemann solvers: Euler/Gas.hpp, DNDS/IdealGasPhysics.hpp
// Physical dimension is always 3 (models NS / NS_3D / NS_SA / NS_SA_3D).
// ---------------------------------------------------------------------------
constexpr int D = 3;

// IdealGasPhysics.hpp:38-44
static void idealGasThermal(real E, real rho, real vSqr, real gamma, real &p, real &asqr, real &H)
{
    p = (gamma - 1) * (E - rho * 0.5 * vSqr);
    asqr = gamma * p / rho;
    H = (E + p) / rho;
}

struct RoePre
{
    real veloLm[3], veloRm[3], asqrLm, asqrRm, pLm, pRm, HLm, HRm, vsqrLm, vsqrRm;
    real veloRoe[3], sqrtRhoLm, sqrtRhoRm, vsqrRoe, HRoe, asqrRoe, rhoRoe, aRoe;
};

// Gas.hpp:229-259
static RoePre roePreamble(const real *ULm, const real *URm, real gamma)
{
    RoePre r{};
    for (int d = 0; d < 3; d++)
        r.veloLm[d] = ULm[1 + d] / ULm[0], r.veloRm[d] = URm[1 + d] / URm[0];
    r.vsqrLm = dot3(r.veloLm, r.veloLm);
    r.vsqrRm = dot3(r.veloRm, r.veloRm);
    idealGasThermal(ULm[4], ULm[0], r.vsqrLm, gamma, r.pLm, r.asqrLm, r.HLm);
    idealGasThermal(URm[4], URm[0], r.vsqrRm, gamma, r.pRm, r.asqrRm, r.HRm);
    r.sqrtRhoLm = sqrt(ULm[0]);
    r.sqrtRhoRm = sqrt(URm[0]);
    for (int d = 0; d < 3; d++)
        r.veloRoe[d] = (r.sqrtRhoLm * r.veloLm[d] + r.sqrtRhoRm * r.veloRm[d]) / (r.sqrtRhoLm + r.sqrtRhoRm);
    r.vsqrRoe = dot3(r.veloRoe, r.veloRoe);
    r.HRoe = (r.sqrtRhoLm * r.HLm + r.sqrtRhoRm * r.HRm) / (r.sqrtRhoLm + r.sqrtRhoRm);
    r.asqrRoe = (gamma - 1) * (r.HRoe - 0.5 * r.vsqrRoe);
    r.rhoRoe = r.sqrtRhoLm * r.sqrtRhoRm;
    r.aRoe = sqrt(r.asqrRoe);
    return r;
}

// Gas.hpp:390-397 GasInviscidFlux_XY
static void inviscidFluxXY(const real *U, const real velo[3], const real vg[3], const real n[3], real p, real F[5])
{
    real vrel[3] = {velo[0] - vg[0], velo[1] - vg[1], velo[2] - vg[2]};
    real vn = dot3(vrel, n);
    for (int i = 0; i < 5; i++)
        F[i] = U[i] * vn;
    for (int d = 0; d < 3; d++)
        F[1 + d] += p * n[d];
    F[4] += dot3(velo, n) * p;
}

// Gas.hpp:878-1007 Roe_EntropyFixer
static void roeEntropyFix(int eigScheme, real aL, real aR, real aAve, real uL, real uR, real uAve, real VL, real VR, real VAve,
                          real dLambda, real fixScale, real incFScale, real &lam0, real &lam123, real &lam4)
{
    const real scaleHartenYee = 0.05 * fixScale, scaleLD = 0.2 * fixScale, scaleHFix = 0.25 * fixScale;
    const real incFScaleA = 1.0;
    (void)VL, (void)VR;
    if (eigScheme == 0)
    {
        auto Flim = [=](real v, real lam, real lamL, real lamR)
        {
            const real thresH = max({real(0.), lam - lamL, lamR - lam}) * scaleHartenYee;
            if (v < thresH)
                return (sqr(v) / thresH + thresH) * 0.5;
            return v;
        };
        lam0 = Flim(lam0 * incFScaleA, uAve - aAve, uL - aL, uR - aR);
        lam123 = Flim(lam123 * incFScale, uAve, uL, uR);
        lam4 = Flim(lam4 * incFScaleA, uAve + aAve, uL + aL, uR + aR);
    }
    else if (eigScheme == 1)
    {
        const real aLm = aL * incFScaleA, aRm = aR * incFScaleA;
        const real uLm = signTol(uL, aLm * smallReal) * max(abs(uL) * incFScale, aLm * scaleLD);
        const real uRm = signTol(uR, aRm * smallReal) * max(abs(uR) * incFScale, aRm * scaleLD);
        lam0 = max(abs(uLm - aLm), abs(uRm - aRm));
        lam123 = max(abs(uLm), abs(uRm));
        lam4 = max(abs(uLm + aLm), abs(uRm + aRm));
    }
    else if (eigScheme == 3)
    {
        const real LDthreshold = abs(uAve) / scaleLD;
        const real aRoeStar = min(LDthreshold, aAve * incFScaleA);
        lam0 = abs(uAve * incFScale - aRoeStar);
        lam4 = abs(uAve * incFScale + aRoeStar);
    }
    else if (eigScheme == 4)
    {
        const real uStar = signTol(uAve, aAve * smallReal) * max(aAve * scaleLD, abs(uAve) * incFScale);
        lam0 = abs(uStar - aAve * incFScaleA);
        lam123 = abs(uStar);
        lam4 = abs(uStar + aAve * incFScaleA);
    }
    else if (eigScheme == 5)
    {
        const real vL = uL * incFScale, vR = uR * incFScale;
        const real aLm = min(aL * incFScaleA, abs(vL) / scaleLD);
        const real aRm = min(aR * incFScaleA, abs(vR) / scaleLD);
        lam0 = max(abs(vL - aLm), abs(vR - aRm));
        lam123 = max(abs(vL), abs(vR));
        lam4 = max(abs(vL + aLm), abs(vR + aRm));
    }
    else if (eigScheme == 6)
    {
        lam0 = max(abs(uAve * incFScale - aAve * incFScaleA), dLambda * scaleHFix);
        lam4 = max(abs(uAve * incFScale + aAve * incFScaleA), dLambda * scaleHFix);
        lam123 = max(abs(uAve * incFScale), dLambda * scaleHFix);
    }
    else if (eigScheme == 7 || eigScheme == 8)
    {
        if (eigScheme == 7)
        {
            lam0 *= abs(uAve * incFScale - aAve * incFScaleA);
            lam4 *= abs(uAve * incFScale + aAve * incFScaleA);
            lam123 *= abs(uAve * incFScale);
        }
        else
        {
            lam0 = max(abs(uAve * incFScale - aAve * incFScaleA), dLambda * scaleHFix);
            lam4 = max(abs(uAve * incFScale + aAve * incFScaleA), dLambda * scaleHFix);
            lam123 = max(abs(uAve * incFScale), dLambda * scaleHFix);
        }
        const real th = scaleHartenYee * (VAve + aAve), thS = sqr(th);
        if (lam0 < th)
            lam0 = (sqr(lam0) + thS) / (2 * th);
        if (lam4 < th)
            lam4 = (sqr(lam4) + thS) / (2 * th);
        if (lam123 < th)
            lam123 = (sqr(lam123) + thS) / (2 * th);
    }
}

// Gas.hpp:1038-1126 RoeFlux_IdealGas_HartenYee
// nE: the normal of the eigenvalues and of the Roe normal velocity.  The per-point flux passes nE = n; the
// batched flux of Gas.hpp:1272-1408 (RoeFlux_IdealGas_HartenYee_Batch, rsMeanValueEig = 1) passes the face's
// mean normal while the physical fluxes, the jump projections and the acoustic eigenvectors keep the point normal
static void roeFlux(int eigScheme, const real *UL, const real *UR, const real *ULm, const real *URm, const real vg[3], const real n[3],
                    const real nE[3], real gamma, real F[5], real dLambda, real fixScale, real incFScale, real &lam0, real &lam123,
                    real &lam4)
{
    real veloL[3], veloR[3];
    for (int d = 0; d < 3; d++)
        veloL[d] = UL[1 + d] / UL[0], veloR[d] = UR[1 + d] / UR[0];
    real asqrL, asqrR, pL, pR, HL, HR;
    idealGasThermal(UL[4], UL[0], dot3(veloL, veloL), gamma, pL, asqrL, HL);
    idealGasThermal(UR[4], UR[0], dot3(veloR, veloR), gamma, pR, asqrR, HR);
    RoePre rp = roePreamble(ULm, URm, gamma);
    real FL[5], FR[5];
    inviscidFluxXY(UL, veloL, vg, n, pL, FL);
    inviscidFluxXY(UR, veloR, vg, n, pR, FR);
    real veloRoeN = dot3(rp.veloRoe, nE), vgN = dot3(vg, nE);
    real veloRoe0 = veloRoeN - vgN;
    lam0 = abs(veloRoe0 - rp.aRoe);
    lam123 = abs(veloRoe0);
    lam4 = abs(veloRoe0 + rp.aRoe);
    real dvL[3], dvR[3], dvRoe[3];
    for (int d = 0; d < 3; d++)
        dvL[d] = rp.veloLm[d] - vg[d], dvR[d] = rp.veloRm[d] - vg[d], dvRoe[d] = rp.veloRoe[d] - vg[d];
    real veloLm0 = dot3(dvL, nE), veloRm0 = dot3(dvR, nE);
    if (eigScheme == 2)
    {
        lam0 = lam123 = lam4 = max(abs(veloLm0) + sqrt(rp.asqrLm), abs(veloRm0) + sqrt(rp.asqrRm));
        for (int i = 0; i < 5; i++)
            F[i] = (FL[i] + FR[i]) * 0.5 - 0.5 * lam0 * (UR[i] - UL[i]);
        return;
    }
    roeEntropyFix(eigScheme, sqrt(rp.asqrLm), sqrt(rp.asqrRm), rp.aRoe, veloLm0, veloRm0, veloRoe0,
                  norm3(dvL), norm3(dvR), norm3(dvRoe), dLambda, fixScale, incFScale, lam0, lam123, lam4);
    real incU[5];
    for (int i = 0; i < 5; i++)
        incU[i] = UR[i] - UL[i];
    real incU123N = incU[1] * n[0] + incU[2] * n[1] + incU[3] * n[2];
    real a23[3];
    for (int d = 0; d < 3; d++)
        a23[d] = incU[1 + d] - incU[0] * rp.veloRoe[d];
    real a23n = dot3(a23, n);
    real a23T[3];
    for (int d = 0; d < 3; d++)
        a23T[d] = a23[d] - n[d] * a23n;
    real incU4b = incU[4] - dot3(a23T, rp.veloRoe);
    real alpha1 = (gamma - 1) / rp.asqrRoe * (incU[0] * (rp.HRoe - veloRoeN * veloRoeN) + veloRoeN * incU123N - incU4b);
    real alpha0 = (incU[0] * (veloRoeN + rp.aRoe) - incU123N - rp.aRoe * alpha1) / (2 * rp.aRoe);
    real alpha4 = incU[0] - (alpha0 + alpha1);
    alpha0 *= lam0;
    alpha1 *= lam123;
    for (int d = 0; d < 3; d++)
        a23T[d] *= lam123;
    alpha4 *= lam4;
    real incF[5];
    incF[0] = alpha0 + alpha1 + alpha4;
    incF[4] = (rp.HRoe - veloRoeN * rp.aRoe) * alpha0 + 0.5 * rp.vsqrRoe * alpha1 + (rp.HRoe + veloRoeN * rp.aRoe) * alpha4 + dot3(a23T, rp.veloRoe);
    for (int d = 0; d < 3; d++)
        incF[1 + d] = (rp.veloRoe[d] - rp.aRoe * n[d]) * alpha0 + (rp.veloRoe[d] + rp.aRoe * n[d]) * alpha4 + rp.veloRoe[d] * alpha1 + a23T[d];
    for (int i = 0; i < 5; i++)
        F[i] = (FL[i] + FR[i]) * 0.5 - 0.5 * incF[i];
}

// Gas.hpp:601-714 HLLEPFlux_IdealGas
static void hllepFlux(int type, const real *UL, const real *UR, const real *ULm, const real *URm, const real vg[3], const real n[3],
                      real gamma, real F[5], real dLambda, real fixScale, real &lam0, real &lam123, real &lam4)
{
    real veloL[3], veloR[3];
    for (int d = 0; d < 3; d++)
        veloL[d] = UL[1 + d] / UL[0], veloR[d] = UR[1 + d] / UR[0];
    real asqrL, asqrR, pL, pR, HL, HR;
    idealGasThermal(UL[4], UL[0], dot3(veloL, veloL), gamma, pL, asqrL, HL);
    idealGasThermal(UR[4], UR[0], dot3(veloR, veloR), gamma, pR, asqrR, HR);
    RoePre rp = roePreamble(ULm, URm, gamma);
    real FL[5], FR[5];
    inviscidFluxXY(UL, veloL, vg, n, pL, FL);
    inviscidFluxXY(UR, veloR, vg, n, pR, FR);
    real veloRoeN = dot3(rp.veloRoe, n), vgN = dot3(vg, n);
    real veloRoe0 = veloRoeN - vgN;
    lam0 = abs(veloRoe0 - rp.aRoe);
    lam123 = abs(veloRoe0);
    lam4 = abs(veloRoe0 + rp.aRoe);
    real dvL[3], dvR[3];
    for (int d = 0; d < 3; d++)
        dvL[d] = rp.veloLm[d] - vg[d], dvR[d] = rp.veloRm[d] - vg[d];
    real veloLm0 = dot3(dvL, n), veloRm0 = dot3(dvR, n);
    real incU[5];
    for (int i = 0; i < 5; i++)
        incU[i] = UR[i] - UL[i];
    real incU123N = incU[1] * n[0] + incU[2] * n[1] + incU[3] * n[2];
    real a23[3];
    for (int d = 0; d < 3; d++)
        a23[d] = incU[1 + d] - incU[0] * rp.veloRoe[d];
    real a23n = dot3(a23, n);
    real a23T[3];
    for (int d = 0; d < 3; d++)
        a23T[d] = a23[d] - n[d] * a23n;
    real incU4b = incU[4] - dot3(a23T, rp.veloRoe);
    real alpha1 = (gamma - 1) / rp.asqrRoe * (incU[0] * (rp.HRoe - veloRoeN * veloRoeN) + veloRoeN * incU123N - incU4b);
    real alpha0 = (incU[0] * (veloRoeN + rp.aRoe) - incU123N - rp.aRoe * alpha1) / (2 * rp.aRoe);
    real alpha4 = incU[0] - (alpha0 + alpha1);
    real SL = min(veloRoe0 - rp.aRoe, veloLm0 - sqrt(asqrL));
    real SR = max(veloRoe0 + rp.aRoe, veloRm0 + sqrt(asqrR));
    real UU = abs(veloRoe0);
    real dfix = rp.aRoe / (rp.aRoe + max(UU, dLambda * fixScale));
    real SP = max(SR, 0.0), SM = min(SL, 0.0);
    if (type != 1)
    {
        real ReV1[5] = {1, rp.veloRoe[0], rp.veloRoe[1], rp.veloRoe[2], rp.vsqrRoe * 0.5};
        real div = SP - SM;
        div += signP(div) * verySmallReal;
        for (int i = 0; i < 5; i++)
            F[i] = (SP * FL[i] - SM * FR[i]) / div + (SP * SM / div) * (UR[i] - UL[i] - dfix * ReV1[i] * alpha1);
    }
    else
    {
        real delta1 = dfix, delta2 = 0.0, delta3 = 0.0;
        lam123 = ((SP + SM) * (veloRoe0)-2.0 * (1.0 - delta1) * (SP * SM)) / (SP - SM);
        lam4 = ((SP + SM) * (veloRoe0 + rp.aRoe) - 2.0 * (1.0 - delta2) * (SP * SM)) / (SP - SM);
        lam0 = ((SP + SM) * (veloRoe0 - rp.aRoe) - 2.0 * (1.0 - delta3) * (SP * SM)) / (SP - SM);
        lam123 = abs(lam123), lam0 = abs(lam0), lam4 = abs(lam4);
        alpha0 *= lam0;
        alpha1 *= lam123;
        for (int d = 0; d < 3; d++)
            a23T[d] *= lam123;
        alpha4 *= lam4;
        real incF[5];
        incF[0] = alpha0 + alpha1 + alpha4;
        incF[4] = (rp.HRoe - veloRoeN * rp.aRoe) * alpha0 + 0.5 * rp.vsqrRoe * alpha1 + (rp.HRoe + veloRoeN * rp.aRoe) * alpha4 + dot3(a23T, rp.veloRoe);
        for (int d = 0; d < 3; d++)
            incF[1 + d] = (rp.veloRoe[d] - rp.aRoe * n[d]) * alpha0 + (rp.veloRoe[d] + rp.aRoe * n[d]) * alpha4 + rp.veloRoe[d] * alpha1 + a23T[d];
        for (int i = 0; i < 5; i++)
            F[i] = (FL[i] + FR[i]) * 0.5 - 0.5 * incF[i];
    }
}

// Gas.hpp:737-~860 HLLCFlux_IdealGas_HartenYee
static void hllcFlux(const real *UL, const real *UR, const real *ULm, const real *URm, const real vg[3], const real n[3],
                     real gamma, real F[5], real dLambda, real &lam0, real &lam123, real &lam4)
{
    real veloL[3], veloR[3];
    for (int d = 0; d < 3; d++)
        veloL[d] = UL[1 + d] / UL[0], veloR[d] = UR[1 + d] / UR[0];
    real asqrL, asqrR, pL, pR, HL, HR;
    idealGasThermal(UL[4], UL[0], dot3(veloL, veloL), gamma, pL, asqrL, HL);
    idealGasThermal(UR[4], UR[0], dot3(veloR, veloR), gamma, pR, asqrR, HR);
    RoePre rp = roePreamble(ULm, URm, gamma);
    real FL[5], FR[5];
    inviscidFluxXY(UL, veloL, vg, n, pL, FL);
    inviscidFluxXY(UR, veloR, vg, n, pR, FR);
    real veloRoeN = dot3(rp.veloRoe, n), vgN = dot3(vg, n);
    real veloRoe0 = veloRoeN - vgN;
    lam0 = abs(veloRoe0 - rp.aRoe);
    lam123 = abs(veloRoe0);
    lam4 = abs(veloRoe0 + rp.aRoe);
    real dvL[3], dvR[3];
    for (int d = 0; d < 3; d++)
        dvL[d] = rp.veloLm[d] - vg[d], dvR[d] = rp.veloRm[d] - vg[d];
    real veloLm0 = dot3(dvL, n), veloRm0 = dot3(dvR, n);
    auto HLLCq = [&](real p, real pS)
    {
        real q = sqrt(1 + (gamma + 1) / 2 / gamma * (pS / p - 1));
        if (pS <= p)
            q = 1;
        return q;
    };
    real pS = 0.5 * (rp.pLm + rp.pRm) - 0.5 * (veloLm0 - veloRm0) * rp.rhoRoe * rp.aRoe;
    pS = max(0.0, pS);
    real SL = veloLm0 - sqrt(rp.asqrLm) * HLLCq(rp.pLm, pS);
    real SR = veloRm0 + sqrt(rp.asqrRm) * HLLCq(rp.pRm, pS);
    (void)dLambda;
    if (0 <= SL)
    {
        std::copy(FL, FL + 5, F);
        return;
    }
    if (SR <= 0)
    {
        std::copy(FR, FR + 5, F);
        return;
    }
    real SS = 0;
    real div = (UL[0] * (SL - veloLm0) - UR[0] * (SR - veloRm0));
    real ULn = UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2], URn = UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2];
    if (abs(div) > verySmallReal)
        SS = (pR - pL + (ULn - vgN * UL[0]) * (SL - veloLm0) - (URn - vgN * UR[0]) * (SR - veloRm0)) / div;
    real DS[5] = {0, n[0], n[1], n[2], SS};
    if (SS >= 0)
    {
        real dv = SL - SS;
        if (abs(dv) < verySmallReal)
            std::copy(FL, FL + 5, F);
        else
            for (int i = 0; i < 5; i++)
                F[i] = ((UL[i] * SL - FL[i]) * SS + DS[i] * ((pL + UL[0] * (SL - veloLm0) * (SS - veloLm0)) * SL)) / dv;
    }
    else
    {
        real dv = SR - SS;
        if (abs(dv) < verySmallReal)
            std::copy(FR, FR + 5, F);
        else
            for (int i = 0; i < 5; i++)
                F[i] = ((UR[i] * SR - FR[i]) * SS + DS[i] * ((pR + UR[0] * (SR - veloRm0) * (SS - veloRm0)) * SR)) / dv;
    }
}

// Riemann solver codes follow Gas.hpp:61-96 RiemannSolverType
enum RS
{
    RS_Roe = 1,
    RS_HLLC = 2,
    RS_HLLEP = 3,
    RS_HLLEP_V1 = 21,
    RS_Roe_M1 = 11,
    RS_Roe_M8 = 18
};

// Gas.hpp:1434-1490 InviscidFlux_IdealGas_Dispatcher
// nMean: the face's mean normal when the settings ask for the batched mean-value eigenvalues
// (EulerEvaluator_EvaluateDt.hxx:1259-1270: rsMeanValueEig != 0 and Roe_M1..Roe_M5), else nullptr
static void riemann(int type, const real *UL, const real *UR, const real *ULm, const real *URm, const real vg[3], const real n[3], real gamma,
                    real F[5], real dLambda, real fixScale, real incFScale, real &lam0, real &lam123, real &lam4,
                    const real *nMean = nullptr)
{
    const real *nE = (nMean && type >= 11 && type <= 15) ? nMean : n;
    if (type == RS_Roe)
        roeFlux(0, UL, UR, ULm, URm, vg, n, n, gamma, F, dLambda, fixScale, incFScale, lam0, lam123, lam4);
    else if (type >= 11 && type <= 18)
        roeFlux(type - 10, UL, UR, ULm, URm, vg, n, nE, gamma, F, dLambda, fixScale, incFScale, lam0, lam123, lam4);
    else if (type == RS_HLLEP)
        hllepFlux(0, UL, UR, ULm, URm, vg, n, gamma, F, dLambda, fixScale, lam0, lam123, lam4);
    else if (type == RS_HLLEP_V1)
        hllepFlux(1, UL, UR, ULm, URm, vg, n, gamma, F, dLambda, fixScale, lam0, lam123, lam4);
    else if (type == RS_HLLC)
        hllcFlux(UL, UR, ULm, URm, vg, n, gamma, F, dLambda, lam0, lam123, lam4);
}

// Gas.hpp:1677-1698 GradientCons2Prim_IdealGas; G is [3][nv]
static void gradCons2Prim(int nv, const real *U, const real *G, real *GP, real gamma)
{
    real velo[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
    for (int i = 0; i < 3 * nv; i++)
        GP[i] = G[i];
    for (int r = 0; r < 3; r++)
        for (int j = 0; j < 3; j++)
            GP[r * nv + 1 + j] = (1.0 / sqr(U[0])) * (U[0] * G[r * nv + 1 + j] - G[r * nv + 0] * U[1 + j]);
    for (int r = 0; r < 3; r++)
    {
        real s = 0;
        for (int j = 0; j < 3; j++)
            s += G[r * nv + 1 + j] * velo[j] + GP[r * nv + 1 + j] * U[1 + j];
        GP[r * nv + 4] = (gamma - 1) * (G[r * nv + 4] - 0.5 * s);
    }
    for (int r = 0; r < 3; r++)
        for (int j = 5; j < nv; j++)
        {
            GP[r * nv + j] -= G[r * nv + 0] * U[j] / U[0];
            GP[r * nv + j] /= U[0];
        }
}

// Gas.hpp:1594-1655 ViscousFlux_IdealGas (no QCR)
static void viscousFlux(int nv, const real *U, const real *GP, const real n[3], bool adiabatic, real gamma, real mu, real k, real Cp, real *Flux)
{
    real velo[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
    const real lambda = -2. / 3.;
    real dV[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            dV[i][j] = GP[i * nv + 1 + j];
    real gradP[3] = {GP[0 * nv + 4], GP[1 * nv + 4], GP[2 * nv + 4]};
    real vSqr = dot3(velo, velo);
    real p = (gamma - 1) * (U[4] - U[0] * 0.5 * vSqr);
    real gradT[3];
    for (int i = 0; i < 3; i++)
        gradT[i] = (gamma / ((gamma - 1) * Cp * U[0] * U[0])) * (U[0] * gradP[i] - p * GP[i * nv + 0]);
    if (adiabatic)
    {
        real gn = dot3(gradT, n);
        for (int i = 0; i < 3; i++)
            gradT[i] -= gn * n[i];
    }
    real tr = dV[0][0] + dV[1][1] + dV[2][2];
    real S[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            S[i][j] = (dV[i][j] + dV[j][i]) * mu + (i == j ? lambda * mu * tr : 0.0);
    Flux[0] = 0;
    real Sv[3];
    for (int i = 0; i < 3; i++)
    {
        Flux[1 + i] = S[i][0] * n[0] + S[i][1] * n[1] + S[i][2] * n[2];
        Sv[i] = S[i][0] * velo[0] + S[i][1] * velo[1] + S[i][2] * velo[2] + k * gradT[i];
    }
    Flux[4] = dot3(Sv, n);
    for (int j = 5; j < nv; j++)
        Flux[j] = 0;
}

// ---------------------------------------------------------------------------
// Settings (field names follow CFV/VRSettings.hpp and Euler/EulerEvaluatorSettings.hpp)
// ---------------------------------------------------------------------------
} // namespace orc

extern "C"
{
    struct OrcVRSettings
    {
        int maxOrder, intOrder;
        double jacobiRelax;
        int SORInstead;
        int anisotropicLengths;
        int scaleType; // 0 MeanAACBB, 1 BaryDiff
        double scaleMultiplier;
        int dirWeightScheme; // 0 Factorial, 1 HQM_OPT, 999 manual
        double manualDirWeights[4];
        int geomWeightScheme; // 0 none, 1 HQM_SD, 2 SD_Power
        double geomWeightBias, geomWeightPower, geomWeightPower1, geomWeightPower2;
        double bcWeight;
    };
    struct OrcEulerSettings
    {
        int nVars;
        int rsType;
        double rsFixScale, rsIncFScale;
        double gamma, Rgas, muGas, prGas, TRef, CSutherland;
        int muModel;
        int ignoreVis;
        int rsMeanValueEig; // EulerEvaluatorSettings.hpp:79: Roe_M1..M5 through the batched dispatcher
    };
}

namespace orc
{
struct Oracle
{
    // mesh
    int dim, cellType, faceType, nvert, nfv, nf;
    long nNode, nCell, nFace;
    std::vector<real> coords, cellShift, faceShift, facePShift;
    std::vector<long> cell2node, face2node, face2cell, cell2face;
    std::vector<int> faceZone;
    OrcVRSettings vs;
    OrcEulerSettings es;
    int NDOF, R, nGf, nGc;
    // geometry (FiniteVolume.hpp:42-56)
    std::vector<real> vol, cellBary, cellCent, cellHBox, cellJDet, cellPP, smoothRatio;
    std::vector<real> faceArea, faceCent, faceJDet, facePP, faceNorm, faceMeanNorm;
    // VR (VariationalReconstruction.hpp:162-233)
    std::vector<real> baseMoment, faceWeight, faceScale;
    std::vector<real> AAInvB, AInvb, matA;
    // evaluator state (EulerEvaluator.hpp lambdaFace*, deltaLambda*)
    std::vector<real> lambdaFace, lambdaFaceC, lambdaFaceVis, lambdaFace0, deltaLambdaFace, deltaLambdaCell;
    // EulerEvaluator.hpp:187-189 lambdaFace0 / lambdaFace123 / lambdaFace4: the convective speed after
    // EvaluateDt (EvaluateDt.hxx:995-996), the face integrals of the Riemann solver's eigenvalues after an
    // EvaluateRHS with useRoeJacobian (EvaluateRHS.hxx:527-545)
    std::vector<real> lambdaFace123, lambdaFace4;
    // EulerEvaluatorSettings.hpp:53-54: jacMode 0 = useScalarJacobian (one diagonal), 1 = block diagonal
    // (useScalarJacobian false, useRoeJacobian false), 2 = block diagonal with the Roe term (useRoeJacobian)
    int jacMode = 0;
    // SA model (nVars = 6): wall distance per cell Gauss point, major length scale per cell,
    // and the source-term Jacobian diagonal of the last RHS
    std::vector<real> dWall, cellHMax, jSource;
    // boundary table indexed by face zone (EulerBC.hpp:35-48 types; value = far / inflow state or wall temperature)
    std::vector<int> bcType;
    std::vector<real> bcVal; // [zone][8]
    int zoneType(long f) const
    {
        int z = faceZone[f];
        return z >= 0 && z < (int)bcType.size() ? bcType[z] : 0;
    }

    void cellCoords(long c, real *out) const
    {
        for (int v = 0; v < nvert; v++)
            for (int d = 0; d < 3; d++)
                out[v * 3 + d] = coords[cell2node[c * nvert + v] * 3 + d] + cellShift[(c * nvert + v) * 3 + d];
    }
    void faceCoords(long f, real *out) const
    {
        for (int v = 0; v < nfv; v++)
            for (int d = 0; d < 3; d++)
                out[v * 3 + d] = coords[face2node[f * nfv + v] * 3 + d] + faceShift[(f * nfv + v) * 3 + d];
    }
    int sideOf(long c, long f) const { return face2cell[f * 2 + 0] == c ? 0 : 1; }
    long otherOf(long c, long f) const { return face2cell[f * 2 + 0] == c ? face2cell[f * 2 + 1] : face2cell[f * 2 + 0]; }
    // point on face f seen from side s (FiniteVolume.hpp:254-271 GetFaceQuadraturePPhysFromCell)
    void fromSide(long f, int s, const real *p, real *out) const
    {
        for (int d = 0; d < 3; d++)
            out[d] = p[d] + (s == 1 ? facePShift[f * 3 + d] : 0.0);
    }
    // barycentre of the other cell seen from cell c (FiniteVolume.hpp:292-311)
    void otherBary(long c, long f, real *out) const
    {
        long o = otherOf(c, f);
        int s = sideOf(c, f);
        for (int d = 0; d < 3; d++)
            out[d] = cellBary[o * 3 + d] + (s == 0 ? -facePShift[f * 3 + d] : facePShift[f * 3 + d]);
    }

    // FiniteVolume.cpp:22-330 + VariationalReconstruction.cpp:10-43
    // FiniteVolume.cpp:288-335 cellMajorHBox and FiniteVolume.hpp:387-393 GetCellMaxLenScale: the
    // largest half extent of the cell's vertices along the principal axes of its inertia tensor
    // (integrated at INT_ORDER_MAX), times 2.  Principal axes by cyclic Jacobi rotations.
    real majorLength(long c, const real *cc) const
    {
        real I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int g = 0; g < quadNPoints(cellType, INT_ORDER_MAX); g++)
        {
            real p[3], w;
            quadPoint(cellType, INT_ORDER_MAX, g, p, w);
            PointGeo pg = pointGeo(cellType, cc, p);
            real J = cellJacDet(dim, pg);
            real x[3] = {pg.x[0] - cellBary[c * 3], pg.x[1] - cellBary[c * 3 + 1], pg.x[2] - cellBary[c * 3 + 2]};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    I[a][b] += x[a] * x[b] * J * w;
        }
        int n = dim;
        real nrm = 0;
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++)
                I[a][b] /= vol[c], nrm += I[a][b] * I[a][b];
        nrm = sqrt(nrm);
        real V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        real A[3][3];
        std::memcpy(A, I, sizeof(A));
        for (int sweep = 0; sweep < 50; sweep++)
        {
            real off = 0;
            for (int a = 0; a < n; a++)
                for (int b = a + 1; b < n; b++)
                    off += A[a][b] * A[a][b];
            if (off <= 1e-34 * nrm * nrm)
                break;
            for (int a = 0; a < n; a++)
                for (int b = a + 1; b < n; b++)
                {
                    if (A[a][b] == 0)
                        continue;
                    real th = (A[b][b] - A[a][a]) / (2 * A[a][b]);
                    real t = (th >= 0 ? 1.0 : -1.0) / (abs(th) + sqrt(th * th + 1));
                    real cs = 1 / sqrt(t * t + 1), sn = t * cs;
                    for (int k = 0; k < n; k++)
                    {
                        real x = A[k][a], y = A[k][b];
                        A[k][a] = cs * x - sn * y, A[k][b] = sn * x + cs * y;
                    }
                    for (int k = 0; k < n; k++)
                    {
                        real x = A[a][k], y = A[b][k];
                        A[a][k] = cs * x - sn * y, A[b][k] = sn * x + cs * y;
                    }
                    for (int k = 0; k < n; k++)
                    {
                        real x = V[k][a], y = V[k][b];
                        V[k][a] = cs * x - sn * y, V[k][b] = sn * x + cs * y;
                    }
                }
        }
        // degenerate inertia (eigenvalue ratio below 1 + smallReal): the reference perturbs the
        // diagonal and keeps the coordinate axes, which is what the identity start gives here
        real h = 0;
        for (int k = 0; k < nvert; k++)
        {
            real x[3] = {cc[k * 3] - cellBary[c * 3], cc[k * 3 + 1] - cellBary[c * 3 + 1], cc[k * 3 + 2] - cellBary[c * 3 + 2]};
            for (int a = 0; a < n; a++)
                h = max(h, abs(V[0][a] * x[0] + V[1][a] * x[1] + V[2][a] * x[2]));
        }
        return h * 2;
    }

    void constructMetrics()
    {
        vol.assign(nCell, 0);
        cellHMax.assign(nCell, 0);
        cellBary.assign(nCell * 3, 0);
        cellCent.assign(nCell * 3, 0);
        cellHBox.assign(nCell * 3, 0);
        nGc = quadNPoints(cellType, vs.intOrder);
        cellJDet.assign(nCell * nGc, 0);
        cellPP.assign(nCell * nGc * 3, 0);
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nCell; c++)
        {
            real cc[24];
            cellCoords(c, cc);
            real v = 0;
            for (int g = 0; g < quadNPoints(cellType, INT_ORDER_MAX); g++)
            {
                real p[3], w;
                quadPoint(cellType, INT_ORDER_MAX, g, p, w);
                PointGeo pg = pointGeo(cellType, cc, p);
                v += cellJacDet(dim, pg) * w;
            }
            v += verySmallReal;
            vol[c] = v;
            real b[3] = {0, 0, 0};
            for (int g = 0; g < nGc; g++)
            {
                real p[3], w;
                quadPoint(cellType, vs.intOrder, g, p, w);
                PointGeo pg = pointGeo(cellType, cc, p);
                real J = cellJacDet(dim, pg);
                for (int d = 0; d < 3; d++)
                    b[d] += pg.x[d] * J * w;
                cellJDet[c * nGc + g] = J + verySmallReal;
                for (int d = 0; d < 3; d++)
                    cellPP[(c * nGc + g) * 3 + d] = pg.x[d];
            }
            for (int d = 0; d < 3; d++)
                cellBary[c * 3 + d] = b[d] / v;
            {
                real p[3], w;
                quadPoint(cellType, 1, 0, p, w);
                PointGeo pg = pointGeo(cellType, cc, p);
                for (int d = 0; d < 3; d++)
                    cellCent[c * 3 + d] = pg.x[d];
            }
            for (int d = 0; d < 3; d++)
            {
                real m = 0;
                for (int k = 0; k < nvert; k++)
                    m = max(m, abs(cc[k * 3 + d] - cellBary[c * 3 + d]));
                cellHBox[c * 3 + d] = m;
            }
            if (dim == 2)
                cellHBox[c * 3 + 2] = 1;
            cellHMax[c] = majorLength(c, cc);
        }
        nGf = quadNPoints(faceType, vs.intOrder);
        faceArea.assign(nFace, 0);
        faceCent.assign(nFace * 3, 0);
        faceJDet.assign(nFace * nGf, 0);
        facePP.assign(nFace * nGf * 3, 0);
        faceNorm.assign(nFace * nGf * 3, 0);
        faceMeanNorm.assign(nFace * 3, 0);
#pragma omp parallel for schedule(static)
        for (long f = 0; f < nFace; f++)
        {
            real fc[12];
            faceCoords(f, fc);
            real a = 0, nm[3] = {0, 0, 0};
            for (int g = 0; g < nGf; g++)
            {
                real p[3], w, n[3];
                quadPoint(faceType, vs.intOrder, g, p, w);
                PointGeo pg = pointGeo(faceType, fc, p);
                real J = faceJDetNorm(dim, pg, n);
                a += J * w;
                faceJDet[f * nGf + g] = J + verySmallReal;
                real nn = norm3(n);
                for (int d = 0; d < 3; d++)
                {
                    facePP[(f * nGf + g) * 3 + d] = pg.x[d];
                    faceNorm[(f * nGf + g) * 3 + d] = n[d] / nn;
                    nm[d] += n[d] / nn * J * w;
                }
            }
            faceArea[f] = a + verySmallReal;
            real nn = norm3(nm);
            for (int d = 0; d < 3; d++)
                faceMeanNorm[f * 3 + d] = nm[d] / nn;
            real p[3], w;
            quadPoint(faceType, 1, 0, p, w);
            PointGeo pg = pointGeo(faceType, fc, p);
            for (int d = 0; d < 3; d++)
                faceCent[f * 3 + d] = pg.x[d];
        }
        // FiniteVolume.cpp:590-648 ConstructCellSmoothScale (nIterCellSmoothScale = 15)
        std::vector<real> scale(nCell), cur(nCell), nxt(nCell);
        for (long c = 0; c < nCell; c++)
        {
            real s = 0;
            for (int k = 0; k < nf; k++)
                s += faceArea[cell2face[c * nf + k]];
            scale[c] = vol[c] / (s + verySmallReal);
            cur[c] = scale[c];
        }
        for (int it = 1; it <= 15; it++)
        {
            for (long c = 0; c < nCell; c++)
            {
                real nAdj = 0, sum = 0;
                for (int k = 0; k < nf; k++)
                {
                    long o = otherOf(c, cell2face[c * nf + k]);
                    if (o >= 0)
                        nAdj += 1., sum += cur[o];
                }
                sum += nAdj * 1 * cur[c];
                sum /= nAdj * 2;
                nxt[c] = min(cur[c], sum);
            }
            cur = nxt;
        }
        smoothRatio.resize(nCell);
        for (long c = 0; c < nCell; c++)
            smoothRatio[c] = cur[c] / scale[c];
    }

    // VariationalReconstruction.hpp:319-368 FDiffBaseValue (localOrientation = false)
    void diffBase(long c, const real *p, real *T, int rows, bool subtractMoment) const
    {
        real s[3] = {cellHBox[c * 3 + 0], cellHBox[c * 3 + 1], cellHBox[c * 3 + 2]};
        if (!vs.anisotropicLengths)
        {
            if (dim == 2)
                s[0] = s[1] = max(s[0], s[1]);
            else
                s[0] = s[1] = s[2] = max({s[0], s[1], s[2]});
        }
        real x = (p[0] - cellCent[c * 3 + 0]) / s[0], y = (p[1] - cellCent[c * 3 + 1]) / s[1], z = (p[2] - cellCent[c * 3 + 2]) / s[2];
        polyFill(dim, T, x, y, z, s[0], s[1], s[2], rows, NDOF);
        if (subtractMoment)
            for (int j = 0; j < NDOF; j++)
                T[j] -= baseMoment[c * NDOF + j];
    }

    // VariationalReconstruction.hpp:460-590 FFaceFunctional (isotropic path) + AccumulateDiffOrderContributions :32-98
    // DiffI: [cn][nI] rows of all diff orders (row-major, leading dim ldI), DiffJ likewise.
    void faceFunctional(long f, const real *DI, int nI, const real *DJ, int nJ, int cn, real *Conj /*nI x nJ*/) const
    {
        real fl[3] = {faceScale[f * 3 + 0], faceScale[f * 3 + 1], faceScale[f * 3 + 2]};
        real faceL = 0;
        if (vs.scaleType == 0)
        {
            real s = 0;
            for (int d = 0; d < dim; d++)
                s += fl[d] * fl[d];
            faceL = sqrt(s / dim);
        }
        else
        {
            real s = 0;
            for (int d = 0; d < dim; d++)
                s += fl[d] * fl[d];
            faceL = sqrt(s);
        }
        faceL *= vs.scaleMultiplier;
        for (int i = 0; i < nI * nJ; i++)
            Conj[i] = 0;
        const int *nc = dim == 2 ? nComb2 : nComb3;
        const int starts2[5] = {0, 1, 3, 6, 10}, starts3[5] = {0, 1, 4, 10, 20};
        const int *st = dim == 2 ? starts2 : starts3;
        int maxOrd = 0; // highest derivative order present in the cn diff rows
        while (maxOrd < 3 && st[maxOrd + 1] < cn)
            maxOrd++;
        for (int ord = maxOrd; ord >= 0; ord--)
        {
            real w = faceWeight[f * (vs.maxOrder + 1) + ord];
            real fLP = 1;
            for (int k = 0; k < ord; k++)
                fLP *= faceL * faceL;
            real scale = w * w * (faceL == 0 ? 1.0 : fLP);
            for (int i = 0; i < nI; i++)
                for (int j = 0; j < nJ; j++)
                {
                    real acc = 0;
                    for (int k = st[ord]; k < st[ord + 1]; k++)
                        acc += DI[k * nI + i] * DJ[k * nJ + j] * nc[k];
                    Conj[i * nJ + j] += acc * scale;
                }
        }
    }

    // VariationalReconstruction.cpp:56-498 ConstructBaseAndWeight (cacheDiffBase = false)
    void constructBaseAndWeight(const real *bcDirWeight /*per zone per order, may be null*/, int nZone)
    {
        baseMoment.assign(nCell * NDOF, 0);
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nCell; c++)
        {
            real cc[24];
            cellCoords(c, cc);
            std::vector<real> m(NDOF, 0.0), vv(NDOF);
            for (int g = 0; g < quadNPoints(cellType, INT_ORDER_MAX); g++)
            {
                real p[3], w;
                quadPoint(cellType, INT_ORDER_MAX, g, p, w);
                PointGeo pg = pointGeo(cellType, cc, p);
                real J = cellJacDet(dim, pg);
                diffBase(c, pg.x, vv.data(), 1, false);
                for (int j = 0; j < NDOF; j++)
                    m[j] += vv[j] * J * w;
            }
            for (int j = 0; j < NDOF; j++)
                baseMoment[c * NDOF + j] = m[j] / m[0];
        }
        int P = vs.maxOrder;
        faceWeight.assign(nFace * (P + 1), 0);
        faceScale.assign(nFace * 3, 0);
        for (long f = 0; f < nFace; f++)
        {
            long c0 = face2cell[f * 2 + 0], c1 = face2cell[f * 2 + 1];
            real dv[3];
            if (c1 >= 0)
            {
                real b1[3];
                otherBary(c0, f, b1);
                for (int d = 0; d < 3; d++)
                    dv[d] = b1[d] - cellBary[c0 * 3 + d];
            }
            else
            {
                real vCB[3];
                for (int d = 0; d < 3; d++)
                    vCB[d] = faceCent[f * 3 + d] - cellBary[c0 * 3 + d];
                real vn = dot3(vCB, &faceMeanNorm[f * 3]);
                for (int d = 0; d < 3; d++)
                    dv[d] = 2 * vn * faceMeanNorm[f * 3 + d];
            }
            if (vs.scaleType == 1)
            {
                for (int d = 0; d < 3; d++)
                    faceScale[f * 3 + d] = dv[d];
                if (dim == 2)
                    faceScale[f * 3 + 2] = 1;
            }
            else
            {
                // MeanAACBB: average of the sides' aligned boxes
                int n = 0;
                for (int s = 0; s < 2; s++)
                {
                    long c = face2cell[f * 2 + s];
                    if (c < 0)
                        continue;
                    for (int d = 0; d < 3; d++)
                        faceScale[f * 3 + d] += cellHBox[c * 3 + d];
                    n++;
                }
                for (int d = 0; d < 3; d++)
                    faceScale[f * 3 + d] /= n;
            }
            real wg = 1;
            real dn = norm3(dv);
            if (vs.geomWeightScheme == 1)
                wg = vs.geomWeightBias + pow(pow(faceArea[f], 1. / real(dim - 1)) / dn, vs.geomWeightPower * 0.5);
            if (vs.geomWeightScheme == 2)
                wg = vs.geomWeightBias + pow(faceArea[f], vs.geomWeightPower1 * 0.5) * pow(dn, vs.geomWeightPower2 * 0.5);
            real wd[4] = {0, 0, 0, 0};
            if (vs.dirWeightScheme == 0)
                for (int p = 0; p <= P; p++)
                    wd[p] = 1. / factorials[p];
            else if (vs.dirWeightScheme == 1)
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
                    wd[p] = vs.manualDirWeights[p];
            int zone = faceZone[f];
            if (c1 < 0)
                for (int p = 0; p <= P; p++)
                    wd[p] *= (bcDirWeight && zone < nZone ? bcDirWeight[zone * 4 + p] : 1.0) * vs.bcWeight;
            for (int p = 0; p <= P; p++)
                faceWeight[f * (P + 1) + p] = wd[p] * wg;
        }
    }

    // Gauss-Jordan inverse with partial pivoting (equals the reference's
    // Jacobi-SVD pseudo-inverse, HardEigen.cpp:13-23, when A has full rank)
    static bool invert(int n, const real *A, real *Ainv)
    {
        std::vector<real> M(n * 2 * n);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < 2 * n; j++)
                M[i * 2 * n + j] = j < n ? A[i * n + j] : (j - n == i ? 1.0 : 0.0);
        for (int col = 0; col < n; col++)
        {
            int piv = col;
            for (int r = col + 1; r < n; r++)
                if (abs(M[r * 2 * n + col]) > abs(M[piv * 2 * n + col]))
                    piv = r;
            if (M[piv * 2 * n + col] == 0)
                return false;
            if (piv != col)
                for (int j = 0; j < 2 * n; j++)
                    std::swap(M[piv * 2 * n + j], M[col * 2 * n + j]);
            real d = M[col * 2 * n + col];
            for (int j = 0; j < 2 * n; j++)
                M[col * 2 * n + j] /= d;
            for (int r = 0; r < n; r++)
                if (r != col)
                {
                    real fct = M[r * 2 * n + col];
                    if (fct != 0)
                        for (int j = 0; j < 2 * n; j++)
                            M[r * 2 * n + j] -= fct * M[col * 2 * n + j];
                }
        }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                Ainv[i * n + j] = M[i * 2 * n + n + j];
        return true;
    }

    // VariationalReconstruction.cpp:507-872 ConstructRecCoeff (greenGauss1Weight = 0, intOrderVR = intOrder)
    int constructRecCoeff()
    {
        AAInvB.assign(nCell * (nf + 1) * R * R, 0);
        AInvb.assign(nCell * nf * R, 0);
        matA.assign(nCell * R * R, 0);
        int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
        for (long c = 0; c < nCell; c++)
        {
            std::vector<real> A(R * R, 0.0), Ai(R * R), Bs(nf * R * R, 0.0), bs(nf * R, 0.0);
            std::vector<real> TI(NDOF * NDOF), TJ(NDOF * NDOF), DI(NDOF * R), DJ(NDOF * R), Cj(R * R), one(1, 1.0);
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                int s = sideOf(c, f);
                long o = otherOf(c, f);
                for (int g = 0; g < nGf; g++)
                {
                    real p[3], pq[3], w;
                    quadPoint(faceType, vs.intOrder, g, pq, w);
                    fromSide(f, s, &facePP[(f * nGf + g) * 3], p);
                    diffBase(c, p, TI.data(), NDOF, true);
                    for (int r = 0; r < NDOF; r++)
                        for (int j = 0; j < R; j++)
                            DI[r * R + j] = TI[r * NDOF + 1 + j];
                    real JD = faceJDet[f * nGf + g];
                    faceFunctional(f, DI.data(), R, DI.data(), R, NDOF, Cj.data());
                    for (int i = 0; i < R * R; i++)
                        A[i] += Cj[i] * JD * w;
                    if (o >= 0)
                    {
                        real po[3];
                        fromSide(f, 1 - s, &facePP[(f * nGf + g) * 3], po);
                        diffBase(o, po, TJ.data(), NDOF, true);
                        for (int r = 0; r < NDOF; r++)
                            for (int j = 0; j < R; j++)
                                DJ[r * R + j] = TJ[r * NDOF + 1 + j];
                        faceFunctional(f, DI.data(), R, DJ.data(), R, NDOF, Cj.data());
                        for (int i = 0; i < R * R; i++)
                            Bs[k * R * R + i] += Cj[i] * JD * w;
                    }
                    // b: only the 0-th diff row, against a 1x1 unit
                    faceFunctional(f, DI.data(), R, one.data(), 1, 1, Cj.data());
                    for (int i = 0; i < R; i++)
                        bs[k * R + i] += Cj[i] * JD * w;
                }
            }
            if (!invert(R, A.data(), Ai.data()))
                bad++;
            for (int i = 0; i < R * R; i++)
            {
                matA[c * R * R + i] = A[i];
                AAInvB[(c * (nf + 1) + 0) * R * R + i] = Ai[i];
            }
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                if (otherOf(c, f) < 0)
                    continue;
                for (int i = 0; i < R; i++)
                {
                    for (int j = 0; j < R; j++)
                    {
                        real acc = 0;
                        for (int l = 0; l < R; l++)
                            acc += Ai[i * R + l] * Bs[k * R * R + l * R + j];
                        AAInvB[(c * (nf + 1) + 1 + k) * R * R + i * R + j] = acc;
                    }
                    real acc = 0;
                    for (int l = 0; l < R; l++)
                        acc += Ai[i * R + l] * bs[k * R + l];
                    AInvb[(c * nf + k) * R + i] = acc;
                }
            }
        }
        return bad;
    }


    // Gas.hpp IdealGasThermalConservative2Primitive / Primitive2Conservative (dim = 3, 5 variables)
    void cons2prim(const real *U, real *P) const
    {
        real g = es.gamma;
        P[0] = U[0];
        for (int d = 0; d < 3; d++)
            P[1 + d] = U[1 + d] / U[0];
        real vsqr = sqr(P[1]) + sqr(P[2]) + sqr(P[3]);
        P[4] = (g - 1) * (U[4] - 0.5 * U[0] * vsqr);
        for (int j = 5; j < es.nVars; j++)
            P[j] = U[j] / U[0];
    }
    void prim2cons(const real *P, real *U) const
    {
        real g = es.gamma;
        U[0] = P[0];
        for (int d = 0; d < 3; d++)
            U[1 + d] = P[1 + d] * P[0];
        real vsqr = sqr(P[1]) + sqr(P[2]) + sqr(P[3]);
        U[4] = P[4] / (g - 1) + 0.5 * P[0] * vsqr;
        for (int j = 5; j < es.nVars; j++)
            U[j] = P[j] * P[0];
    }

    // EulerEvaluator_EvaluateDt.hxx:1743-2468 generateBoundaryValue, linMode 0, no rotating frame,
    // no anchors or CL driver, zero grid velocity.  Types: 1 BCFar, 2 BCWall, 3 BCWallInvis,
    // 4 BCWallIsothermal, 5 BCOut, 6 BCOutP, 7 BCIn, 9 BCSym.  Returns false for an unsupported type.
    bool bcValue(int type, int zone, const real *UL, const real *n, real *UR) const
    {
        real ULc[8];
        std::copy(UL, UL + es.nVars, ULc);
        return bcValueFix(type, zone, ULc, n, UR, false);
    }

    // fixUL (USE_FIX_ZERO_SA_NUT_AT_WALL, EvaluateDt.hxx:2291-2296): on wall types the SA variable of
    // both the inner state UL (modified) and the ghost is set to zero
    bool bcValueFix(int type, int zone, real *UL, const real *n, real *UR, bool fixUL) const
    {
        bool ok = bcValueRaw(type, zone, UL, n, UR);
        if (ok && fixUL && (type == 2 || type == 4))
            for (int j = 5; j < es.nVars; j++)
                UL[j] = UR[j] = 0;
        return ok;
    }

    bool bcValueRaw(int type, int zone, const real *UL, const real *n, real *UR) const
    {
        int nv = es.nVars;
        real g = es.gamma;
        const real *far = &bcVal[zone * 8];
        switch (type)
        {
        case 1:
        case 6:
        {
            // generateBV_FarField (:1870-1945): characteristic switching on the normal velocity
            real un = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) / UL[0];
            real vsqr = (sqr(UL[1]) + sqr(UL[2]) + sqr(UL[3])) / sqr(UL[0]);
            real p, asqr, H;
            idealGasThermal(UL[4], UL[0], vsqr, g, p, asqr, H);
            real a = sqrt(asqr);
            if (un - a > 0)
                std::copy(UL, UL + nv, UR);
            else if (un > 0)
            {
                real fp[8], lp[8];
                cons2prim(far, fp), cons2prim(UL, lp);
                lp[4] = fp[4];
                prim2cons(lp, UR);
            }
            else if (un + a > 0)
            {
                real fp[8], lp[8];
                cons2prim(far, fp), cons2prim(UL, lp);
                fp[4] = lp[4];
                prim2cons(fp, UR);
            }
            else
                std::copy(far, far + nv, UR);
            return true;
        }
        case 3:
        case 9:
        {
            // generateBV_InviscidWall (:2199-2215): mirrored momentum
            std::copy(UL, UL + nv, UR);
            real mn = UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2];
            for (int d = 0; d < 3; d++)
                UR[1 + d] -= 2 * mn * n[d];
            return true;
        }
        case 2:
        case 4:
        {
            // generateBV_ViscousWall (:2241-2330): reversed momentum (and SA variable); isothermal density
            std::copy(UL, UL + nv, UR);
            for (int d = 0; d < 3; d++)
                UR[1 + d] = -UR[1 + d];
            if (type == 4)
            {
                real P[8];
                cons2prim(UR, P);
                P[0] = P[4] / far[0] / es.Rgas;
                prim2cons(P, UR);
            }
            for (int j = 5; j < nv; j++)
                UR[j] = -UR[j];
            return true;
        }
        case 5:
            std::copy(UL, UL + nv, UR); // generateBV_Outflow
            return true;
        case 7:
            std::copy(far, far + nv, UR); // generateBV_Inflow
            return true;
        }
        return false;
    }

    // EulerEvaluator.hpp:1541-1625 CompressRecPart: fall back to the mean when rho or e < 0
    void compressRec(const real *um, const real *U, real *out) const
    {
        int nv = es.nVars;
        std::copy(U, U + nv, out);
        if (out[0] < 0)
            std::copy(um, um + nv, out);
        real eK = (sqr(out[1]) + sqr(out[2]) + sqr(out[3])) * 0.5 / (verySmallReal + out[0]);
        if (out[4] - eK < 0)
            std::copy(um, um + nv, out);
    }

    // VariationalReconstruction_Reconstruction.hxx:19-176 GetBoundaryRHS with the Euler FBoundary of
    // EulerSolver.hxx:163-175 (intOrderVRBC = intOrder): sum over Gauss points of
    // w0^2 phi_i (uBV - u_c) |J| w, returned as [R][nv]
    void boundaryRHS(long c, long f, const real *uRec, const real *u, real *BCC) const
    {
        int nv = es.nVars;
        std::fill(BCC, BCC + R * nv, 0.0);
        int type = zoneType(f);
        real w0 = faceWeight[f * (vs.maxOrder + 1) + 0];
        std::vector<real> T(NDOF);
        for (int g = 0; g < nGf; g++)
        {
            real pq[3], w;
            quadPoint(faceType, vs.intOrder, g, pq, w);
            const real *p = &facePP[(f * nGf + g) * 3];
            const real *n = &faceNorm[(f * nGf + g) * 3];
            diffBase(c, p, T.data(), 1, true);
            real UL[8], ULf[8], UB[8];
            for (int v = 0; v < nv; v++)
            {
                real a = 0;
                for (int j = 0; j < R; j++)
                    a += T[1 + j] * uRec[(c * R + j) * nv + v];
                UL[v] = u[c * nv + v] + a;
            }
            compressRec(u + c * nv, UL, ULf);
            if (!bcValueFix(type, faceZone[f], ULf, n, UB, true))
                std::copy(ULf, ULf + nv, UB);
            real JW = faceJDet[f * nGf + g] * w * w0 * w0;
            for (int i = 0; i < R; i++)
                for (int v = 0; v < nv; v++)
                    BCC[i * nv + v] += T[1 + i] * (UB[v] - u[c * nv + v]) * JW;
        }
    }

    // VariationalReconstruction_Reconstruction.hxx:485-615 DoReconstructionIter, Jacobi branch
    // (SORInstead = false), periodic/interior faces.  uRec rows: [cell][R][nv].
    void vrIterJacobi(const real *uRec, real *uRecNew, const real *u, bool recordInc, bool uRecIsZero) const
    {
        int nv = es.nVars;
        real relax = vs.jacobiRelax;
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nCell; c++)
        {
            real *out = uRecNew + c * R * nv;
            const real *in = uRec + c * R * nv;
            for (int i = 0; i < R * nv; i++)
                out[i] = recordInc ? (uRecIsZero ? 0.0 : in[i]) : in[i] * (1 - relax);
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                long o = otherOf(c, f);
                if (o < 0)
                {
                    // boundary face: + relax A^-1 BCC (recordInc: - A^-1 BCC, skipped when uRecIsZero)
                    if (recordInc && uRecIsZero)
                        continue;
                    std::vector<real> BCC(R * nv);
                    boundaryRHS(c, f, uRec, u, BCC.data());
                    const real *Ai = &AAInvB[(c * (nf + 1)) * R * R];
                    for (int i = 0; i < R; i++)
                        for (int v = 0; v < nv; v++)
                        {
                            real acc = 0;
                            for (int j = 0; j < R; j++)
                                acc += Ai[i * R + j] * BCC[j * nv + v];
                            if (recordInc)
                                out[i * nv + v] -= acc;
                            else
                                out[i * nv + v] += relax * acc;
                        }
                    continue;
                }
                const real *M = &AAInvB[(c * (nf + 1) + 1 + k) * R * R];
                const real *b = &AInvb[(c * nf + k) * R];
                for (int i = 0; i < R; i++)
                    for (int v = 0; v < nv; v++)
                    {
                        real acc = 0;
                        if (!(recordInc && uRecIsZero))
                            for (int j = 0; j < R; j++)
                                acc += M[i * R + j] * uRec[(o * R + j) * nv + v];
                        acc += b[i] * (u[o * nv + v] - u[c * nv + v]);
                        if (recordInc)
                            out[i * nv + v] -= acc;
                        else
                            out[i * nv + v] += relax * acc;
                    }
            }
        }
    }

    // DoReconstructionIter with SORInstead (VariationalReconstruction_Reconstruction.hxx:534-611, not recordInc): uRec is
    // updated in place in natural cell order, row_c = (1 - relax) row_c + relax sum_k (A^-1 B_k uRec_o + A^-1 b_k (u_o - u_c))
    // with the neighbours' current rows; a boundary face's GetBoundaryRHS reads the cell's partially updated row, since the
    // reference adds each face's term to uRec[iCell] as it goes
    void vrIterSOR(real *uRec, const real *u) const
    {
        int nv = es.nVars;
        real relax = vs.jacobiRelax;
        std::vector<real> t(R * nv), BCC(R * nv);
        for (long c = 0; c < nCell; c++)
        {
            real *row = uRec + c * R * nv;
            for (int i = 0; i < R * nv; i++)
                row[i] *= 1 - relax;
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                long o = otherOf(c, f);
                if (o < 0)
                {
                    boundaryRHS(c, f, uRec, u, BCC.data());
                    const real *Ai = &AAInvB[(c * (nf + 1)) * R * R];
                    for (int i = 0; i < R; i++)
                        for (int v = 0; v < nv; v++)
                        {
                            real acc = 0;
                            for (int j = 0; j < R; j++)
                                acc += Ai[i * R + j] * BCC[j * nv + v];
                            t[i * nv + v] = acc;
                        }
                }
                else
                {
                    const real *M = &AAInvB[(c * (nf + 1) + 1 + k) * R * R];
                    const real *b = &AInvb[(c * nf + k) * R];
                    for (int i = 0; i < R; i++)
                        for (int v = 0; v < nv; v++)
                        {
                            real acc = 0;
                            for (int j = 0; j < R; j++)
                                acc += M[i * R + j] * uRec[(o * R + j) * nv + v];
                            t[i * nv + v] = acc + b[i] * (u[o * nv + v] - u[c * nv + v]);
                        }
                }
                for (int i = 0; i < R * nv; i++)
                    row[i] += relax * t[i];
            }
        }
    }

    // EulerEvaluator.hpp:751-789 muEff
    real muEff(const real *U, real T) const
    {
        switch (es.muModel)
        {
        case 0:
            return es.muGas;
        case 1:
        {
            real TRel = T / es.TRef;
            return es.muGas * TRel * sqrt(TRel) * (es.TRef + es.CSutherland) / (T + es.CSutherland);
        }
        case 2:
            return es.muGas * U[0];
        }
        return std::nan("0");
    }

    real cp() const { return es.Rgas * es.gamma / (es.gamma - 1); }

    // EulerEvaluator_EvaluateDt.hxx:840-1048 EvaluateDt (no grid velocity, laminar)
    void evaluateDt(const real *u, real CFL, real MaxDt, bool useLocalDt, real *dt, real *dtMin)
    {
        int nv = es.nVars;
        real gamma = es.gamma;
        lambdaFace.assign(nFace, 0);
        lambdaFaceC.assign(nFace, 0);
        lambdaFaceVis.assign(nFace, 0);
        lambdaFace0.assign(nFace, 0);
        lambdaFace123.assign(nFace, 0);
        lambdaFace4.assign(nFace, 0);
        deltaLambdaFace.assign(nFace, 0);
        deltaLambdaCell.assign(nCell, 0);
#pragma omp parallel for schedule(static)
        for (long f = 0; f < nFace; f++)
        {
            long c0 = face2cell[f * 2 + 0], c1 = face2cell[f * 2 + 1];
            const real *n = &faceMeanNorm[f * 3];
            std::vector<real> uMean(u + c0 * nv, u + c0 * nv + nv);
            const real *UL = u + c0 * nv;
            real vL[3] = {UL[1] / UL[0], UL[2] / UL[0], UL[3] / UL[0]}, vR[3];
            real pL, asqrL, HL, pR, asqrR, HR;
            idealGasThermal(UL[4], UL[0], dot3(vL, vL), gamma, pL, asqrL, HL);
            std::copy(vL, vL + 3, vR);
            pR = pL, HR = HL, asqrR = asqrL;
            if (c1 >= 0)
            {
                const real *UR = u + c1 * nv;
                for (int i = 0; i < nv; i++)
                    uMean[i] = (uMean[i] + UR[i]) * 0.5;
                for (int d = 0; d < 3; d++)
                    vR[d] = UR[1 + d] / UR[0];
                idealGasThermal(UR[4], UR[0], dot3(vR, vR), gamma, pR, asqrR, HR);
            }
            real vsum[3] = {vL[0] + vR[0], vL[1] + vR[1], vL[2] + vR[2]};
            real veloNMean = 0.5 * dot3(vsum, n);
            real veloNL = dot3(vL, n), veloNR = dot3(vR, n), vgN = 0;
            real pMean = (pL + pR) * 0.5;
            real aL = sqrt(asqrL), aR = sqrt(asqrR);
            real lambdaConvection = max(aL + abs(veloNL - vgN), aR + abs(veloNR - vgN));
            real T = pMean / ((gamma - 1) / gamma * cp() * uMean[0]);
            real muf = muEff(uMean.data(), T);
            muf += muTurSA(uMean.data(), muf);
            real lamVis = muf / uMean[0] * max(4. / 3., gamma / es.prGas);
            real area = faceArea[f];
            real volR = c1 >= 0 ? vol[c1] : vol[c0];
            lambdaFace[f] = lambdaConvection + lamVis * area * (1. / vol[c0] + 1. / volR);
            lambdaFaceC[f] = abs(veloNMean - vgN) + lamVis * area * (1. / vol[c0] + 1. / volR);
            lambdaFaceVis[f] = lamVis * area * (1. / vol[c0] + 1. / volR);
            lambdaFace0[f] = lambdaFace123[f] = lambdaFace4[f] = lambdaConvection;
            real dvn = veloNR - veloNL;
            deltaLambdaFace[f] = max({abs(dvn + aR - aL), abs(dvn - aR + aL), abs(aL - aR)});
        }
        real mn = veryLargeReal;
        for (long c = 0; c < nCell; c++)
        {
            real lc = 0;
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                lc += lambdaFace[f] * faceArea[f];
            }
            dt[c] = min(CFL * vol[c] * smoothRatio[c] / (lc + 1e-100), MaxDt);
            mn = min(mn, dt[c]);
            real dl = 0;
            for (int k = 0; k < nf; k++)
                dl = max(dl, deltaLambdaFace[cell2face[c * nf + k]]);
            deltaLambdaCell[c] = dl;
        }
        *dtMin = mn;
        if (!useLocalDt)
            for (long c = 0; c < nCell; c++)
                dt[c] = mn;
    }

    // EulerEvaluator.hpp:791-833 getMuTur (SA, negative-model smoothing of chi)
    real muTurSA(const real *U, real muf) const
    {
        if (es.nVars < 6)
            return 0;
        const real cnu1 = 7.1;
        real Chi = U[5] * es.muGas / muf;
        if (Chi < 10)
            Chi = 0.05 * log(1 + exp(20 * Chi));
        real Chi3 = Chi * Chi * Chi;
        real fnu1 = Chi3 / (Chi3 + cnu1 * cnu1 * cnu1);
        return muf * max(Chi * fnu1, 0.0);
    }

    // fluxFace viscous part at one point (EvaluateDt.hxx:1167-1209) with the SA terms of
    // visFluxTurVariable (EulerEvaluator.hpp:835-877): mu + mu_t, heat conduction with Pr_t = 0.9,
    // and the nuTilde diffusion flux
    void pointViscousFlux(const real *UM, const real *GMP, const real *n, bool adiabatic, real *vis) const
    {
        int nv = es.nVars;
        real gamma = es.gamma;
        real velo2 = (sqr(UM[1]) + sqr(UM[2]) + sqr(UM[3])) / sqr(UM[0]);
        real pM, aM, HM;
        idealGasThermal(UM[4], UM[0], velo2, gamma, pM, aM, HM);
        real Tm = pM / ((gamma - 1) / gamma * cp() * UM[0]);
        real mufPhy = muEff(UM, Tm);
        real muTur = muTurSA(UM, mufPhy);
        real muf = mufPhy + muTur;
        real k = cp() * muTur / 0.9 + cp() * mufPhy / es.prGas;
        viscousFlux(nv, UM, GMP, n, adiabatic, gamma, muf, k, cp(), vis);
        if (nv >= 6)
        {
            const real sigma = 2.0 / 3.0, cn1 = 16.0;
            real fn = 1;
            if (UM[5] < 0)
            {
                real Chi = UM[5] * es.muGas / mufPhy;
                fn = (cn1 + Chi * Chi * Chi) / (cn1 - Chi * Chi * Chi);
            }
            vis[5] = (GMP[0 * nv + 5] * n[0] + GMP[1 * nv + 5] * n[1] + GMP[2 * nv + 5] * n[2]) * (mufPhy + UM[5] * es.muGas * fn) / sigma;
        }
    }

    // passive-scalar upwind flux of the SA variable (EvaluateDt.hxx:1413-1425), with the
    // Riemann solver's lam123 as the dissipation speed (ransEigScheme 0)
    void scalarConvectiveFlux(const real *UL, const real *UR, const real *n, real lam123, real *F) const
    {
        for (int j = 5; j < es.nVars; j++)
        {
            real vnL = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) / UL[0];
            real vnR = (UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2]) / UR[0];
            F[j] = ((vnL * UL[j] + vnR * UR[j]) - (UR[j] - UL[j]) * lam123) * 0.5;
        }
    }

    // RANS_ke.hpp:985-1195 GetSource_SA with the settings defaults (SADESMode 1, rotation
    // correction on, SAVersion 0) and the compiled options USE_NS_SA_NEGATIVE_MODEL and
    // SA_USE_FT2_TERM; mode 0 source, mode 1 diagonal Jacobian.  G is the conservative gradient [3][nv].
    real saSource(const real *U, const real *G, real mufPhy, real d, real lLES, real hMax, int mode) const
    {
        const int nv = es.nVars;
        const real muRef = es.muGas;
        const real cb1 = 0.1355, cb2 = 0.622, sigma = 2.0 / 3.0, cnu1 = 7.1, cnu2 = 0.7, cnu3 = 0.9, cw2 = 0.3, cw3 = 2,
                   kappa = 0.41, rlim = 10, cn1 = 16.0;
        const real cw1 = cb1 / sqr(kappa) + (1 + cb2) / sigma;
        const real ct3 = 1.2, ct4 = 0.5;
        real nuh = U[5] * muRef / U[0];
        real Chi = U[5] * muRef / mufPhy;
        real Chi3 = Chi * Chi * Chi;
        real fnu1 = Chi3 / (Chi3 + cnu1 * cnu1 * cnu1);
        real fnu2 = 1 - Chi / (1 + Chi * fnu1);
        real velo[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
        real diffRho[3], diffNu[3], diffU[3][3];
        for (int i = 0; i < 3; i++)
        {
            diffRho[i] = G[i * nv + 0];
            diffNu[i] = (G[i * nv + 5] * muRef - nuh * diffRho[i]) / U[0];
            for (int j = 0; j < 3; j++)
                diffU[i][j] = (G[i * nv + 1 + j] - diffRho[i] * velo[j]) / U[0];
        }
        real om2 = 0, ss2 = 0, du2 = 0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
            {
                real o = 0.5 * (diffU[j][i] - diffU[i][j]);
                real sij = diffU[i][j] + diffU[j][i];
                om2 += o * o, ss2 += sij * sij, du2 += diffU[i][j] * diffU[i][j];
            }
        real S = sqrt(om2) * sqrt(2.0);
        real SS = sqrt(ss2) * (1. / sqrt(2.0));
        real SRotCor = 2.0 * min(0.0, S - SS);
        real diffUNorm = sqrt(du2);
        real ft2 = ct3 * exp(-ct4 * sqr(Chi));
        real lDES = d;
        {
            real lRANS = d, fwStar = .424;
            real nuTur = mufPhy / U[0] * max(Chi * fnu1, 0.0);
            real nufPhy = mufPhy / U[0];
            real den = sqr(kappa) * sqr(d) * max(smallReal, diffUNorm);
            real rd = (nuTur + nufPhy) / den;
            real fd = 1. - tanh(pow(8 * rd, 3));
            real psiSqr = Chi <= 0 ? 100.0
                                   : min(100.0, (1 - cb1 / (cw1 * sqr(kappa) * fwStar) * (ft2 + (1 - ft2) * fnu2)) /
                                                         (fnu1 * max(smallReal, 1 - ft2)));
            real psi = sqrt(max(psiSqr, 1.0));
            lDES = lRANS - fd * max(0., lRANS - lLES * psi);
            // IDDES (SADESMode 1)
            real alphaIDDES = 0.25 - d / hMax;
            real fB = min(2 * exp(-9. * sqr(alphaIDDES)), 1.0);
            const real cl = 3.55, ct = 1.63;
            real rdt = nuTur / den, rdl = nufPhy / den;
            real ftt = tanh(pow(sqr(ct) * rdt, 3));
            real flt = sqr(sqr(cl) * rdl);
            real fl = tanh(sqr(sqr(flt)) * flt);
            real fe1 = 2. * exp(-(alphaIDDES >= 0 ? 11.09 : 9.0) * sqr(alphaIDDES));
            real fe2 = 1. - max(ftt, fl);
            real fe = max(fe1 - 1., 0.) * psi * fe2;
            real fdTilde = max(fB, tanh(pow(8 * rdt, 3)));
            real lIDDES = fdTilde * (1 + fe) * lRANS + (1 - fdTilde) * lLES * psi;
            lDES = max(lLES * smallReal, lIDDES);
        }
        d = lDES;
        real Sbar = nuh / (sqr(kappa) * sqr(d)) * fnu2;
        real Sh = Sbar < -cnu2 * S ? S + S * (sqr(cnu2) * S + cnu3 * Sbar) / ((cnu3 - 2 * cnu2) * S - Sbar) : S + Sbar;
        real r = min(nuh / (Sh * sqr(kappa * d) + verySmallReal), rlim);
        real g = r + cw2 * (pow(r, 6) - r);
        real fw = g * pow((1 + pow(cw3, 6)) / (pow(g, 6) + pow(cw3, 6)), 1. / 6.);
        real D = (cw1 * fw - cb1 / sqr(kappa) * ft2) * sqr(nuh / lDES);
        real P = cb1 * (1 - ft2) * (Sh + SRotCor) * nuh;
        real fn = 1;
        if (U[5] < 0)
        {
            real Chi_ = U[5] * muRef / mufPhy;
            fn = (cn1 + pow(Chi_, 3)) / (cn1 - pow(Chi_, 3));
            D = -cw1 * sqr(nuh / lDES);
            P = cb1 * (1 - ct3) * abs(S + SRotCor) * nuh;
        }
        real dd = diffRho[0] * diffNu[0] + diffRho[1] * diffNu[1] + diffRho[2] * diffNu[2];
        real nn = diffNu[0] * diffNu[0] + diffNu[1] * diffNu[1] + diffNu[2] * diffNu[2];
        if (mode == 0)
            return U[0] * (P - D + nn * cb2 / sigma) / muRef - (U[5] * fn * muRef + mufPhy) / (U[0] * sigma) * dd / muRef;
        return -min(U[0] * (min(P, 0.0) * 1 - D * 2) / muRef / (abs(U[5]) + verySmallReal), -verySmallReal);
    }

    // EvaluateRHS.hxx:665-801 source integration (SA only; the NS source is zero) and the
    // source-term Jacobian diagonal JSource, both cell means
    // EvaluateRHS.hxx:677-801: values from uRec, gradients from uRecUnlim (uRecG), the integral scaled by
    // cellRHSAlpha / V (alpha == nullptr: 1)
    void addSource(const real *u, const real *uRec, real *rhs, const real *uRecG = nullptr, const real *alpha = nullptr)
    {
        if (!uRecG)
            uRecG = uRec;
        int nv = es.nVars;
        jSource.assign(nCell * nv, 0.0);
        if (nv < 6)
            return;
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nCell; c++)
        {
            std::vector<real> T((dim + 1) * NDOF);
            real S = 0, J = 0;
            for (int g = 0; g < nGc; g++)
            {
                real pq[3], w;
                quadPoint(cellType, vs.intOrder, g, pq, w);
                diffBase(c, &cellPP[(c * nGc + g) * 3], T.data(), dim + 1, true);
                real U[8], G[3 * 8] = {0};
                for (int v = 0; v < nv; v++)
                {
                    real a = u[c * nv + v];
                    for (int j = 0; j < R; j++)
                        a += T[1 + j] * uRec[(c * R + j) * nv + v];
                    U[v] = a;
                    for (int d = 0; d < dim; d++)
                    {
                        real ga = 0;
                        for (int j = 0; j < R; j++)
                            ga += T[(1 + d) * NDOF + 1 + j] * uRecG[(c * R + j) * nv + v];
                        G[d * nv + v] = ga;
                    }
                }
                real velo2 = (sqr(U[1]) + sqr(U[2]) + sqr(U[3])) / sqr(U[0]);
                real pM, aM, HM;
                idealGasThermal(U[4], U[0], velo2, es.gamma, pM, aM, HM);
                real Tm = pM / ((es.gamma - 1) / es.gamma * cp() * U[0]);
                real muf = muEff(U, Tm);
                real d = min(dWall.empty() ? veryLargeReal : dWall[c * nGc + g], pow(veryLargeReal, 1. / 6.));
                real hMax = cellHMax[c];
                real lLES = min(hMax * veryLargeReal, max(d * 1.0, hMax * 1.0));
                real JW = cellJDet[c * nGc + g] * w;
                S += saSource(U, G, muf, d, lLES, hMax, 0) * JW;
                J += saSource(U, G, muf, d, lLES, hMax, 1) * JW;
            }
            real a = alpha ? alpha[c] : 1.0;
            rhs[c * nv + 5] += S * a / vol[c];
            jSource[c * nv + 5] = J * a / vol[c];
        }
    }

    // EulerEvaluator_EvaluateRHS.hxx:171-562 for a boundary face (f2c[1] == UnInitIndex): ghost
    // state from generateBoundaryValue at every Gauss point, Roe means from the ghost of the cell
    // mean at the face centre (:198-210), gradient copied from the inside (:360-362), GRP
    // distance from the face centre (:363-386), viscous flux removed on slip, far-field and
    // outflow faces (:423-430, EvaluateDt.hxx:1203-1207)
    // lam3 (may be nullptr): the face integrals of the eigenvalues l0, l123, l4 divided by the area (EvaluateRHS.hxx:527-545)
    void boundaryFaceFlux(long f, const real *u, const real *uRec, real *fluxEs, const real *uRecG, real *lam3 = nullptr) const
    {
        real lamEs[3] = {0, 0, 0};
        int nv = es.nVars;
        real gamma = es.gamma;
        long c0 = face2cell[f * 2 + 0];
        int type = zoneType(f);
        int zone = faceZone[f];
        std::vector<real> T0(4 * NDOF);
        for (int v = 0; v < nv; v++)
            fluxEs[v] = 0;
        const real *ULm = u + c0 * nv;
        real URm[8];
        if (!bcValue(type, zone, ULm, &faceMeanNorm[f * 3], URm))
            std::copy(ULm, ULm + nv, URm);
        real dLambda = deltaLambdaCell[c0];
        bool zeroGrad = type == 3 || type == 5 || type == 1 || type == 9; // BCWallInvis, BCOut, BCFar, BCSym
        bool noVis = type == 3 || type == 9;
        for (int g = 0; g < nGf; g++)
        {
            real pq[3], w;
            quadPoint(faceType, vs.intOrder, g, pq, w);
            const real *n = &faceNorm[(f * nGf + g) * 3];
            const real *p0 = &facePP[(f * nGf + g) * 3];
            diffBase(c0, p0, T0.data(), dim + 1, true);
            real UL[8], UR[8], GL[3 * 8] = {0};
            for (int v = 0; v < nv; v++)
            {
                real a = 0;
                for (int j = 0; j < R; j++)
                    a += T0[1 + j] * uRec[(c0 * R + j) * nv + v];
                UL[v] = u[c0 * nv + v] + a;
                for (int d = 0; d < dim; d++)
                {
                    real ga = 0;
                    for (int j = 0; j < R; j++)
                        ga += T0[(1 + d) * NDOF + 1 + j] * uRecG[(c0 * R + j) * nv + v];
                    GL[d * nv + v] = ga;
                }
            }
            if (!bcValueFix(type, zone, UL, n, UR, true))
                std::copy(UL, UL + nv, UR);
            real dc[3] = {faceCent[f * 3 + 0] - cellBary[c0 * 3 + 0], faceCent[f * 3 + 1] - cellBary[c0 * 3 + 1],
                          faceCent[f * 3 + 2] - cellBary[c0 * 3 + 2]};
            real distBaryPerp = abs(dot3(dc, n)) * 2.;
            real distGRP = vol[c0] / faceArea[f] * 2;
            distGRP = max(min(distBaryPerp, distGRP * 2), distGRP * 0.25);
            if (type == 3 || type == 9)
                distGRP += veryLargeReal;
            real UM[8], GM[3 * 8], GMP[3 * 8];
            for (int v = 0; v < nv; v++)
                UM[v] = 0.5 * (UL[v] + UR[v]);
            for (int d = 0; d < 3; d++)
                for (int v = 0; v < nv; v++)
                    GM[d * nv + v] = GL[d * nv + v] + (1.0 / distGRP) * (n[d] * (UR[v] - UL[v]));
            if (es.ignoreVis || zeroGrad)
                for (int i = 0; i < 3 * nv; i++)
                    GM[i] = 0;
            gradCons2Prim(nv, UM, GM, GMP, gamma);
            real vis[8] = {0};
            if (!es.ignoreVis && !noVis)
                pointViscousFlux(UM, GMP, n, type == 2, vis);
            real F[8] = {0}, l0, l1, l4, vg[3] = {0, 0, 0};
            riemann(es.rsType, UL, UR, ULm, URm, vg, n, gamma, F, dLambda, es.rsFixScale, es.rsIncFScale, l0, l1, l4,
                    es.rsMeanValueEig ? &faceMeanNorm[f * 3] : nullptr);
            scalarConvectiveFlux(UL, UR, n, l1, F);
            real JD = faceJDet[f * nGf + g];
            for (int v = 0; v < nv; v++)
                fluxEs[v] += -(F[v] - vis[v]) * JD * w;
            lamEs[0] += l0 * JD * w, lamEs[1] += l1 * JD * w, lamEs[2] += l4 * JD * w;
        }
        if (lam3)
            for (int i = 0; i < 3; i++)
                lam3[i] = lamEs[i] / faceArea[f];
    }

    // EulerEvaluator_EvaluateRHS.hxx:55-818 EvaluateRHS with the flux of
    // EulerEvaluator_EvaluateDt.hxx:1084-1511 fluxFace (interior/periodic faces,
    // no limiter, source term ignored, no grid velocity)
    // uRecG: the unlimited reconstruction the gradients come from (EvaluateRHS.hxx:264-327, uRecUnlim;
    // nullptr: uRec); alpha: cellRHSAlpha of the source term (nullptr: 1); fluxWall (may be nullptr): the
    // wall-flux integral of :599-607, minus the face fluxes of BCWall / BCWallIsothermal faces (and of
    // BCWallInvis faces when muGas < 1e-99), summed in face order
    void evaluateRHS(const real *u, const real *uRec, real *rhs, real *faceFluxOut, const real *uRecG = nullptr, const real *alpha = nullptr,
                     real *fluxWall = nullptr)
    {
        if (!uRecG)
            uRecG = uRec;
        int nv = es.nVars;
        real gamma = es.gamma;
        std::vector<real> faceFlux(nFace * nv, 0.0);
        if (deltaLambdaCell.empty())
            deltaLambdaCell.assign(nCell, 0.0);
        const bool recLam = jacMode == 2;
        if (recLam && (long)lambdaFace0.size() != nFace)
            lambdaFace0.assign(nFace, 0), lambdaFace123.assign(nFace, 0), lambdaFace4.assign(nFace, 0);
#pragma omp parallel for schedule(static)
        for (long f = 0; f < nFace; f++)
        {
            long c0 = face2cell[f * 2 + 0], c1 = face2cell[f * 2 + 1];
            if (c1 < 0)
            {
                real lam3[3];
                boundaryFaceFlux(f, u, uRec, &faceFlux[f * nv], uRecG, lam3);
                if (recLam)
                    lambdaFace0[f] = lam3[0], lambdaFace123[f] = lam3[1], lambdaFace4[f] = lam3[2];
                continue;
            }
            real lamEs[3] = {0, 0, 0};
            std::vector<real> T0(4 * NDOF), T1(4 * NDOF);
            real fluxEs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            const real *ULm = u + c0 * nv, *URm = u + c1 * nv;
            real dLambda = max(deltaLambdaCell[c0], deltaLambdaCell[c1]);
            for (int g = 0; g < nGf; g++)
            {
                real pq[3], w;
                quadPoint(faceType, vs.intOrder, g, pq, w);
                const real *n = &faceNorm[(f * nGf + g) * 3];
                real p0[3], p1[3];
                fromSide(f, 0, &facePP[(f * nGf + g) * 3], p0);
                fromSide(f, 1, &facePP[(f * nGf + g) * 3], p1);
                int rows = dim + 1;
                diffBase(c0, p0, T0.data(), rows, true);
                diffBase(c1, p1, T1.data(), rows, true);
                real UL[8], UR[8], GL[3 * 8] = {0}, GR[3 * 8] = {0};
                for (int v = 0; v < nv; v++)
                {
                    real a = 0, b = 0;
                    for (int j = 0; j < R; j++)
                    {
                        a += T0[1 + j] * uRec[(c0 * R + j) * nv + v];
                        b += T1[1 + j] * uRec[(c1 * R + j) * nv + v];
                    }
                    UL[v] = u[c0 * nv + v] + a;
                    UR[v] = u[c1 * nv + v] + b;
                    for (int d = 0; d < dim; d++)
                    {
                        real ga = 0, gb = 0;
                        for (int j = 0; j < R; j++)
                        {
                            ga += T0[(1 + d) * NDOF + 1 + j] * uRecG[(c0 * R + j) * nv + v];
                            gb += T1[(1 + d) * NDOF + 1 + j] * uRecG[(c1 * R + j) * nv + v];
                        }
                        GL[d * nv + v] = ga, GR[d * nv + v] = gb;
                    }
                }
                real minVol = min(vol[c0], vol[c1]);
                real b1[3];
                otherBary(c0, f, b1);
                real db[3] = {b1[0] - cellBary[c0 * 3 + 0], b1[1] - cellBary[c0 * 3 + 1], b1[2] - cellBary[c0 * 3 + 2]};
                real distBaryPerp = abs(dot3(db, n));
                real distGRP = minVol / faceArea[f] * 2;
                distGRP = max(min(distBaryPerp, distGRP * 2), distGRP * 0.25);
                real UM[8], GM[3 * 8], GMP[3 * 8];
                for (int v = 0; v < nv; v++)
                    UM[v] = 0.5 * (UL[v] + UR[v]);
                for (int d = 0; d < 3; d++)
                    for (int v = 0; v < nv; v++)
                        GM[d * nv + v] = (GR[d * nv + v] + GL[d * nv + v]) * 0.5 + (1.0 / distGRP) * (n[d] * (UR[v] - UL[v]));
                if (es.ignoreVis)
                    for (int i = 0; i < 3 * nv; i++)
                        GM[i] = 0;
                gradCons2Prim(nv, UM, GM, GMP, gamma);
                // fluxFace (EulerEvaluator_EvaluateDt.hxx:1084-1511)
                real vis[8] = {0};
                if (!es.ignoreVis)
                    pointViscousFlux(UM, GMP, n, false, vis);
                real F[8] = {0}, l0, l1, l4, vg[3] = {0, 0, 0};
                riemann(es.rsType, UL, UR, ULm, URm, vg, n, gamma, F, dLambda, es.rsFixScale, es.rsIncFScale, l0, l1, l4,
                        es.rsMeanValueEig ? &faceMeanNorm[f * 3] : nullptr);
                scalarConvectiveFlux(UL, UR, n, l1, F);
                real JD = faceJDet[f * nGf + g];
                for (int v = 0; v < nv; v++)
                    fluxEs[v] += -(F[v] - vis[v]) * JD * w;
                lamEs[0] += l0 * JD * w, lamEs[1] += l1 * JD * w, lamEs[2] += l4 * JD * w;
            }
            for (int v = 0; v < nv; v++)
                faceFlux[f * nv + v] = fluxEs[v];
            if (recLam)
                lambdaFace0[f] = lamEs[0] / faceArea[f], lambdaFace123[f] = lamEs[1] / faceArea[f], lambdaFace4[f] = lamEs[2] / faceArea[f];
        }
        // cell-wise gather (equivalent to the reference's face scatter, EvaluateRHS.hxx:550-562)
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nCell; c++)
        {
            for (int v = 0; v < nv; v++)
                rhs[c * nv + v] = 0;
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                real sgn = sideOf(c, f) == 0 ? 1.0 : -1.0;
                for (int v = 0; v < nv; v++)
                    rhs[c * nv + v] += sgn * faceFlux[f * nv + v] / vol[c];
            }
        }
        addSource(u, uRec, rhs, uRecG, alpha);
        if (faceFluxOut)
            std::copy(faceFlux.begin(), faceFlux.end(), faceFluxOut);
        if (fluxWall)
        {
            for (int v = 0; v < nv; v++)
                fluxWall[v] = 0;
            for (long f = 0; f < nFace; f++)
            {
                if (face2cell[f * 2 + 1] >= 0)
                    continue;
                int t = zoneType(f);
                if (t == 2 || t == 4 || (t == 3 && es.muGas < 1e-99))
                    for (int v = 0; v < nv; v++)
                        fluxWall[v] -= faceFlux[f * nv + v];
            }
        }
    }

    // EulerEvaluator.hxx:37-159 LUSGSMatrixInit, scalar Jacobian, source ignored
    void lusgsInit(const real *dTau, real dt, real alphaDiag, real *jdiag) const
    {
        // the SA model keeps one diagonal per variable (JDiag.getDiag plus alphaDiag JSource, :139-153)
        int nv = es.nVars, nd = nv >= 6 ? nv : 1;
        for (long c = 0; c < nCell; c++)
        {
            real fp = 1.0 / dTau[c] + 1.0 / dt;
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                fp += (0.5 * alphaDiag) * faceArea[f] * lambdaFace[f] / vol[c];
            }
            for (int v = 0; v < nd; v++)
                jdiag[c * nd + v] = fp + (nd > 1 && !jSource.empty() ? alphaDiag * jSource[c * nv + v] : 0.0);
        }
    }

    // EulerEvaluator.hpp:1100-1158 fluxJacobian0_Right_Times_du, useRoeTerm = 0
    void fluxJacTimesDu(const real *U, const real n[3], const real *dU, real lambdaMain, real *dF) const
    {
        int nv = es.nVars;
        real gamma = es.gamma;
        real velo[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
        real p, H, asqr;
        idealGasThermal(U[4], U[0], dot3(velo, velo), gamma, p, asqr, H);
        // Gas.hpp:462-471 IdealGasUIncrement
        real dVelo[3];
        for (int d = 0; d < 3; d++)
            dVelo[d] = (dU[1 + d] - U[1 + d] / U[0] * dU[0]) / U[0];
        real dp = (gamma - 1) * (dU[4] - 0.5 * (dU[1] * velo[0] + dU[2] * velo[1] + dU[3] * velo[2] + U[1] * dVelo[0] + U[2] * dVelo[1] + U[3] * dVelo[2]));
        // Gas.hpp:495-513 GasInviscidFluxFacialIncrement (vg = 0)
        real vn = dot3(velo, n), dvn = dot3(dVelo, n);
        dF[0] = dU[1] * n[0] + dU[2] * n[1] + dU[3] * n[2];
        for (int d = 0; d < 3; d++)
            dF[1 + d] = dU[1 + d] * vn + U[1 + d] * dvn + n[d] * dp;
        dF[4] = (dU[4] + dp) * vn + (U[4] + p) * dvn;
        for (int j = 5; j < nv; j++)
            dF[j] = dU[j] * vn + U[j] * dvn;
        for (int j = 0; j < nv; j++)
            dF[j] += -1 * lambdaMain * dU[j];
    }

    // Gas.hpp:1149-1181 GetRoeAverage of (U, UOther) and Gas.hpp:1210-1243 RoeFluxIncFDiff: incF += the Roe
    // dissipation of the jump incU with the eigenvalues l0, l123, l4 (passive scalars carried with l123)
    void roeFluxIncFDiff(const real *U, const real *UOther, const real n[3], const real *incU, real l0, real l123, real l4, real *incF) const
    {
        roeFluxIncFDiffS(es.nVars, es.gamma, U, UOther, n, incU, l0, l123, l4, incF);
    }
    static void roeFluxIncFDiffS(int nv, real gamma, const real *U, const real *UOther, const real n[3], const real *incU, real l0, real l123,
                                 real l4, real *incF)
    {
        real vL[3], vR[3];
        for (int d = 0; d < 3; d++)
            vL[d] = U[1 + d] / U[0], vR[d] = UOther[1 + d] / UOther[0];
        real pL, aL2, HL, pR, aR2, HR;
        idealGasThermal(U[4], U[0], dot3(vL, vL), gamma, pL, aL2, HL);
        idealGasThermal(UOther[4], UOther[0], dot3(vR, vR), gamma, pR, aR2, HR);
        real sL = sqrt(U[0]), sR = sqrt(UOther[0]);
        real vRoe[3];
        for (int d = 0; d < 3; d++)
            vRoe[d] = (sL * vL[d] + sR * vR[d]) / (sL + sR);
        real vsqrRoe = dot3(vRoe, vRoe);
        real HRoe = (sL * HL + sR * HR) / (sL + sR);
        real asqrRoe = (gamma - 1) * (HRoe - 0.5 * vsqrRoe);
        real aRoe = sqrt(asqrRoe);
        real vn = dot3(vRoe, n);
        real incU123N = incU[1] * n[0] + incU[2] * n[1] + incU[3] * n[2];
        real a23[3];
        for (int d = 0; d < 3; d++)
            a23[d] = incU[1 + d] - incU[0] * vRoe[d];
        real a23n = dot3(a23, n);
        for (int d = 0; d < 3; d++)
            a23[d] -= n[d] * a23n; // tangential part
        real incU4b = incU[4] - dot3(a23, vRoe);
        real alpha1 = (gamma - 1) / asqrRoe * (incU[0] * (HRoe - vn * vn) + vn * incU123N - incU4b);
        real alpha0 = (incU[0] * (vn + aRoe) - incU123N - aRoe * alpha1) / (2 * aRoe);
        real alpha4 = incU[0] - (alpha0 + alpha1);
        alpha0 *= l0, alpha1 *= l123, alpha4 *= l4;
        for (int d = 0; d < 3; d++)
            a23[d] *= l123;
        incF[0] += alpha0 + alpha1 + alpha4;
        incF[4] += (HRoe - vn * aRoe) * alpha0 + 0.5 * vsqrRoe * alpha1 + (HRoe + vn * aRoe) * alpha4 + dot3(a23, vRoe);
        for (int d = 0; d < 3; d++)
            incF[1 + d] += (vRoe[d] - aRoe * n[d]) * alpha0 + (vRoe[d] + aRoe * n[d]) * alpha4 + vRoe[d] * alpha1 + a23[d];
        for (int j = 5; j < nv; j++)
            incF[j] += incU[j] * l123;
    }

    // EulerEvaluator.hpp:1100-1158 fluxJacobian0_Right_Times_du with useRoeTerm != 0:
    // dF = (omitF ? 0 : A(U; n) dU) + RoeFluxIncFDiff(dU; Roe(U, UOther), s l0, s l123, s l4) + s lambdaVis dU,  s = incFsign
    void fluxJacRoeTimesDu(const real *U, const real *UOther, const real n[3], const real *dU, real lamVis, real l0, real l123, real l4,
                           int incFsign, bool omitF, real *dF) const
    {
        int nv = es.nVars;
        if (omitF)
            for (int j = 0; j < nv; j++)
                dF[j] = 0;
        else
            fluxJacTimesDu(U, n, dU, 0.0, dF);
        roeFluxIncFDiff(U, UOther, n, dU, incFsign * l0, incFsign * l123, incFsign * l4, dF);
        for (int j = 0; j < nv; j++)
            dF[j] += incFsign * lamVis * dU[j];
    }

    // the flux increment of neighbour o of cell c across face f (UpdateSGS / LUSGSMatrixVec, EulerEvaluator.hxx:226-247):
    // the scalar form with lambdaFace, or with useRoeJacobian the Roe form with lambda0 / lambda4 swapped on side 1
    void neighbourFInc(long c, long f, long o, const real *u, const real *dU, real *dF) const
    {
        int nv = es.nVars;
        int side = sideOf(c, f);
        real n[3];
        for (int d = 0; d < 3; d++)
            n[d] = faceMeanNorm[f * 3 + d] * (side ? -1 : 1);
        if (jacMode == 2)
        {
            real l0 = side ? lambdaFace4[f] : lambdaFace0[f], l4 = side ? lambdaFace0[f] : lambdaFace4[f];
            fluxJacRoeTimesDu(u + o * nv, u + c * nv, n, dU, lambdaFaceVis[f], l0, lambdaFace123[f], l4, -1, false, dF);
        }
        else
            fluxJacTimesDu(u + o * nv, n, dU, lambdaFace[f], dF);
    }

    // generateBoundaryValue with linMode 1 (EvaluateDt.hxx:1743-1835, generateBV_InviscidWall :2199-2214 and
    // generateBV_ViscousWall :2241-2270 up to their linMode return): the ghost's derivative, column-major nv x nv
    void bcLinear(int type, const real n[3], real *J) const
    {
        int nv = es.nVars;
        for (int i = 0; i < nv * nv; i++)
            J[i] = 0;
        if (type == 3 || type == 9) // BCWallInvis, BCSym: momentum mirrored
        {
            for (int i = 0; i < nv; i++)
                J[i * nv + i] = 1;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    J[(1 + b) * nv + 1 + a] -= 2 * n[a] * n[b];
        }
        else if (type == 2 || type == 4) // BCWall, BCWallIsothermal: momentum reversed
            for (int i = 0; i < nv; i++)
                J[i * nv + i] = (i >= 1 && i <= 3) ? -1 : 1;
        // far field, outflow and inflow types: zero
    }

    // JacobianDiagBlock::GetInvert (EulerJacobian.hpp:150-180): scale the rows by the inverse diagonal, invert by
    // Gauss-Jordan elimination with full pivoting, scale the columns back.  Row-major n x n.
    static bool invertBlock(int n, const real *A, real *Ainv)
    {
        real M[64], X[64], D[8];
        for (int i = 0; i < n; i++)
        {
            if (A[i * n + i] == 0)
                return false;
            D[i] = 1.0 / A[i * n + i];
        }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                M[i * n + j] = D[i] * A[i * n + j], X[i * n + j] = i == j ? 1 : 0;
        int colOf[8];
        for (int i = 0; i < n; i++)
            colOf[i] = i;
        for (int k = 0; k < n; k++)
        {
            int pr = k, pc = k;
            real best = -1;
            for (int i = k; i < n; i++)
                for (int j = k; j < n; j++)
                    if (abs(M[i * n + j]) > best)
                        best = abs(M[i * n + j]), pr = i, pc = j;
            if (!(best > 0))
                return false;
            for (int j = 0; j < n; j++)
            {
                std::swap(M[k * n + j], M[pr * n + j]);
                std::swap(X[k * n + j], X[pr * n + j]);
            }
            for (int i = 0; i < n; i++)
                std::swap(M[i * n + k], M[i * n + pc]);
            std::swap(colOf[k], colOf[pc]);
            real ip = 1.0 / M[k * n + k];
            for (int j = 0; j < n; j++)
                M[k * n + j] *= ip, X[k * n + j] *= ip;
            for (int i = 0; i < n; i++)
            {
                if (i == k)
                    continue;
                real fct = M[i * n + k];
                if (fct == 0)
                    continue;
                for (int j = 0; j < n; j++)
                    M[i * n + j] -= fct * M[k * n + j], X[i * n + j] -= fct * X[k * n + j];
            }
        }
        // M P = I after the column swaps P, so (D A)^-1 = P X: row colOf[k] of the inverse is row k of X
        real Y[64];
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                Y[colOf[k] * n + j] = X[k * n + j];
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                Ainv[i * n + j] = Y[i * n + j] * D[j];
        return true;
    }

    // LUSGSMatrixInit (EulerEvaluator.hxx:37-159) in block mode (jacMode 1 / 2): jd [nCell][2][nv][nv] receives
    // the block (row-major) and its inverse.  With useRoeJacobian every face adds (alpha/2)(A_f/V_c) times the
    // Roe dissipation matrix of (u_c, u_j) plus lambdaVis I (omitF, incFsign +1), a boundary face also the
    // Roe-form flux Jacobian of the ghost times the linearised ghost (:98-124); the diagonal then gains
    // 1/dTau + 1/dt.  Without it the block is the scalar diagonal.  The SA source Jacobian diagonal
    // (EvaluateDt.hxx:1650-1654, diagonal in block mode too) is added with alphaDiag.  Returns false on a
    // singular block.
    bool lusgsInitBlock(const real *dTau, real dt, real alphaDiag, const real *u, real *jd) const
    {
        int nv = es.nVars;
        bool ok = true;
#pragma omp parallel for schedule(static) reduction(&& : ok)
        for (long c = 0; c < nCell; c++)
        {
            real B[64] = {0};
            real fp = 1.0 / dTau[c] + 1.0 / dt;
            const real *uc = u + c * nv;
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                fp += (0.5 * alphaDiag) * faceArea[f] * lambdaFace[f] / vol[c];
                if (jacMode != 2)
                    continue;
                long o = otherOf(c, f);
                int side = sideOf(c, f);
                real n[3];
                for (int d = 0; d < 3; d++)
                    n[d] = faceMeanNorm[f * 3 + d] * (side ? -1 : 1);
                real uj[8];
                bool bnd = o < 0;
                if (bnd)
                {
                    if (!bcValue(zoneType(f), faceZone[f], uc, n, uj))
                        std::copy(uc, uc + nv, uj);
                }
                else
                    std::copy(u + o * nv, u + o * nv + nv, uj);
                real l0 = side ? lambdaFace4[f] : lambdaFace0[f], l4 = side ? lambdaFace0[f] : lambdaFace4[f];
                real cf = (0.5 * alphaDiag) * faceArea[f] / vol[c];
                real JII[64], JIJ[64];
                for (int i = 0; i < nv; i++)
                {
                    real e[8] = {0}, col[8];
                    e[i] = 1;
                    fluxJacRoeTimesDu(uc, uj, n, e, lambdaFaceVis[f], l0, lambdaFace123[f], l4, +1, true, col);
                    for (int r = 0; r < nv; r++)
                        JII[r * nv + i] = col[r];
                    if (bnd)
                    {
                        fluxJacRoeTimesDu(uj, uc, n, e, lambdaFaceVis[f], l0, lambdaFace123[f], l4, -1, false, col);
                        for (int r = 0; r < nv; r++)
                            JIJ[r * nv + i] = col[r];
                    }
                }
                if (bnd)
                {
                    real JBC[64]; // column-major
                    bcLinear(zoneType(f), n, JBC);
                    for (int r = 0; r < nv; r++)
                        for (int i = 0; i < nv; i++)
                        {
                            real acc = 0;
                            for (int l = 0; l < nv; l++)
                                acc += JIJ[r * nv + l] * JBC[i * nv + l];
                            B[r * nv + i] += cf * acc;
                        }
                }
                for (int i = 0; i < nv * nv; i++)
                    B[i] += cf * JII[i];
            }
            for (int i = 0; i < nv; i++)
            {
                if (jacMode == 2)
                    B[i * nv + i] += 1.0 / dTau[c] + 1.0 / dt;
                else
                    B[i * nv + i] = fp;
                if (nv >= 6 && !jSource.empty())
                    B[i * nv + i] += alphaDiag * jSource[c * nv + i];
            }
            real *out = jd + c * 2 * nv * nv;
            std::copy(B, B + nv * nv, out);
            ok = invertBlock(nv, B, out + nv * nv) && ok;
        }
        return ok;
    }

    // JDiag^-1 b (JacobianDiagBlock::MatVecLeftInvert) for the jdiag layout of the mode
    void jdSolve(long c, const real *jdiag, const real *b, real *x) const
    {
        int nv = es.nVars;
        if (jacMode == 0)
        {
            for (int v = 0; v < nv; v++)
                x[v] = b[v] / jdiag[nv >= 6 ? c * nv + v : c];
            return;
        }
        const real *Ai = jdiag + c * 2 * nv * nv + nv * nv;
        for (int r = 0; r < nv; r++)
        {
            real acc = 0;
            for (int l = 0; l < nv; l++)
                acc += Ai[r * nv + l] * b[l];
            x[r] = acc;
        }
    }
    // JDiag x (JacobianDiagBlock::MatVecLeft)
    void jdMul(long c, const real *jdiag, const real *x, real *y) const
    {
        int nv = es.nVars;
        if (jacMode == 0)
        {
            for (int v = 0; v < nv; v++)
                y[v] = jdiag[nv >= 6 ? c * nv + v : c] * x[v];
            return;
        }
        const real *A = jdiag + c * 2 * nv * nv;
        for (int r = 0; r < nv; r++)
        {
            real acc = 0;
            for (int l = 0; l < nv; l++)
                acc += A[r * nv + l] * x[l];
            y[r] = acc;
        }
    }

    // LUSGSMatrixToJacobianLU (EulerEvaluator.hxx:290-359) and JacobianLocalLU::InPlaceDecompose
    // (Solver/Direct.hpp:312-405, InPlaceDecomposeV1) for iluCode 0 (the face-neighbour pattern, no fill), natural
    // ordering and one partition.  luOff [nCell][nf][nv][nv]: per face slot the block (alpha/2)(A_f/V_c) dF/dU_o,
    // after the decomposition L (lower neighbours, o < c) or U (upper neighbours); luDinv [nCell][nv][nv]: the
    // inverted pivots.  Slots of boundary faces and of a cell's periodic image of itself stay zero.
    std::vector<real> luOff, luDinv;
    int slotOf(long c, long o) const
    {
        for (int k = 0; k < nf; k++)
        {
            long f = cell2face[c * nf + k];
            if (otherOf(c, f) == o)
                return k;
        }
        return -1;
    }
    static void blockMulSub(int n, const real *A, const real *B, real *C) // C -= A B
    {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
            {
                real acc = 0;
                for (int l = 0; l < n; l++)
                    acc += A[i * n + l] * B[l * n + j];
                C[i * n + j] -= acc;
            }
    }
    bool jacobianLU(real alphaDiag, const real *u, const real *jdiag)
    {
        int nv = es.nVars, nn = nv * nv;
        luOff.assign(nCell * nf * nn, 0);
        luDinv.assign(nCell * nn, 0);
        std::vector<real> D(nCell * nn, 0);
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nCell; c++)
        {
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                long o = otherOf(c, f);
                if (o < 0 || o == c)
                    continue;
                real cf = (0.5 * alphaDiag) * faceArea[f] / vol[c];
                real *B = &luOff[(c * nf + k) * nn];
                for (int i = 0; i < nv; i++)
                {
                    real e[8] = {0}, col[8];
                    e[i] = 1;
                    neighbourFInc(c, f, o, u, e, col);
                    for (int r = 0; r < nv; r++)
                        B[r * nv + i] = cf * col[r];
                }
            }
            real e[8] = {0}, y[8];
            for (int i = 0; i < nv; i++) // JDiag.getValue (the scalar diagonal as a matrix)
            {
                std::fill(e, e + 8, 0.0);
                e[i] = 1;
                jdMul(c, jdiag, e, y);
                for (int r = 0; r < nv; r++)
                    D[c * nn + r * nv + i] = y[r];
            }
        }
        bool ok = true;
        for (long i = 0; i < nCell; i++)
        {
            // lower neighbours in ascending index order
            std::vector<std::pair<long, int>> low, upp;
            for (int k = 0; k < nf; k++)
            {
                long o = otherOf(i, cell2face[i * nf + k]);
                if (o >= 0 && o != i)
                    (o < i ? low : upp).push_back({o, k});
            }
            std::sort(low.begin(), low.end());
            for (size_t a = 0; a < low.size(); a++)
            {
                long j = low[a].first;
                real *Lij = &luOff[(i * nf + low[a].second) * nn];
                for (size_t b = 0; b < a; b++) // k in lower(i) with k < j and j in upper(k)
                {
                    long k = low[b].first;
                    int sk = slotOf(k, j);
                    if (sk >= 0)
                        blockMulSub(nv, &luOff[(i * nf + low[b].second) * nn], &luOff[(k * nf + sk) * nn], Lij);
                }
                real T[64];
                std::copy(Lij, Lij + nn, T);
                for (int r = 0; r < nv * nv; r++)
                    Lij[r] = 0;
                blockMulSub(nv, T, &luDinv[j * nn], Lij); // Lij = -(-T Dinv_j) = T Dinv_j
                for (int r = 0; r < nn; r++)
                    Lij[r] = -Lij[r];
            }
            real *Di = &D[i * nn];
            for (auto &lk : low) // D_i -= L_ik U_ki
            {
                int si = slotOf(lk.first, i);
                if (si >= 0)
                    blockMulSub(nv, &luOff[(i * nf + lk.second) * nn], &luOff[(lk.first * nf + si) * nn], Di);
            }
            ok = invertBlock(nv, Di, &luDinv[i * nn]) && ok;
            for (auto &uj : upp) // U_ij -= L_ik U_kj over k in lower(i) adjacent to j
            {
                real *Uij = &luOff[(i * nf + uj.second) * nn];
                for (auto &lk : low)
                {
                    int sk = slotOf(lk.first, uj.first);
                    if (sk >= 0)
                        blockMulSub(nv, &luOff[(i * nf + lk.second) * nn], &luOff[(lk.first * nf + sk) * nn], Uij);
                }
            }
        }
        return ok;
    }

    // LUSGSMatrixSolveJacobianLU (EulerEvaluator.hxx:838-927) with JacobianLocalLU::Solve (Direct.hpp:487-540):
    // bBuf = rhs - A uInc (rhs alone when uIncIsZero), uIncNew = (LU)^-1 bBuf (+ uInc); sumInc = |uIncNew| column sums
    // before adding uInc
    void solveJacobianLU(real alphaDiag, const real *rhs, const real *u, const real *uInc, real *uIncNew, const real *jdiag, bool uIncIsZero,
                         real *sumInc) const
    {
        int nv = es.nVars, nn = nv * nv;
        std::vector<real> b(nCell * nv);
        if (uIncIsZero)
            std::copy(rhs, rhs + nCell * nv, b.begin());
        else
        {
            lusgsMatVec(alphaDiag, u, uInc, jdiag, b.data());
            for (long i = 0; i < nCell * nv; i++)
                b[i] = rhs[i] - b[i];
        }
        std::vector<real> x(nCell * nv);
        for (long i = 0; i < nCell; i++)
        {
            for (int v = 0; v < nv; v++)
                x[i * nv + v] = b[i * nv + v];
            for (int k = 0; k < nf; k++)
            {
                long o = otherOf(i, cell2face[i * nf + k]);
                if (o < 0 || o >= i)
                    continue;
                const real *L = &luOff[(i * nf + k) * nn];
                for (int r = 0; r < nv; r++)
                    for (int l = 0; l < nv; l++)
                        x[i * nv + r] -= L[r * nv + l] * x[o * nv + l];
            }
        }
        for (long i = nCell - 1; i >= 0; i--)
        {
            for (int k = 0; k < nf; k++)
            {
                long o = otherOf(i, cell2face[i * nf + k]);
                if (o < 0 || o <= i)
                    continue;
                const real *U = &luOff[(i * nf + k) * nn];
                for (int r = 0; r < nv; r++)
                    for (int l = 0; l < nv; l++)
                        x[i * nv + r] -= U[r * nv + l] * x[o * nv + l];
            }
            real t[8];
            const real *Di = &luDinv[i * nn];
            for (int r = 0; r < nv; r++)
            {
                real acc = 0;
                for (int l = 0; l < nv; l++)
                    acc += Di[r * nv + l] * x[i * nv + l];
                t[r] = acc;
            }
            for (int r = 0; r < nv; r++)
                x[i * nv + r] = t[r];
        }
        for (int v = 0; v < nv; v++)
            sumInc[v] = 0;
        for (long i = 0; i < nCell; i++)
            for (int v = 0; v < nv; v++)
            {
                sumInc[v] += abs(x[i * nv + v]);
                uIncNew[i * nv + v] = x[i * nv + v] + (uIncIsZero ? 0.0 : uInc[i * nv + v]);
            }
    }

    // EulerEvaluator.hxx:550-693 UpdateSGS (sequential, natural cell order)
    void updateSGS(real alphaDiag, const real *rhs, const real *u, const real *uInc, real *uIncNew, const real *jdiag, bool forward,
                   bool gsUpdate, bool uIncIsZero, real *sumInc) const
    {
        int nv = es.nVars;
        for (int v = 0; v < nv; v++)
            sumInc[v] = 0;
        for (long s = 0; s < nCell; s++)
        {
            long c = forward ? s : nCell - 1 - s;
            real buf[8];
            for (int v = 0; v < nv; v++)
                buf[v] = rhs[c * nv + v];
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                long o = otherOf(c, f);
                if (o < 0 || o == c)
                    continue;
                bool useNew = gsUpdate && (forward ? (o < c) : (o > c));
                if (uIncIsZero && !useNew)
                    continue;
                const real *dU = useNew ? uIncNew + o * nv : uInc + o * nv;
                real dF[8];
                neighbourFInc(c, f, o, u, dU, dF);
                for (int v = 0; v < nv; v++)
                    buf[v] -= (0.5 * alphaDiag) * faceArea[f] / vol[c] * dF[v];
            }
            real x[8];
            jdSolve(c, jdiag, buf, x);
            for (int v = 0; v < nv; v++)
            {
                real old = uIncNew[c * nv + v];
                uIncNew[c * nv + v] = x[v];
                sumInc[v] += abs(uIncNew[c * nv + v] - old);
            }
        }
    }

    // EulerEvaluator.hxx:376-529 UpdateLUSGSForward / UpdateLUSGSBackward (sequential, natural cell order).
    // Forward: uIncNew_c = D_c^-1 (rhs_c - sum over lower neighbours of (alpha/2)(A_f/V_c) dF(uInc_o));
    // backward: uIncNew_c += D_c^-1 (- sum over upper neighbours of the same).  uInc may alias uIncNew
    // (the reference's callers pass one array), which turns the neighbour reads into Gauss-Seidel reads.
    void updateLUSGS(real alphaDiag, const real *rhs, const real *u, const real *uInc, real *uIncNew, const real *jdiag, bool forward) const
    {
        int nv = es.nVars;
        for (long s = 0; s < nCell; s++)
        {
            long c = forward ? s : nCell - 1 - s;
            real buf[8];
            for (int v = 0; v < nv; v++)
                buf[v] = forward ? rhs[c * nv + v] : 0.0;
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                long o = otherOf(c, f);
                if (o < 0 || !(forward ? (o < c) : (o > c)))
                    continue;
                real dF[8];
                neighbourFInc(c, f, o, u, uInc + o * nv, dF);
                for (int v = 0; v < nv; v++)
                    buf[v] -= (0.5 * alphaDiag) * faceArea[f] / vol[c] * dF[v];
            }
            real x[8];
            jdSolve(c, jdiag, buf, x);
            for (int v = 0; v < nv; v++)
                uIncNew[c * nv + v] = forward ? x[v] : uIncNew[c * nv + v] + x[v];
        }
    }

    // EulerEvaluator.hxx:175-274 LUSGSMatrixVec
    void lusgsMatVec(real alphaDiag, const real *u, const real *uInc, const real *jdiag, real *AuInc) const
    {
        int nv = es.nVars;
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nCell; c++)
        {
            real buf[8] = {0};
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[c * nf + k];
                long o = otherOf(c, f);
                if (o < 0)
                    continue;
                real dF[8];
                neighbourFInc(c, f, o, u, uInc + o * nv, dF);
                for (int v = 0; v < nv; v++)
                    buf[v] -= (0.5 * alphaDiag) * faceArea[f] / vol[c] * dF[v];
            }
            real y[8];
            jdMul(c, jdiag, uInc + c * nv, y);
            for (int v = 0; v < nv; v++)
                AuInc[c * nv + v] = y[v] - buf[v];
        }
    }

    // transpose of fluxJacTimesDu: out = (dF/dU at U along n, minus lambda I)^T y, written as the reverse
    // sweep of the same statements (adjoint LU-SGS operator, no reference counterpart)
    void fluxJacTransposeTimes(const real *U, const real n[3], const real *y, real lambdaMain, real *out) const
    {
        int nv = es.nVars;
        real gamma = es.gamma;
        real ir = 1.0 / U[0];
        real velo[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
        real p, H, asqr;
        idealGasThermal(U[4], U[0], dot3(velo, velo), gamma, p, asqr, H);
        real vn = dot3(velo, n);
        for (int j = 0; j < nv; j++)
            out[j] = -lambdaMain * y[j] + vn * (j >= 1 ? y[j] : 0.0);
        real bvn = 0, bp = 0;
        for (int d = 0; d < 3; d++)
        {
            out[1 + d] += n[d] * y[0];
            bvn += U[1 + d] * y[1 + d];
            bp += n[d] * y[1 + d];
        }
        bp += vn * y[4];
        bvn += (U[4] + p) * y[4];
        for (int j = 5; j < nv; j++)
            bvn += U[j] * y[j];
        out[4] += (gamma - 1) * bp;
        for (int d = 0; d < 3; d++)
        {
            real bv = n[d] * bvn - 0.5 * (gamma - 1) * U[1 + d] * bp;
            out[1 + d] += -0.5 * (gamma - 1) * velo[d] * bp + ir * bv;
            out[0] += -U[1 + d] * ir * ir * bv;
        }
    }

    // transpose of LUSGSMatrixVec: (A^T y)_q = D_q y_q + sum_c w_cq (J_q(n_cq) - lambda)^T y_c with
    // w_cq = alpha A_f / (2 V_c) and n_cq the normal out of the neighbour c
    void lusgsMatVecT(real alphaDiag, const real *u, const real *y, const real *jdiag, real *ATy) const
    {
        int nv = es.nVars;
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nCell; q++)
        {
            real buf[8] = {0};
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[q * nf + k];
                long c = otherOf(q, f);
                if (c < 0)
                    continue;
                int side = sideOf(q, f);
                real n[3];
                for (int d = 0; d < 3; d++)
                    n[d] = -faceMeanNorm[f * 3 + d] * (side ? -1 : 1);
                real t[8];
                fluxJacTransposeTimes(u + q * nv, n, y + c * nv, lambdaFace[f], t);
                for (int v = 0; v < nv; v++)
                    buf[v] += (0.5 * alphaDiag) * faceArea[f] / vol[c] * t[v];
            }
            for (int v = 0; v < nv; v++)
                ATy[q * nv + v] = jdiag[nv >= 6 ? q * nv + v : q] * y[q * nv + v] + buf[v];
        }
    }

    // one Gauss-Seidel sweep on A^T y = b, sequential in natural cell order (the transposed UpdateSGS)
    void updateSGST(real alphaDiag, const real *b, const real *u, const real *y, real *yNew, const real *jdiag, bool forward, bool gsUpdate) const
    {
        int nv = es.nVars;
        for (long s = 0; s < nCell; s++)
        {
            long q = forward ? s : nCell - 1 - s;
            real buf[8];
            for (int v = 0; v < nv; v++)
                buf[v] = b[q * nv + v];
            for (int k = 0; k < nf; k++)
            {
                long f = cell2face[q * nf + k];
                long c = otherOf(q, f);
                if (c < 0 || c == q)
                    continue;
                bool useNew = gsUpdate && (forward ? (c < q) : (c > q));
                int side = sideOf(q, f);
                real n[3];
                for (int d = 0; d < 3; d++)
                    n[d] = -faceMeanNorm[f * 3 + d] * (side ? -1 : 1);
                real t[8];
                fluxJacTransposeTimes(u + q * nv, n, (useNew ? yNew : y) + c * nv, lambdaFace[f], t);
                for (int v = 0; v < nv; v++)
                    buf[v] -= (0.5 * alphaDiag) * faceArea[f] / vol[c] * t[v];
            }
            for (int v = 0; v < nv; v++)
                yNew[q * nv + v] = buf[v] / jdiag[nv >= 6 ? q * nv + v : q];
        }
    }

    // Pressure force along dir on the boundary faces of one zone:
    //   J = sum_f sum_g |J|_g w_g p(U_L(x_g)) (n_g . dir),  U_L = u + phi . uRec of the face's cell
    // (the reconstructed state the boundary flux starts from, boundaryFaceFlux above), with its gradient
    // with respect to u and uRec (objective of the adjoint, no reference counterpart)
    real pressureForce(int zone, const real *dir, const real *u, const real *uRec, real *gU, real *gRec) const
    {
        int nv = es.nVars;
        real gamma = es.gamma;
        std::vector<real> T0(4 * NDOF);
        real J = 0;
        if (gU)
            std::fill(gU, gU + nCell * nv, 0.0);
        if (gRec)
            std::fill(gRec, gRec + nCell * R * nv, 0.0);
        for (long f = 0; f < nFace; f++)
        {
            if (face2cell[f * 2 + 1] >= 0 || faceZone[f] != zone)
                continue;
            long c0 = face2cell[f * 2 + 0];
            for (int g = 0; g < nGf; g++)
            {
                real pq[3], w;
                quadPoint(faceType, vs.intOrder, g, pq, w);
                const real *n = &faceNorm[(f * nGf + g) * 3];
                const real *p0 = &facePP[(f * nGf + g) * 3];
                diffBase(c0, p0, T0.data(), 1, true);
                real UL[8];
                for (int v = 0; v < nv; v++)
                {
                    real a = 0;
                    for (int j = 0; j < R; j++)
                        a += T0[1 + j] * uRec[(c0 * R + j) * nv + v];
                    UL[v] = u[c0 * nv + v] + a;
                }
                real vel[3] = {UL[1] / UL[0], UL[2] / UL[0], UL[3] / UL[0]};
                real p = (gamma - 1) * (UL[4] - 0.5 * UL[0] * dot3(vel, vel));
                real wt = faceJDet[f * nGf + g] * w * dot3(n, dir);
                J += wt * p;
                real dp[8] = {0};
                dp[0] = (gamma - 1) * 0.5 * dot3(vel, vel);
                for (int d = 0; d < 3; d++)
                    dp[1 + d] = -(gamma - 1) * vel[d];
                dp[4] = gamma - 1;
                for (int v = 0; v < nv; v++)
                {
                    if (gU)
                        gU[c0 * nv + v] += wt * dp[v];
                    if (gRec)
                        for (int j = 0; j < R; j++)
                            gRec[(c0 * R + j) * nv + v] += wt * T0[1 + j] * dp[v];
                }
            }
        }
        return J;
    }

    // EulerEvaluator.hxx:1039-1143 InitializeUDOF: 2 = isentropic vortex (chi given), 3 = Taylor-Green (M0 = 0.1)
    void initField(int kind, real chi, real *u) const
    {
        int nv = es.nVars;
        real gamma = es.gamma;
        for (long c = 0; c < nCell; c++)
        {
            real um[8] = {0};
            for (int g = 0; g < nGc; g++)
            {
                real pq[3], w;
                quadPoint(cellType, vs.intOrder, g, pq, w);
                const real *x = &cellPP[(c * nGc + g) * 3];
                real inc[8] = {0};
                if (kind == 2)
                {
                    // SpecialFields.hpp:42-77 IsentropicVortex10 at t = 0
                    real xyc = 5;
                    real px = x[0] - floor(x[0] / 10) * 10, py = x[1] - floor(x[1] / 10) * 10;
                    real r = sqrt(sqr(px - xyc) + sqr(py - xyc));
                    real dT = -(gamma - 1) / (8 * gamma * sqr(pi)) * sqr(chi) * exp(1 - sqr(r));
                    real dux = chi / 2 / pi * exp((1 - sqr(r)) / 2) * -(py - xyc);
                    real duy = chi / 2 / pi * exp((1 - sqr(r)) / 2) * +(px - xyc);
                    real T = dT + 1, ux = dux + 1, uy = duy + 1;
                    real rho = pow(T, 1 / (gamma - 1));
                    real p = T * rho;
                    inc[0] = rho, inc[1] = rho * ux, inc[2] = rho * uy, inc[4] = 0.5 * (sqr(ux) + sqr(uy)) * rho + p / (gamma - 1);
                }
                else
                {
                    real M0 = 0.1;
                    real ux = sin(x[0]) * cos(x[1]) * cos(x[2]);
                    real uy = -cos(x[0]) * sin(x[1]) * cos(x[2]);
                    real p = 1. / (gamma * sqr(M0)) + 1. / 16 * ((cos(2 * x[0]) + cos(2 * x[1])) * (2 + cos(2 * x[2])));
                    real rho = gamma * sqr(M0) * p;
                    inc[0] = rho, inc[1] = rho * ux, inc[2] = rho * uy, inc[4] = 0.5 * (sqr(ux) + sqr(uy)) * rho + p / (gamma - 1);
                }
                for (int v = 0; v < nv; v++)
                    um[v] += inc[v] * cellJDet[c * nGc + g] * w;
            }
            for (int v = 0; v < nv; v++)
                u[c * nv + v] = um[v] / vol[c];
        }
    }
};
} // namespace orc

using namespace orc;

#ifdef ORC_OPCOUNT
// the counting build: the same entry points with the counting scalar in place of double (one double in
// a struct: the same calling convention, so the ctypes binding is unchanged)
#define double real
#endif
extern "C"
{
    void *orc_create(int dim, int cellType, int faceType, long nNode, const double *coords, long nCell, int nvert, const long *cell2node,
                     const double *cellShift, long nFace, int nfv, const long *face2node, const double *faceShift, const long *face2cell,
                     const int *faceZone, const double *facePShift, int nf, const long *cell2face, const OrcVRSettings *vs,
                     const OrcEulerSettings *es)
    {
        auto *o = new Oracle();
        o->dim = dim, o->cellType = cellType, o->faceType = faceType;
        o->nNode = nNode, o->nCell = nCell, o->nFace = nFace, o->nvert = nvert, o->nfv = nfv, o->nf = nf;
        o->coords.assign(coords, coords + nNode * 3);
        o->cell2node.assign(cell2node, cell2node + nCell * nvert);
        o->cellShift.assign(cellShift, cellShift + nCell * nvert * 3);
        o->face2node.assign(face2node, face2node + nFace * nfv);
        o->faceShift.assign(faceShift, faceShift + nFace * nfv * 3);
        o->face2cell.assign(face2cell, face2cell + nFace * 2);
        o->faceZone.assign(faceZone, faceZone + nFace);
        o->facePShift.assign(facePShift, facePShift + nFace * 3);
        o->cell2face.assign(cell2face, cell2face + nCell * nf);
        o->vs = *vs;
        o->es = *es;
        o->NDOF = nDofOf(dim, vs->maxOrder);
        o->R = o->NDOF - 1;
        return o;
    }
    void orc_destroy(void *h) { delete (Oracle *)h; }

    // wall distance at the cell Gauss points [nCell][nGc] (the SA model's dWall)
    void orc_set_wall_dist(void *h, const double *d)
    {
        Oracle *o = (Oracle *)h;
        o->dWall.assign(d, d + o->nCell * o->nGc);
    }

    // boundary table per face zone (zone 0 = interior): EulerBC.hpp:35-48 type codes, values [nZone][nVars]
    void orc_set_bc(void *h, int nZone, const int *type, const double *value, int nv)
    {
        Oracle *o = (Oracle *)h;
        o->bcType.assign(type, type + nZone);
        o->bcVal.assign(nZone * 8, 0.0);
        for (int z = 0; z < nZone; z++)
            for (int v = 0; v < nv && v < 8; v++)
                o->bcVal[z * 8 + v] = value[z * nv + v];
    }

    int orc_construct(void *h, const double *bcDirWeight, int nZone)
    {
        auto *o = (Oracle *)h;
        o->constructMetrics();
        o->constructBaseAndWeight(bcDirWeight, nZone);
        return o->constructRecCoeff();
    }

    void orc_sizes(void *h, long *out)
    {
        auto *o = (Oracle *)h;
        out[0] = o->NDOF, out[1] = o->R, out[2] = o->nGf, out[3] = o->nGc;
    }

    // copies a named internal array; returns its length (copies only if out != null)
    long orc_get(void *h, const char *name, double *out)
    {
        auto *o = (Oracle *)h;
        const std::vector<real> *v = nullptr;
        std::string n(name);
        if (n == "volume") v = &o->vol;
        else if (n == "cellBary") v = &o->cellBary;
        else if (n == "cellCent") v = &o->cellCent;
        else if (n == "cellHBox") v = &o->cellHBox;
        else if (n == "cellJDet") v = &o->cellJDet;
        else if (n == "smoothRatio") v = &o->smoothRatio;
        else if (n == "faceArea") v = &o->faceArea;
        else if (n == "cellPP") v = &o->cellPP;
        else if (n == "cellHMax") v = &o->cellHMax;
        else if (n == "jSource") v = &o->jSource;
        else if (n == "deltaLambdaCell") v = &o->deltaLambdaCell;
        else if (n == "faceCent") v = &o->faceCent;
        else if (n == "faceJDet") v = &o->faceJDet;
        else if (n == "facePP") v = &o->facePP;
        else if (n == "faceNorm") v = &o->faceNorm;
        else if (n == "faceMeanNorm") v = &o->faceMeanNorm;
        else if (n == "baseMoment") v = &o->baseMoment;
        else if (n == "faceWeight") v = &o->faceWeight;
        else if (n == "faceScale") v = &o->faceScale;
        else if (n == "matrixAAInvB") v = &o->AAInvB;
        else if (n == "vectorAInvB") v = &o->AInvb;
        else if (n == "matrixA") v = &o->matA;
        else if (n == "lambdaFace") v = &o->lambdaFace;
        else if (n == "lambdaFaceC") v = &o->lambdaFaceC;
        else if (n == "lambdaFaceVis") v = &o->lambdaFaceVis;
        else if (n == "luOff") v = &o->luOff;
        else if (n == "luDinv") v = &o->luDinv;
        else if (n == "lambdaFace0") v = &o->lambdaFace0;
        else if (n == "lambdaFace123") v = &o->lambdaFace123;
        else if (n == "lambdaFace4") v = &o->lambdaFace4;
        else if (n == "deltaLambdaCell") v = &o->deltaLambdaCell;
        if (!v)
            return -1;
        if (out)
            std::copy(v->begin(), v->end(), out);
        return (long)v->size();
    }

    void orc_set_delta_lambda(void *h, const double *dl)
    {
        auto *o = (Oracle *)h;
        o->deltaLambdaCell.assign(dl, dl + o->nCell);
    }

    void orc_init_field(void *h, int kind, double chi, double *u) { ((Oracle *)h)->initField(kind, chi, u); }

    void orc_vr_iter(void *h, const double *uRec, double *uRecNew, const double *u, int recordInc, int uRecIsZero)
    {
        ((Oracle *)h)->vrIterJacobi(uRec, uRecNew, u, recordInc, uRecIsZero);
    }

    // one SOR sweep in place (SORInstead)
    void orc_vr_iter_sor(void *h, double *uRec, const double *u) { ((Oracle *)h)->vrIterSOR(uRec, u); }

    void orc_eval_dt(void *h, const double *u, double CFL, double MaxDt, int useLocalDt, double *dt, double *dtMin)
    {
        ((Oracle *)h)->evaluateDt(u, CFL, MaxDt, useLocalDt, dt, dtMin);
    }

    void orc_eval_rhs(void *h, const double *u, const double *uRec, double *rhs, double *faceFlux)
    {
        ((Oracle *)h)->evaluateRHS(u, uRec, rhs, faceFlux);
    }
    // EvaluateRHS(rhs, JSource, u, uRecUnlim, uRec, uRecBeta, cellRHSAlpha, ...): jSource (may be null)
    // receives the source Jacobian diagonal [nCell][nv], fluxWall (may be null) the wall-flux integral [nv]
    void orc_eval_rhs_full(void *h, const double *u, const double *uRecUnlim, const double *uRec, const double *alpha, double *rhs,
                           double *jSource, double *fluxWall)
    {
        Oracle *o = (Oracle *)h;
        o->evaluateRHS(u, uRec, rhs, nullptr, uRecUnlim, alpha, fluxWall);
        if (jSource)
            std::copy(o->jSource.begin(), o->jSource.end(), jSource);
    }

    void orc_lusgs_init(void *h, const double *dTau, double dt, double alphaDiag, double *jdiag)
    {
        ((Oracle *)h)->lusgsInit(dTau, dt, alphaDiag, jdiag);
    }

    // LUSGSMatrixToJacobianLU with the decomposition (iluCode 0, natural ordering); 0, or -1 on a singular pivot
    int orc_jacobian_lu(void *h, double alphaDiag, const double *u, const double *jdiag)
    {
        return ((Oracle *)h)->jacobianLU(alphaDiag, u, jdiag) ? 0 : -1;
    }
    void orc_solve_jacobian_lu(void *h, double alphaDiag, const double *rhs, const double *u, const double *uInc, double *uIncNew,
                               const double *jdiag, int uIncIsZero, double *sumInc)
    {
        ((Oracle *)h)->solveJacobianLU(alphaDiag, rhs, u, uInc, uIncNew, jdiag, uIncIsZero != 0, sumInc);
    }

    // useScalarJacobian / useRoeJacobian as jacMode 0 / 1 / 2 (see Oracle::jacMode)
    void orc_set_jacobian_mode(void *h, int mode) { ((Oracle *)h)->jacMode = mode; }
    // block-mode LUSGSMatrixInit: jd [nCell][2][nv][nv]; returns 0, or -1 on a singular block
    int orc_lusgs_init_block(void *h, const double *dTau, double dt, double alphaDiag, const double *u, double *jd)
    {
        return ((Oracle *)h)->lusgsInitBlock(dTau, dt, alphaDiag, u, jd) ? 0 : -1;
    }

    void orc_update_sgs(void *h, double alphaDiag, const double *rhs, const double *u, const double *uInc, double *uIncNew,
                        const double *jdiag, int forward, int gsUpdate, int uIncIsZero, double *sumInc)
    {
        ((Oracle *)h)->updateSGS(alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward, gsUpdate, uIncIsZero, sumInc);
    }

    void orc_lusgs_matvec(void *h, double alphaDiag, const double *u, const double *uInc, const double *jdiag, double *AuInc)
    {
        ((Oracle *)h)->lusgsMatVec(alphaDiag, u, uInc, jdiag, AuInc);
    }

    void orc_lusgs_matvec_t(void *h, double alphaDiag, const double *u, const double *y, const double *jdiag, double *ATy)
    {
        ((Oracle *)h)->lusgsMatVecT(alphaDiag, u, y, jdiag, ATy);
    }

    void orc_update_sgs_t(void *h, double alphaDiag, const double *b, const double *u, const double *y, double *yNew, const double *jdiag,
                          int forward, int gsUpdate)
    {
        ((Oracle *)h)->updateSGST(alphaDiag, b, u, y, yNew, jdiag, forward, gsUpdate);
    }

    double orc_pressure_force(void *h, int zone, const double *dir, const double *u, const double *uRec, double *gU, double *gRec)
    {
        return ((Oracle *)h)->pressureForce(zone, dir, u, uRec, gU, gRec);
    }

    // single Riemann flux evaluation (Gas.hpp:1434 dispatcher), 5 conservative variables
    // uInc may equal uIncNew (in-place sweep, as the reference's callers use it)
    void orc_update_lusgs(void *h, double alphaDiag, const double *rhs, const double *u, const double *uInc, double *uIncNew,
                          const double *jdiag, int forward)
    {
        ((Oracle *)h)->updateLUSGS(alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward != 0);
    }
    void orc_riemann(int type, const double *UL, const double *UR, const double *ULm, const double *URm, const double *n, double gamma,
                     double dLambda, double fixScale, double incFScale, double *F, double *lam)
    {
        real vg[3] = {0, 0, 0};
        riemann(type, UL, UR, ULm, URm, vg, n, gamma, F, dLambda, fixScale, incFScale, lam[0], lam[1], lam[2]);
    }

    // GetRoeAverage(U, UOther) + RoeFluxIncFDiff (Gas.hpp:1149-1243): incF += the Roe dissipation of incU
    void orc_roe_fdiff(int nv, double gamma, const double *U, const double *UOther, const double *n, const double *incU, double l0, double l123,
                       double l4, double *incF)
    {
        Oracle::roeFluxIncFDiffS(nv, gamma, U, UOther, n, incU, l0, l123, l4, incF);
    }

    void orc_viscous_flux(const double *U, const double *GradU /*3 x 5 cons*/, const double *n, double gamma, double mu, double k, double Cp,
                          int adiabatic, double *Flux)
    {
        real GP[15];
        gradCons2Prim(5, U, GradU, GP, gamma);
        viscousFlux(5, U, GP, n, adiabatic, gamma, mu, k, Cp, Flux);
    }

    // point values u + D0 . uRec at the cell quadrature points: out[nCell][nGc][nv]
    void orc_cell_point_values(void *h, const double *u, const double *uRec, double *out)
    {
        auto *o = (Oracle *)h;
        int nv = o->es.nVars, R = o->R, NDOF = o->NDOF;
#pragma omp parallel for schedule(static)
        for (long c = 0; c < o->nCell; c++)
        {
            std::vector<real> T(NDOF);
            for (int g = 0; g < o->nGc; g++)
            {
                o->diffBase(c, &o->cellPP[(c * o->nGc + g) * 3], T.data(), 1, true);
                for (int v = 0; v < nv; v++)
                {
                    real acc = u[c * nv + v];
                    for (int j = 0; j < R; j++)
                        acc += T[1 + j] * uRec[(c * R + j) * nv + v];
                    out[(c * o->nGc + g) * nv + v] = acc;
                }
            }
        }
    }

    // cell quadrature weights (intOrder rule of the cell element)
    void orc_cell_quad_weights(void *h, double *w)
    {
        auto *o = (Oracle *)h;
        for (int g = 0; g < o->nGc; g++)
        {
            real p[3];
            quadPoint(o->cellType, o->vs.intOrder, g, p, w[g]);
        }
    }
}
#ifdef ORC_OPCOUNT
#undef double
extern "C"
{
    // counts of the operations since the last reset: {add/sub, mul, div, sqrt, exp/pow/log/trig calls}
    void orc_opcount_reset() { orc_cnt::ctr() = orc_cnt::Counter{}; }
    void orc_opcount_get(uint64_t *out)
    {
        const orc_cnt::Counter &c = orc_cnt::ctr();
        out[0] = c.add, out[1] = c.mul, out[2] = c.div, out[3] = c.sqrt, out[4] = c.fn;
    }
}
#else

// ---------------------------------------------------------------------------
// Positivity-preserving increment limiting (5 conservative variables, the SA variable 6th).
// ---------------------------------------------------------------------------
namespace
{
const double kPPSmall = 1e-10, kPPVerySmall = 1e-200;

double ppRhoE(const double *u) { return u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]; }

// Gas.hpp:1750-1860 IdealGasGetCompressionRatioPressure, scheme 0 (quadratic in alpha, then decay)
double ppCompressionRatio(const double *u, const double *inc, double newRhoE, bool &bad)
{
    const double safety = 1 - 1e-5;
    double r[5], un[5];
    for (int i = 0; i < 5; i++)
        r[i] = inc[i], un[i] = u[i] + inc[i];
    double m2 = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
    double rhoEOld = u[4] - m2 / (u[0] + kPPVerySmall) * 0.5;
    newRhoE = max(kPPSmall * rhoEOld, newRhoE);
    double rhoENew = un[4] - (un[1] * un[1] + un[2] * un[2] + un[3] * un[3]) / (un[0] + kPPVerySmall) * 0.5;
    double alpha = (rhoEOld - newRhoE) / max(-rhoENew + rhoEOld, kPPVerySmall);
    if (rhoENew > rhoEOld)
        alpha = 1;
    alpha = max(min(alpha, 1.), 0.);
    double c0 = 2 * u[4] * u[0] - m2 - 2 * u[0] * newRhoE;
    double c1 = 2 * u[4] * r[0] + 2 * u[0] * r[4] - 2 * (u[1] * r[1] + u[2] * r[2] + u[3] * r[3]) - 2 * r[0] * newRhoE;
    double c2 = 2 * r[4] * r[0] - (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    c2 += (c2 >= 0 ? 1 : -1) * kPPVerySmall;
    double dC = c1 * c1 - 4 * c0 * c2;
    if (dC <= -c0 * c0 * kPPSmall)
        bad = true;
    dC = max(0., dC);
    double aL = (-sqrt(dC) - c1) / (2 * c2);
    if (abs(c2) < 1e-10 * c0)
        alpha = abs(c1) < 1e-10 * c0 ? 0 : min(-c0 / c1, 1.);
    else
        alpha = min(aL, 1.);
    alpha = max(0., alpha) * safety;
    if (alpha < kPPSmall)
        alpha = 0;
    for (int i = 0; i < 5; i++)
        r[i] *= alpha;
    int it = 0;
    for (; it < 1000; it++)
    {
        double s[3] = {u[1] + r[1], u[2] + r[2], u[3] + r[3]};
        double ek = 0.5 * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) / (u[0] + r[0] + kPPVerySmall);
        if (r[4] + u[4] - ek < newRhoE)
        {
            for (int i = 0; i < 5; i++)
                r[i] *= 1 - 1e-2;
            alpha *= 1 - 1e-2;
        }
        else
            break;
    }
    if (it >= 1000)
        bad = true;
    return alpha;
}

// EulerEvaluator.hpp:1645-1773 CompressInc
void ppCompressInc(int nv, double gamma, const double *u, const double *inc, double rhoEps, double pEps, double *ret, bool &bad)
{
    for (int i = 0; i < nv; i++)
        ret[i] = inc[i];
    if (!(u[0] > 0))
        bad = true;
    if (u[0] + ret[0] <= rhoEps)
    {
        double f = (rhoEps - u[0]) / (ret[0] - kPPVerySmall);
        for (int i = 0; i < nv; i++)
            ret[i] *= f;
    }
    double rhoEint = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / (u[0] + kPPVerySmall);
    if (!(rhoEint > 0))
        bad = true;
    auto ekOf = [&]()
    {
        double s[3] = {u[1] + ret[1], u[2] + ret[2], u[3] + ret[3]};
        return 0.5 * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) / (u[0] + ret[0] + kPPVerySmall);
    };
    double rhoEintNew = u[4] + ret[4] - ekOf();
    if (rhoEintNew <= pEps)
    {
        double e = pEps / (gamma - 1);
        double m2 = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
        double c0 = 2 * u[4] * u[0] - m2 - 2 * u[0] * e;
        double c1 = 2 * u[4] * ret[0] + 2 * u[0] * ret[4] - 2 * (u[1] * ret[1] + u[2] * ret[2] + u[3] * ret[3]) - 2 * ret[0] * e;
        double c2 = 2 * ret[4] * ret[0] - (ret[1] * ret[1] + ret[2] * ret[2] + ret[3] * ret[3]);
        double dC = c1 * c1 - 4 * c0 * c2;
        if (!(dC > 0))
            bad = true;
        double alpha = max(0., min((-sqrt(max(dC, 0.)) - c1) / (2 * c2), 1.));
        for (int i = 0; i < nv; i++)
            ret[i] *= alpha * 0.99;
        for (int it = 0; it < 1000; it++)
        {
            if (ret[4] + u[4] - ekOf() < e)
                for (int i = 0; i < nv; i++)
                    ret[i] *= 1 - 1e-1;
            else
                break;
        }
        if (ret[4] + u[4] - ekOf() < e * 0.5)
            bad = true;
    }
    if (nv > 5 && u[5] + ret[5] < 0)
    {
        if (u[5] < 0)
            bad = true;
        double nu = max(1e-6, u[5] * exp(ret[5] / (u[5] + 1e-6)));
        ret[5] = nu - u[5];
    }
}
} // namespace

// Gas.hpp IdealGasGetCompressionRatioPressure, exported for its unit cases; *bad receives the quadratic's failure flag
extern "C" double orc_pp_compression_ratio(const double *u, const double *inc, double newRhoE, int *bad)
{
    bool b = false;
    double a = ppCompressionRatio(u, inc, newRhoE, b);
    if (bad)
        *bad = b;
    return a;
}

extern "C"
{
    // EulerEvaluator.hxx:1938-2062 EvaluateCellRHSAlpha (refRho, refP = refUPrim(0), refUPrim(I4));
    // returns 1 when an assertion of the reference would fire
    int orc_cell_rhs_alpha(long nCell, int nv, double gamma, const double *u, const double *res, double *alpha, double refRho, double refP,
                           double relax, int compress, double compressPower, int ppEpsIsRelaxed, int flag, long *nLimOut,
                           double *alphaMinOut)
    {
        double rhoEps = kPPSmall * refRho * 1e-1, pEps = kPPSmall * refP * 1e-1;
        const double safety = 1 - 1e-5;
        if (ppEpsIsRelaxed)
            pEps *= 0, rhoEps *= 0;
        long nLim = 0;
        double aMin = 1;
        bool bad = false;
        for (long c = 0; c < nCell; c++)
        {
            const double *uc = u + c * nv;
            double inc[5];
            for (int i = 0; i < 5; i++)
                inc[i] = res[c * nv + i];
            if (!(uc[0] >= rhoEps))
                bad = true;
            double aRho = 1, relRho = rhoEps * relax + uc[0] * (1 - relax);
            if (inc[0] < 0)
                aRho = min(1.0, (uc[0] - relRho) / (-inc[0] - kPPSmall * inc[0]));
            if (!(aRho >= 0 && aRho <= 1))
                bad = true;
            double un[5];
            for (int i = 0; i < 5; i++)
                inc[i] *= aRho, un[i] = uc[i] + inc[i];
            double pNew = ppRhoE(un) * (gamma - 1), pOld = ppRhoE(uc) * (gamma - 1);
            double relP = pEps;
            if (pNew < pOld)
                relP = pEps + (pOld - pEps) * (1 - relax);
            double aP = 1;
            if (pNew < relP)
                aP = min(aP, ppCompressionRatio(uc, inc, relP / (gamma - 1), bad));
            double a = aRho * aP;
            if (a < 1)
            {
                a = pow(a, compress * (int)round(compressPower));
                nLim++;
                a *= safety;
                aMin = min(aMin, a);
            }
            alpha[c] = a;
        }
        if (flag & 1)
            for (long c = 0; c < nCell; c++)
                if (alpha[c] < 1)
                    alpha[c] = aMin;
        if (flag & 2)
            for (long c = 0; c < nCell; c++)
                alpha[c] = aMin;
        *nLimOut = nLim, *alphaMinOut = aMin;
        return bad ? 1 : 0;
    }

    // EulerEvaluator.hxx:2064-2140 EvaluateCellRHSAlphaExpansion
    void orc_cell_rhs_alpha_expansion(long nCell, int nv, double gamma, const double *u, const double *res, double *alpha, double refRho,
                                      double refP, double alphaMin)
    {
        double rhoEps = kPPSmall * refRho * 1e-1, pEps = kPPSmall * refP * 1e-1;
        for (long c = 0; c < nCell; c++)
        {
            double un[5];
            for (int i = 0; i < 5; i++)
                un[i] = u[c * nv + i] + res[c * nv + i];
            if (ppRhoE(un) * (gamma - 1) < pEps || un[0] < rhoEps)
                alpha[c] = alphaMin;
        }
    }

    // EulerEvaluator.hpp:1795-1857 AddFixedIncrement: u += CompressInc(u, alpha inc)
    int orc_add_fixed_increment(long nCell, int nv, double gamma, double *u, const double *inc, double alpha, double refRho, double refP,
                                int ppEpsIsRelaxed, double *alphaFixMinOut)
    {
        double rhoEps = kPPSmall * refRho * 1e-1, pEps = kPPSmall * refP * 1e-1;
        if (ppEpsIsRelaxed)
            pEps *= kPPVerySmall, rhoEps *= kPPVerySmall;
        double fixMin = 1;
        bool bad = false;
        for (long c = 0; c < nCell; c++)
        {
            double a[8], comp[8];
            for (int i = 0; i < nv; i++)
                a[i] = inc[c * nv + i] * alpha;
            ppCompressInc(nv, gamma, u + c * nv, a, rhoEps, pEps, comp, bad);
            double na = abs(comp[0]) / abs(a[0]);
            if (abs(a[0]) < kPPVerySmall)
                na = 1.;
            fixMin = min(fixMin, na);
            for (int i = 0; i < nv; i++)
                u[c * nv + i] += comp[i];
        }
        *alphaFixMinOut = fixMin;
        return bad ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// WBAP_C limiter (3-D, 5 or 6 variables): DoCalculateSmoothIndicator (procedure 0) and DoLimiterWBAP_C
// with the WBAP-L2 biway (limiterBiwayAlter 0) and multiway (normWBAP false) functions, in the
// characteristic variables of EulerSolver.hxx:455-556.
// ---------------------------------------------------------------------------
namespace
{
// solve A X = B, A n x n (row-major, overwritten), B n x m (overwritten by X); Gauss-Jordan, partial pivoting
bool ocSolve(int n, int m, double *A, double *B)
{
    for (int c = 0; c < n; c++)
    {
        int piv = c;
        for (int r = c + 1; r < n; r++)
            if (abs(A[r * n + c]) > abs(A[piv * n + c]))
                piv = r;
        if (A[piv * n + c] == 0)
            return false;
        if (piv != c)
        {
            for (int j = 0; j < n; j++)
                std::swap(A[piv * n + j], A[c * n + j]);
            for (int j = 0; j < m; j++)
                std::swap(B[piv * m + j], B[c * m + j]);
        }
        double id = 1.0 / A[c * n + c];
        for (int j = 0; j < n; j++)
            A[c * n + j] *= id;
        for (int j = 0; j < m; j++)
            B[c * m + j] *= id;
        for (int r = 0; r < n; r++)
            if (r != c && A[r * n + c] != 0)
            {
                double f = A[r * n + c];
                for (int j = 0; j < n; j++)
                    A[r * n + j] -= f * A[c * n + j];
                for (int j = 0; j < m; j++)
                    B[r * m + j] -= f * B[c * m + j];
            }
    }
    return true;
}

// Geometric.hpp:135-160 NormBuildLocalBaseV (3-D): columns n, t1, t2
void ocNormBase(const double *n, double B[3][3])
{
    double t[3];
    if (abs(n[2]) < 0.9) // -(n x e_z)
        t[0] = -(n[1] * 1 - n[2] * 0), t[1] = -(n[2] * 0 - n[0] * 1), t[2] = -(n[0] * 0 - n[1] * 0);
    else // -(n x e_y)
        t[0] = -(n[1] * 0 - n[2] * 1), t[1] = -(n[2] * 0 - n[0] * 0), t[2] = -(n[0] * 1 - n[1] * 0);
    double tn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    for (int d = 0; d < 3; d++)
        t[d] /= tn;
    double s[3] = {n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2], n[0] * t[1] - n[1] * t[0]};
    double sn = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (int d = 0; d < 3; d++)
        B[d][0] = n[d], B[d][1] = t[d], B[d][2] = s[d] / sn;
}

// Gas.hpp:120-200 Euler eigenvectors of the state UC (5 conservative), right (R) and left (L)
void ocEigen(const double *UC, double gamma, double Rv[5][5], double Lv[5][5])
{
    double v[3] = {UC[1] / UC[0], UC[2] / UC[0], UC[3] / UC[0]};
    double vsq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    double p = (gamma - 1) * (UC[4] - 0.5 * UC[0] * vsq);
    double a2 = gamma * p / UC[0], a = sqrt(a2), H = (UC[4] + p) / UC[0];
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++)
            Rv[i][j] = Lv[i][j] = 0;
    Rv[0][0] = Rv[0][1] = Rv[0][4] = 1;
    Rv[2][2] = Rv[3][3] = 1;
    for (int d = 0; d < 3; d++)
        Rv[1 + d][0] = v[d], Rv[1 + d][1] = v[d], Rv[1 + d][4] = v[d];
    Rv[1][0] -= a, Rv[1][4] += a;
    Rv[4][0] = H - v[0] * a, Rv[4][4] = H + v[0] * a, Rv[4][1] = 0.5 * vsq;
    Rv[4][2] = v[1], Rv[4][3] = v[2];
    const double gb = gamma - 1;
    Lv[0][0] = H + a / gb * (v[0] - a), Lv[0][1] = -v[0] - a / gb, Lv[0][2] = -v[1], Lv[0][3] = -v[2], Lv[0][4] = 1;
    Lv[1][0] = -2 * H + 4 / gb * a2, Lv[1][1] = 2 * v[0], Lv[1][2] = 2 * v[1], Lv[1][3] = 2 * v[2], Lv[1][4] = -2;
    Lv[2][0] = v[1] * (-2 * a2 / gb), Lv[3][0] = v[2] * (-2 * a2 / gb);
    Lv[2][2] = Lv[3][3] = 2 * a2 / gb;
    Lv[4][0] = H - a / gb * (v[0] + a), Lv[4][1] = -v[0] + a / gb, Lv[4][2] = -v[1], Lv[4][3] = -v[2], Lv[4][4] = 1;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++)
            Lv[i][j] *= gb / (2 * a2);
}

// EulerSolver.hxx:466-505 fML / fMR: rows of `data` (one per DOF, nv values) to characteristic
// variables (left) or back (right), in the face's normal-aligned frame
void ocCharTransform(const double *uL, const double *uR, const double *n, double gamma, bool toChar, int rows, int nv, double *data)
{
    double UC[5], B[3][3];
    for (int i = 0; i < 5; i++)
        UC[i] = (uL[i] + uR[i]) * 0.5;
    ocNormBase(n, B);
    double m[3] = {UC[1], UC[2], UC[3]};
    for (int d = 0; d < 3; d++)
        UC[1 + d] = B[0][d] * m[0] + B[1][d] * m[1] + B[2][d] * m[2];
    double Rv[5][5], Lv[5][5], M[5][5];
    ocEigen(UC, gamma, Rv, Lv);
    if (toChar) // M = L; M(:, 1..3) = M(:, 1..3) B^T
        for (int i = 0; i < 5; i++)
        {
            M[i][0] = Lv[i][0], M[i][4] = Lv[i][4];
            for (int d = 0; d < 3; d++)
                M[i][1 + d] = Lv[i][1] * B[d][0] + Lv[i][2] * B[d][1] + Lv[i][3] * B[d][2];
        }
    else // M = R; M(1..3, :) = B M(1..3, :)
        for (int j = 0; j < 5; j++)
        {
            M[0][j] = Rv[0][j], M[4][j] = Rv[4][j];
            for (int d = 0; d < 3; d++)
                M[1 + d][j] = B[d][0] * Rv[1][j] + B[d][1] * Rv[2][j] + B[d][2] * Rv[3][j];
        }
    for (int r = 0; r < rows; r++)
    {
        double x[5], y[5];
        for (int i = 0; i < 5; i++)
            x[i] = data[r * nv + i];
        for (int i = 0; i < 5; i++)
        {
            y[i] = 0;
            for (int j = 0; j < 5; j++)
                y[i] += M[i][j] * x[j];
        }
        for (int i = 0; i < 5; i++)
            data[r * nv + i] = y[i];
    }
}

double ocSign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
const double kPDiP = 1e-50; // verySmallReal^(1/4)

// Limiters.hpp:432-466 FWBAP_L2_Biway (the fast version) for one entry: u1 (n + th^3) / (n + th^4) |sign(u2)|,
// th = u1 / (|u2| + eps) sign(u2)
double ocWbapBiway(double u1, double u2, double n)
{
    double fr = u1 / (abs(u2) + kPDiP) * ocSign(u2);
    double t1 = fr * fr * fr, t2 = (fr * fr) * (fr * fr);
    return u1 * (n + t1) / (n + t2) * abs(ocSign(u2));
}

// Limiters.hpp:361-385 FWBAP_L2_Multiway (the fast version) for one entry: others[0] is the cell's own value
double ocWbapMultiway(const double *others, int nOther, double n1)
{
    double up = 0, down = 0, cent = others[0];
    for (int q = 1; q < nOther; q++)
    {
        double ti = others[0] / (abs(others[q]) + kPDiP) * ocSign(others[q]);
        down += (ti * ti) * (ti * ti);
        up += ti * ti * ti;
        cent *= abs(ocSign(others[q]));
    }
    return cent * (up + n1) / (down + n1);
}
} // namespace

extern "C"
{
    // Gas.hpp IdealGas_EulerGasRight/LeftEigenVector of a conservative state (the characteristic projection of the
    // limiter), R and L row-major 5 x 5
    void orc_euler_eigen(const double *U, double gamma, double *R, double *L)
    {
        double Rv[5][5], Lv[5][5];
        ocEigen(U, gamma, Rv, Lv);
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++)
                R[i * 5 + j] = Rv[i][j], L[i * 5 + j] = Lv[i][j];
    }

    // the limiter functions on arrays of entries (the reference's FWBAP_L2_Biway / FWBAP_L2_Multiway test surface):
    // biway out[i] = f(u1[i], u2[i]); multiway out[i] = f(others[0][i], ..., others[nOther - 1][i]), others [nOther][n]
    void orc_wbap_l2_biway(long n, const double *u1, const double *u2, double nPar, double *out)
    {
        for (long i = 0; i < n; i++)
            out[i] = ocWbapBiway(u1[i], u2[i], nPar);
    }
    void orc_wbap_l2_multiway(long n, int nOther, const double *others, double n1, double *out)
    {
        double vals[16];
        for (long i = 0; i < n; i++)
        {
            for (int q = 0; q < nOther && q < 16; q++)
                vals[q] = others[(long)q * n + i];
            out[i] = ocWbapMultiway(vals, nOther < 16 ? nOther : 16, n1);
        }
    }

    // VariationalReconstruction_LimiterProcedure.hxx:40-108 DoCalculateSmoothIndicator, varsSee {0, 4}
    void orc_smooth_indicator(void *h, const double *u, const double *uRec, double *si)
    {
        Oracle *o = (Oracle *)h;
        const int nv = o->es.nVars, NDOF = o->NDOF, R = o->R;
        std::vector<double> T(NDOF * NDOF);
        const int vs[2] = {0, 4};
        for (long c = 0; c < o->nCell; c++)
        {
            double S[2][2] = {{0, 0}, {0, 0}};
            for (int k = 0; k < o->nf; k++)
            {
                long fp = o->cell2face[c * o->nf + k], f = fp;
                long other = o->otherOf(c, f);
                if (other < 0)
                    continue;
                double val[2][20 * 2], jmp[20 * 2], avg[20 * 2];
                for (int side = 0; side < 2; side++)
                {
                    long cc = side == 0 ? c : other;
                    int sd = o->face2cell[f * 2] == cc ? 0 : 1;
                    double p[3];
                    for (int d = 0; d < 3; d++)
                        p[d] = o->faceCent[f * 3 + d] + (sd ? o->facePShift[f * 3 + d] : 0.0);
                    o->diffBase(cc, p, T.data(), NDOF, true);
                    for (int r = 0; r < NDOF; r++)
                        for (int q = 0; q < 2; q++)
                        {
                            double a = 0;
                            for (int j = 0; j < R; j++)
                                a += T[r * NDOF + 1 + j] * uRec[(cc * R + j) * nv + vs[q]];
                            if (r == 0)
                                a += u[cc * nv + vs[q]];
                            val[side][r * 2 + q] = a;
                        }
                }
                for (int i = 0; i < NDOF * 2; i++)
                    avg[i] = (val[0][i] + val[1][i]) * 0.5, jmp[i] = (val[0][i] - val[1][i]) * 0.5;
                double IJ[4], IS[4];
                o->faceFunctional(f, jmp, 2, jmp, 2, NDOF, IJ);
                o->faceFunctional(f, avg, 2, avg, 2, NDOF, IS);
                for (int q = 0; q < 2; q++)
                    S[q][0] += IJ[q * 2 + q] * o->faceArea[f], S[q][1] += IS[q * 2 + q] * o->faceArea[f];
            }
            double sm = 0;
            for (int q = 0; q < 2; q++)
                sm = max(sm, abs(S[q][0] / (S[q][1] + 1e-200)));
            si[c] = sqrt(sm) * o->vs.maxOrder * o->vs.maxOrder;
        }
    }

    // VariationalReconstruction_LimiterProcedure.hxx:188-334 DoLimiterWBAP_C (putIntoNew), with
    // VariationalReconstruction.cpp:840-866 matrixSecondary and Limiters.hpp:361-470 WBAP-L2
    int orc_limiter_wbap_c(void *h, const double *u, const double *uRec, const double *si, double *uRecNew, double threshold, double nStd,
                           int ifAll, double gamma)
    {
        Oracle *o = (Oracle *)h;
        const int nv = o->es.nVars, NDOF = o->NDOF, R = o->R, P = o->vs.maxOrder;
        // matrixSecondary per interior face: [0] = DiffI^-1 DiffJ (for side 0), [1] = DiffJ^-1 DiffI (side 1)
        std::vector<double> sec((size_t)o->nFace * 2 * R * R, 0.0), T(NDOF * NDOF);
        for (long f = 0; f < o->nFace; f++)
        {
            long cL = o->face2cell[f * 2], cR = o->face2cell[f * 2 + 1];
            if (cR < 0)
                continue;
            std::vector<double> DI(R * R), DJ(R * R);
            double p[3];
            for (int d = 0; d < 3; d++)
                p[d] = o->faceCent[f * 3 + d];
            o->diffBase(cL, p, T.data(), NDOF, true);
            for (int r = 0; r < R; r++)
                for (int j = 0; j < R; j++)
                    DI[r * R + j] = T[(r + 1) * NDOF + 1 + j];
            for (int d = 0; d < 3; d++)
                p[d] += o->facePShift[f * 3 + d];
            o->diffBase(cR, p, T.data(), NDOF, true);
            for (int r = 0; r < R; r++)
                for (int j = 0; j < R; j++)
                    DJ[r * R + j] = T[(r + 1) * NDOF + 1 + j];
            std::vector<double> A = DI, X = DJ;
            if (!ocSolve(R, R, A.data(), X.data()))
                return 1;
            std::copy(X.begin(), X.end(), sec.begin() + (size_t)f * 2 * R * R);
            A = DJ, X = DI;
            if (!ocSolve(R, R, A.data(), X.data()))
                return 1;
            std::copy(X.begin(), X.end(), sec.begin() + ((size_t)f * 2 + 1) * R * R);
        }
        const int st3[5] = {0, 1, 4, 10, 20};
        for (long c = 0; c < o->nCell; c++)
        {
            double *out = uRecNew + c * R * nv;
            const double *rc = uRec + c * R * nv;
            if (!ifAll && si[c] < threshold)
            {
                std::copy(rc, rc + R * nv, out);
                continue;
            }
            std::vector<double> uFaces((size_t)o->nf * R * nv, 0.0);
            for (int cp = P; cp >= 1; cp--)
            {
                const int ls = st3[cp] - 1, le = st3[cp + 1] - 2, nr = le - ls + 1;
                std::vector<std::vector<double>> others;
                others.emplace_back(rc + ls * nv, rc + (le + 1) * nv);
                for (int k = 0; k < o->nf; k++)
                {
                    long f = o->cell2face[c * o->nf + k];
                    long oc = o->otherOf(c, f);
                    if (oc < 0)
                        continue;
                    int side = o->face2cell[f * 2] == c ? 0 : 1;
                    const double *Mt = &sec[((size_t)f * 2 + side) * R * R], *Mo = &sec[((size_t)f * 2 + 1 - side) * R * R];
                    std::vector<double> uoo(uRec + oc * R * nv, uRec + (oc + 1) * R * nv);
                    double *uf = &uFaces[(size_t)k * R * nv];
                    for (int i = le + 1; i < R; i++)
                        for (int v = 0; v < nv; v++)
                        {
                            double a = 0;
                            for (int j = le + 1; j < R; j++)
                                a += Mo[i * R + j] * uf[j * nv + v];
                            uoo[i * nv + v] = a;
                        }
                    std::vector<double> oin(nr * nv), tin(rc + ls * nv, rc + (le + 1) * nv);
                    for (int i = 0; i < nr; i++)
                        for (int v = 0; v < nv; v++)
                        {
                            double a = 0;
                            for (int j = 0; j < R; j++)
                                a += Mt[(ls + i) * R + j] * uoo[j * nv + v];
                            oin[i * nv + v] = a;
                        }
                    const double *uL = side == 0 ? u + c * nv : u + oc * nv, *uR = side == 0 ? u + oc * nv : u + c * nv;
                    const double *n = &o->faceMeanNorm[f * 3];
                    ocCharTransform(uL, uR, n, gamma, true, nr, nv, oin.data());
                    ocCharTransform(uL, uR, n, gamma, true, nr, nv, tin.data());
                    std::vector<double> lim(nr * nv);
                    for (int i = 0; i < nr * nv; i++)
                        lim[i] = ocWbapBiway(tin[i], oin[i], 1.0);
                    ocCharTransform(uL, uR, n, gamma, false, nr, nv, lim.data());
                    for (int i = 0; i < nr * nv; i++)
                        uf[ls * nv + i] = lim[i];
                    others.push_back(lim);
                }
                for (int i = 0; i < nr * nv; i++)
                {
                    double vals[16];
                    for (size_t q = 0; q < others.size(); q++)
                        vals[q] = others[q][i];
                    out[ls * nv + i] = ocWbapMultiway(vals, (int)others.size(), nStd);
                }
            }
        }
        return 0;
    }
}

// ---------------------------------------------------------------------------
// Block ILU(0) of a general block-sparse matrix with a symmetric pattern, natural order: the restatement of
// JacobianLocalLU::InPlaceDecompose (Solver/Direct.hpp:312-405) with iluCode 0 and of its Solve
// (Direct.hpp:487-540) on an arbitrary neighbour table, in the same update order as Oracle::jacobianLU.  It is
// checked against the reference's own unit case of the local LU (test/cpp/Solver/test_Direct.cpp: a periodic
// grid with 2 x 2 blocks) and against Oracle::jacobianLU on mesh operators.
// nbr [n][K]: neighbour indices, -1 for none; off [n][K][bs][bs]: A_(i, nbr[i][k]) in, L (neighbour < i) or U
// (neighbour > i) out; diag [n][bs][bs]: A_ii; dinv [n][bs][bs] out: the inverted pivots.  bs <= 8.
// ---------------------------------------------------------------------------
namespace
{
int ocSlot(const int64_t *nbr, int K, int64_t c, int64_t o)
{
    for (int k = 0; k < K; k++)
        if (nbr[c * K + k] == o)
            return k;
    return -1;
}

bool ocBlockIlu0(int64_t n, int bs, int K, const int64_t *nbr, double *off, const double *diag, double *dinv)
{
    const int nn = bs * bs;
    bool ok = true;
    std::vector<double> Di(nn), T(nn);
    for (int64_t i = 0; i < n; i++)
    {
        std::vector<std::pair<int64_t, int>> low, upp;
        for (int k = 0; k < K; k++)
        {
            int64_t o = nbr[i * K + k];
            if (o >= 0 && o != i)
                (o < i ? low : upp).push_back({o, k});
        }
        std::sort(low.begin(), low.end());
        for (size_t a = 0; a < low.size(); a++) // L_ij = (A_ij - sum_{k < j} L_ik U_kj) Dinv_j
        {
            int64_t j = low[a].first;
            double *Lij = off + (i * K + low[a].second) * nn;
            for (size_t b = 0; b < a; b++)
            {
                int sk = ocSlot(nbr, K, low[b].first, j);
                if (sk >= 0)
                    Oracle::blockMulSub(bs, off + (i * K + low[b].second) * nn, off + (low[b].first * K + sk) * nn, Lij);
            }
            std::copy(Lij, Lij + nn, T.begin());
            for (int r = 0; r < bs; r++)
                for (int c = 0; c < bs; c++)
                {
                    double acc = 0;
                    for (int l = 0; l < bs; l++)
                        acc += T[r * bs + l] * dinv[j * nn + l * bs + c];
                    Lij[r * bs + c] = acc;
                }
        }
        std::copy(diag + i * nn, diag + (i + 1) * nn, Di.begin());
        for (auto &lk : low) // D_i = A_ii - sum_k L_ik U_ki
        {
            int si = ocSlot(nbr, K, lk.first, i);
            if (si >= 0)
                Oracle::blockMulSub(bs, off + (i * K + lk.second) * nn, off + (lk.first * K + si) * nn, Di.data());
        }
        ok = Oracle::invertBlock(bs, Di.data(), dinv + i * nn) && ok;
        for (auto &uj : upp) // U_ij = A_ij - sum_{k < i} L_ik U_kj
        {
            double *Uij = off + (i * K + uj.second) * nn;
            for (auto &lk : low)
            {
                int sk = ocSlot(nbr, K, lk.first, uj.first);
                if (sk >= 0)
                    Oracle::blockMulSub(bs, off + (i * K + lk.second) * nn, off + (lk.first * K + sk) * nn, Uij);
            }
        }
    }
    return ok;
}

void ocBlockIlu0Solve(int64_t n, int bs, int K, const int64_t *nbr, const double *off, const double *dinv, const double *b, double *x)
{
    const int nn = bs * bs;
    for (int64_t i = 0; i < n; i++) // (L + I) y = b, lower neighbours in slot order
    {
        for (int r = 0; r < bs; r++)
            x[i * bs + r] = b[i * bs + r];
        for (int k = 0; k < K; k++)
        {
            int64_t o = nbr[i * K + k];
            if (o < 0 || o >= i)
                continue;
            for (int r = 0; r < bs; r++)
                for (int l = 0; l < bs; l++)
                    x[i * bs + r] -= off[(i * K + k) * nn + r * bs + l] * x[o * bs + l];
        }
    }
    double t[8];
    for (int64_t i = n - 1; i >= 0; i--) // (D + U) x = y
    {
        for (int k = 0; k < K; k++)
        {
            int64_t o = nbr[i * K + k];
            if (o < 0 || o <= i)
                continue;
            for (int r = 0; r < bs; r++)
                for (int l = 0; l < bs; l++)
                    x[i * bs + r] -= off[(i * K + k) * nn + r * bs + l] * x[o * bs + l];
        }
        for (int r = 0; r < bs; r++)
        {
            double acc = 0;
            for (int l = 0; l < bs; l++)
                acc += dinv[i * nn + r * bs + l] * x[i * bs + l];
            t[r] = acc;
        }
        for (int r = 0; r < bs; r++)
            x[i * bs + r] = t[r];
    }
}
} // namespace

extern "C"
{
    // block ILU(0) in place on a general neighbour table (see ocBlockIlu0); 0, or -1 on a singular pivot or bs > 8
    int orc_block_ilu0(int64_t n, int bs, int K, const int64_t *nbr, double *off, const double *diag, double *dinv)
    {
        if (bs < 1 || bs > 8)
            return -1;
        return ocBlockIlu0(n, bs, K, nbr, off, diag, dinv) ? 0 : -1;
    }
    // the quadrature rules of QuadratureHub.hpp:39-380 on the reference element (elem: 0 line [-1, 1], 1 triangle
    // (0,0)-(1,0)-(0,1), 2 quadrilateral [-1, 1]^2, 3 tetrahedron (0,0,0)-(1,0,0)-(0,1,0)-(0,0,1), 4 hexahedron
    // [-1, 1]^3): the number of points of an integration order, and point iG with its weight
    int orc_quad_npoints(int elem, int order) { return quadNPoints(elem, order); }
    void orc_quad_point(int elem, int order, int iG, double *p, double *w)
    {
        real pp[3], ww;
        quadPoint(elem, order, iG, pp, ww);
        for (int d = 0; d < 3; d++)
            p[d] = pp[d];
        *w = ww;
    }
    // the shape functions of Geom/Elements/{Line2,Tri3,Quad4,Tet4,Hex8}.hpp (elem as in orc_quad_point) at a
    // parametric point: N [nNode], dN [3][8] (d/dxi, d/deta, d/dzeta by node)
    void orc_shape(int elem, const double *p, double *N, double *dN)
    {
        real pp[3] = {p[0], p[1], p[2]}, Nv[8], dNv[3][8];
        shapeD01(elem, pp, Nv, dNv);
        for (int i = 0; i < elemNNode(elem); i++)
        {
            N[i] = Nv[i];
            for (int d = 0; d < 3; d++)
                dN[d * 8 + i] = dNv[d][i];
        }
    }
    // x = (L U)^-1 b with the factors of orc_block_ilu0
    void orc_block_ilu0_solve(int64_t n, int bs, int K, const int64_t *nbr, const double *off, const double *dinv, const double *b, double *x)
    {
        ocBlockIlu0Solve(n, bs, K, nbr, off, dinv, b, x);
    }
}

#endif // ORC_OPCOUNT
