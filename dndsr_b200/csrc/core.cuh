// Shared host/device math of the VR + Euler residual path.
//
// Quadrature rules, element shape functions, the Taylor-type polynomial basis
// of the variational reconstruction, ideal-gas thermodynamics, the Riemann
// solvers and the viscous flux.  Every function is a plain __host__ __device__
// routine on fixed-size arrays so that setup kernels and hot kernels share one
// definition.  Each block cites the reference routine whose results it must
// reproduce (paths relative to the reference project root).
#pragma once
#include "platform.cuh"
#include "dual.cuh"
#include <math.h>

namespace dndsb
{
constexpr real kVerySmall = 1e-200; // DNDS/Defines.hpp:199 verySmallReal
constexpr real kSmall = 1e-10;      // DNDS/Defines.hpp:201 smallReal
constexpr real kVeryLarge = 3e200;  // DNDS/Defines.hpp:195 veryLargeReal
constexpr real kPi = 3.14159265358979323846;
constexpr int kIntOrderMax = 6; // Geom/Quadratures/QuadratureBase.hpp:70

enum ElemKind : int
{
    E_LINE2 = 0,
    E_TRI3 = 1,
    E_QUAD4 = 2,
    E_TET4 = 3,
    E_HEX8 = 4
};

DNDSB_HD real sqr(real x) { return x * x; }
DNDSB_HD real dmax(real a, real b) { return a > b ? a : b; }
DNDSB_HD real dmin(real a, real b) { return a < b ? a : b; }
DNDSB_HD real dot3(const real *a, const real *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// ---------------------------------------------------------------------------
// Quadrature.  Scheme choice per integration order follows
// Geom/QuadratureHub.hpp:39-140; the point sets are the published rules the
// reference tabulates (Gauss-Legendre; Strang-Fix / Dunavant triangle rules of
// degree 1,2,4,5,6; Keast tetrahedron rules of degree 1,2,3,5,6), generated
// here from their symmetric orbits.
// ---------------------------------------------------------------------------
DNDSB_HD int gl_n(int order) { return order <= 1 ? 1 : order <= 3 ? 2 : order <= 5 ? 3 : 4; }

DNDSB_HD void gl_point(int n, int i, real &x, real &w)
{
    switch (n)
    {
    case 1:
        x = 0, w = 2;
        return;
    case 2:
        x = (i == 0 ? -1 : 1) * 0.57735026918962576451, w = 1;
        return;
    case 3:
        if (i == 1)
            x = 0, w = 8.0 / 9.0;
        else
            x = (i == 0 ? -1 : 1) * 0.77459666924148337704, w = 5.0 / 9.0;
        return;
    default:
    {
        const real a = 0.86113631159405257522, b = 0.33998104358485626480;
        const real wa = 0.34785484513745385737, wb = 0.65214515486254614263;
        const real xs[4] = {-a, -b, b, a}, ws[4] = {wa, wb, wb, wa};
        x = xs[i], w = ws[i];
        return;
    }
    }
}

DNDSB_HD int tri_n(int order) { return order <= 1 ? 1 : order == 2 ? 3 : order <= 4 ? 6 : order == 5 ? 7 : 12; }
DNDSB_HD int tet_n(int order) { return order <= 1 ? 1 : order == 2 ? 4 : order == 3 ? 8 : order <= 5 ? 14 : 24; }

DNDSB_HD int quad_n(int elem, int order)
{
    switch (elem)
    {
    case E_LINE2:
        return gl_n(order);
    case E_QUAD4:
        return gl_n(order) * gl_n(order);
    case E_HEX8:
        return gl_n(order) * gl_n(order) * gl_n(order);
    case E_TRI3:
        return tri_n(order);
    default:
        return tet_n(order);
    }
}

// barycentric orbit helpers (area of the reference triangle is 1/2, volume of the reference tet 1/6)
DNDSB_HD void tri_s21(int k, real a, real &x, real &y)
{
    // permutations of (a, a, 1-2a)
    real b = 1 - 2 * a;
    if (k == 0)
        x = a, y = a;
    else if (k == 1)
        x = b, y = a;
    else
        x = a, y = b;
}

DNDSB_HD void tri_s111(int k, real a, real b, real &x, real &y)
{
    real c = 1 - a - b;
    real v[6][2] = {{a, b}, {b, a}, {a, c}, {c, a}, {b, c}, {c, b}};
    x = v[k][0], y = v[k][1];
}

DNDSB_HD void tri_point(int order, int i, real p[3], real &w)
{
    p[2] = 0;
    switch (tri_n(order))
    {
    case 1:
        p[0] = p[1] = 1.0 / 3.0, w = 0.5;
        return;
    case 3:
        tri_s21(i, 1.0 / 6.0, p[0], p[1]), w = 1.0 / 6.0;
        return;
    case 6:
        if (i < 3)
            tri_s21(i, 0.091576213509770743460, p[0], p[1]), w = 0.5 * 0.10995174365532186764;
        else
            tri_s21(i - 3, 0.44594849091596488632, p[0], p[1]), w = 0.5 * 0.22338158967801146570;
        return;
    case 7:
    {
        const real s15 = 3.87298334620741688518; // sqrt(15)
        if (i == 0)
            p[0] = p[1] = 1.0 / 3.0, w = 0.5 * 9.0 / 40.0;
        else if (i < 4)
            tri_s21(i - 1, (6 + s15) / 21, p[0], p[1]), w = 0.5 * (155 + s15) / 1200;
        else
            tri_s21(i - 4, (6 - s15) / 21, p[0], p[1]), w = 0.5 * (155 - s15) / 1200;
        return;
    }
    default:
        if (i < 3)
            tri_s21(i, 0.24928674517091042129, p[0], p[1]), w = 0.5 * 0.11678627572637936603;
        else if (i < 6)
            tri_s21(i - 3, 0.063089014491502228340, p[0], p[1]), w = 0.5 * 0.050844906370206816921;
        else
            tri_s111(i - 6, 0.053145049844816947353, 0.31035245103378440542, p[0], p[1]), w = 0.5 * 0.082851075618373575194;
        return;
    }
}

DNDSB_HD void tet_s31(int k, real a, real p[3])
{
    real b = 1 - 3 * a;
    p[0] = p[1] = p[2] = a;
    if (k < 3)
        p[k] = b;
}

DNDSB_HD void tet_s22(int k, real a, real p[3])
{
    real b = 0.5 - a;
    // barycentric (a,a,b,b) permutations; p holds the last three coordinates
    const int pat[6][3] = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int d = 0; d < 3; d++)
        p[d] = pat[k][d] ? b : a;
}

DNDSB_HD void tet_s211(int k, real a, real b, real c, real p[3])
{
    // barycentric (a, a, b, c) with b, c at distinct slots among 4
    const int slots[12][2] = {{0, 1}, {1, 0}, {0, 2}, {2, 0}, {0, 3}, {3, 0}, {1, 2}, {2, 1}, {1, 3}, {3, 1}, {2, 3}, {3, 2}};
    real l[4] = {a, a, a, a};
    l[slots[k][0]] = b, l[slots[k][1]] = c;
    p[0] = l[1], p[1] = l[2], p[2] = l[3];
}

DNDSB_HD void tet_point(int order, int i, real p[3], real &w)
{
    switch (tet_n(order))
    {
    case 1:
        p[0] = p[1] = p[2] = 0.25, w = 1.0 / 6.0;
        return;
    case 4:
        tet_s31(i, 0.13819660112501051518, p), w = 1.0 / 24.0;
        return;
    case 8:
        if (i < 4)
            tet_s31(i, 0.1069940147705369, p), w = 0.01859314997209119;
        else
            tet_s31(i - 4, 0.3280585716625127, p), w = 0.02307351669457548;
        return;
    case 14:
        if (i < 4)
            tet_s31(i, 0.09273525031089125, p), w = 0.01224884051939367;
        else if (i < 8)
            tet_s31(i - 4, 0.3108859192633008, p), w = 0.01878132095300264;
        else
            tet_s22(i - 8, 0.04550370412564952, p), w = 0.0070910034628469;
        return;
    default:
        if (i < 4)
            tet_s31(i, 0.2146028712591523, p), w = 0.006653791709694545;
        else if (i < 8)
            tet_s31(i - 4, 0.3223378901422754, p), w = 0.009226196923942479;
        else if (i < 12)
            tet_s31(i - 8, 0.04067395853461131, p), w = 0.001679535175886773;
        else
            tet_s211(i - 12, 0.06366100187501755, 0.2696723314583158, 0.6030056647916491, p), w = 9.0 / 1120.0;
        return;
    }
}

DNDSB_HD void quad_point(int elem, int order, int i, real p[3], real &w)
{
    p[0] = p[1] = p[2] = 0;
    if (elem == E_TRI3)
        return tri_point(order, i, p, w);
    if (elem == E_TET4)
        return tet_point(order, i, p, w);
    int n = gl_n(order);
    real w0, w1, w2;
    if (elem == E_LINE2)
    {
        gl_point(n, i, p[0], w);
        return;
    }
    if (elem == E_QUAD4)
    {
        gl_point(n, i % n, p[0], w0);
        gl_point(n, i / n, p[1], w1);
        w = w0 * w1;
        return;
    }
    gl_point(n, i % n, p[0], w0);
    gl_point(n, (i / n) % n, p[1], w1);
    gl_point(n, i / (n * n), p[2], w2);
    w = w0 * w1 * w2;
}

// ---------------------------------------------------------------------------
// Shape functions of the linear elements (Geom/Elements/{Line2,Tri3,Quad4,
// Tet4,Hex8}.hpp: standard nodes in [-1,1]^d or the unit simplex).
// ---------------------------------------------------------------------------
DNDSB_HD int elem_nnode(int e) { return e == E_LINE2 ? 2 : e == E_TRI3 ? 3 : e == E_HEX8 ? 8 : 4; }

// point and Jacobian of an element map; templated on the coordinate type (real, or dual numbers
// for derivatives with respect to the node coordinates)
template <typename T>
struct PtGeoT
{
    T x[3];
    T J[3][3]; // J[r][c] = d x_r / d xi_c
};
using PtGeo = PtGeoT<real>;

template <typename T>
DNDSB_HD void pt_geo(int e, const T *cs /*nn x 3*/, const real p[3], PtGeoT<T> &g)
{
    real N[8], dN[3][8];
    int nn = elem_nnode(e);
    for (int i = 0; i < 8; i++)
        N[i] = dN[0][i] = dN[1][i] = dN[2][i] = 0;
    const real xi = p[0], et = p[1], zt = p[2];
    if (e == E_LINE2)
    {
        N[0] = 0.5 * (1 - xi), N[1] = 0.5 * (1 + xi);
        dN[0][0] = -0.5, dN[0][1] = 0.5;
    }
    else if (e == E_TRI3)
    {
        N[0] = 1 - xi - et, N[1] = xi, N[2] = et;
        dN[0][0] = -1, dN[0][1] = 1, dN[1][0] = -1, dN[1][2] = 1;
    }
    else if (e == E_TET4)
    {
        N[0] = 1 - xi - et - zt, N[1] = xi, N[2] = et, N[3] = zt;
        dN[0][0] = -1, dN[0][1] = 1, dN[1][0] = -1, dN[1][2] = 1, dN[2][0] = -1, dN[2][3] = 1;
    }
    else if (e == E_QUAD4)
    {
        const real sx[4] = {-1, 1, 1, -1}, sy[4] = {-1, -1, 1, 1};
        for (int i = 0; i < 4; i++)
        {
            real a = 1 + sx[i] * xi, b = 1 + sy[i] * et;
            N[i] = 0.25 * a * b;
            dN[0][i] = 0.25 * sx[i] * b;
            dN[1][i] = 0.25 * a * sy[i];
        }
    }
    else
    {
        const real sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1}, sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
        for (int i = 0; i < 8; i++)
        {
            real a = 1 + sx[i] * xi, b = 1 + sy[i] * et, c = 1 + sz[i] * zt;
            N[i] = 0.125 * a * b * c;
            dN[0][i] = 0.125 * sx[i] * b * c;
            dN[1][i] = 0.125 * a * sy[i] * c;
            dN[2][i] = 0.125 * a * b * sz[i];
        }
    }
    for (int r = 0; r < 3; r++)
    {
        T s = 0, j0 = 0, j1 = 0, j2 = 0;
        for (int i = 0; i < nn; i++)
        {
            const T &c = cs[i * 3 + r];
            s += c * N[i], j0 += c * dN[0][i], j1 += c * dN[1][i], j2 += c * dN[2][i];
        }
        g.x[r] = s, g.J[r][0] = j0, g.J[r][1] = j1, g.J[r][2] = j2;
    }
}

// Geom/Quadrature.hpp:480-490 (cell) and :500-511 with Geom/Geometric.hpp:113-128 (face)
template <typename T>
DNDSB_HD T cell_jdet(int dim, const PtGeoT<T> &g)
{
    if (dim == 2)
    {
        T c2 = g.J[0][0] * g.J[1][1] - g.J[1][0] * g.J[0][1];
        T c0 = g.J[1][0] * g.J[2][1] - g.J[2][0] * g.J[1][1];
        T c1 = g.J[2][0] * g.J[0][1] - g.J[0][0] * g.J[2][1];
        return sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    }
    const T(*J)[3] = g.J;
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

// returns |J| of the face map and writes the (unnormalised) normal
template <typename T>
DNDSB_HD T face_jdet_normal(int dim, const PtGeoT<T> &g, T n[3])
{
    if (dim == 2)
    {
        n[0] = g.J[1][0], n[1] = -g.J[0][0], n[2] = 0;
        return sqrt(g.J[0][0] * g.J[0][0] + g.J[1][0] * g.J[1][0] + g.J[2][0] * g.J[2][0]);
    }
    T a[3] = {g.J[0][0], g.J[1][0], g.J[2][0]}, b[3] = {g.J[0][1], g.J[1][1], g.J[2][1]};
    n[0] = a[1] * b[2] - a[2] * b[1];
    n[1] = a[2] * b[0] - a[0] * b[2];
    n[2] = a[0] * b[1] - a[1] * b[0];
    return sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
}

// ---------------------------------------------------------------------------
// Polynomial basis (Geom/BaseFunction.hpp).  Monomials up to degree 3 are
// ordered 1; x,y(,z); then the second and third degree terms in the
// reference's order (BaseFunction.hpp:55-107).  A row "d" of the diff table
// holds the derivative d of every monomial, scaled by the cell length scales
// (FPolynomialFill2D/3D, BaseFunction.hpp:285-700).
// ---------------------------------------------------------------------------
template <int DIM>
struct Basis;

template <>
struct Basis<2>
{
    static DNDSB_HD int ndof(int p) { return p == 0 ? 1 : p == 1 ? 3 : p == 2 ? 6 : 10; }
    static DNDSB_HD void exps(int k, int e[3])
    {
        const signed char t[10][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}, {3, 0}, {2, 1}, {1, 2}, {0, 3}};
        e[0] = t[k][0], e[1] = t[k][1], e[2] = 0;
    }
    static DNDSB_HD int ncomb(int k)
    {
        const signed char c[10] = {1, 1, 1, 1, 2, 1, 1, 3, 3, 1};
        return c[k];
    }
    static DNDSB_HD int order_start(int o)
    {
        const signed char s[5] = {0, 1, 3, 6, 10};
        return s[o];
    }
};

template <>
struct Basis<3>
{
    static DNDSB_HD int ndof(int p) { return p == 0 ? 1 : p == 1 ? 4 : p == 2 ? 10 : 20; }
    static DNDSB_HD void exps(int k, int e[3])
    {
        const signed char t[20][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1},
                                      {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {1, 2, 0}, {0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {2, 0, 1}, {1, 1, 1}};
        e[0] = t[k][0], e[1] = t[k][1], e[2] = t[k][2];
    }
    static DNDSB_HD int ncomb(int k)
    {
        const signed char c[20] = {1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 3, 3, 3, 3, 3, 3, 6};
        return c[k];
    }
    static DNDSB_HD int order_start(int o)
    {
        const signed char s[5] = {0, 1, 4, 10, 20};
        return s[o];
    }
};

// p!/(p-d)! for d <= p, else 0
DNDSB_HD real falling(int p, int d)
{
    if (d > p)
        return 0;
    real r = 1;
    for (int i = 0; i < d; i++)
        r *= (p - i);
    return r;
}

template <typename T>
DNDSB_HD T ipow(const T &x, int e)
{
    T r = 1;
    for (int i = 0; i < e; i++)
        r *= x;
    return r;
}

// Diff table of the basis at scaled offset (x,y,z) = (p - cent) / L with
// scales L; rows [0, rows), columns [0, NDOF).  Column 0 is the constant.
template <int DIM, int NDOF, typename S>
DNDSB_HD void basis_table(S *T, int rows, const S &x, const S &y, const S &z, const S L[3])
{
    for (int r = 0; r < rows; r++)
    {
        int d[3];
        Basis<DIM>::exps(r, d);
        S lscale = ipow(L[0], d[0]) * ipow(L[1], d[1]);
        if (DIM == 3)
            lscale = lscale * ipow(L[2], d[2]);
        for (int k = 0; k < NDOF; k++)
        {
            int e[3];
            Basis<DIM>::exps(k, e);
            real c = falling(e[0], d[0]) * falling(e[1], d[1]) * falling(e[2], d[2]);
            if (c == 0)
                T[r * NDOF + k] = 0.0;
            else
                T[r * NDOF + k] = c * ipow(x, e[0] - d[0]) * ipow(y, e[1] - d[1]) * ipow(z, e[2] - d[2]) / lscale;
        }
    }
}

// ---------------------------------------------------------------------------
// Ideal gas (DNDS/IdealGasPhysics.hpp:38-44) and Riemann solvers
// (Euler/Gas.hpp:229-259 Roe averages, :601-714 HLLEP, :878-1126 Roe with its
// entropy fixes, :1434-1490 dispatch).  Physics is 3-D with 5 conservative
// variables (NS / NS_3D; the SA variable is handled by the caller).
// ---------------------------------------------------------------------------
// The state-dependent routines below are templated on the scalar type T: real
// for the solver, Dual<N> (dual.cuh) for directional derivatives.
template <typename T>
DNDSB_HD void gas_thermal(T E, T rho, T vSqr, real gamma, T &p, T &asqr, T &H)
{
    p = (gamma - 1) * (E - rho * 0.5 * vSqr);
    T ir = 1.0 / rho;
    asqr = gamma * p * ir;
    H = (E + p) * ir;
}

enum RSType : int
{
    RS_Roe = 1,
    RS_HLLC = 2,
    RS_HLLEP = 3,
    RS_HLLEP_V1 = 21,
    RS_Roe_M1 = 11,
    RS_Roe_M2 = 12,
    RS_Roe_M3 = 13,
    RS_Roe_M4 = 14,
    RS_Roe_M5 = 15,
    RS_Roe_M6 = 16,
    RS_Roe_M7 = 17,
    RS_Roe_M8 = 18
};

template <typename T>
DNDSB_HD real sign_tol(const T &a, const T &tol) { return a > tol ? 1 : (a < -tol ? -1 : 0); }

template <typename T, typename TN>
DNDSB_HD T dot3v(const T *a, const TN *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
template <typename T>
DNDSB_HD T dot3s(const T *a, const T *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

template <typename T>
struct RoeAvgT
{
    T vL[3], vR[3], aL, aR, pLm, pRm;
    T v[3], vsqr, H, asqr, a, rho;
    T gOverA2, inv2a; // (gamma - 1) / asqr and 1 / (2 a), shared by the Gauss points of a face
};
using RoeAvg = RoeAvgT<real>;

template <typename T>
DNDSB_HD void roe_average(const T *ULm, const T *URm, real gamma, RoeAvgT<T> &r)
{
    T iL = 1.0 / ULm[0], iR = 1.0 / URm[0];
    for (int d = 0; d < 3; d++)
        r.vL[d] = ULm[1 + d] * iL, r.vR[d] = URm[1 + d] * iR;
    T pL, pR, aL2, aR2, HL, HR;
    gas_thermal(ULm[4], ULm[0], dot3s(r.vL, r.vL), gamma, pL, aL2, HL);
    gas_thermal(URm[4], URm[0], dot3s(r.vR, r.vR), gamma, pR, aR2, HR);
    r.aL = sqrt(aL2), r.aR = sqrt(aR2), r.pLm = pL, r.pRm = pR;
    T sL = sqrt(ULm[0]), sR = sqrt(URm[0]);
    T is = 1.0 / (sL + sR);
    for (int d = 0; d < 3; d++)
        r.v[d] = (sL * r.vL[d] + sR * r.vR[d]) * is;
    r.vsqr = dot3s(r.v, r.v);
    r.H = (sL * HL + sR * HR) * is;
    r.asqr = (gamma - 1) * (r.H - 0.5 * r.vsqr);
    r.rho = sL * sR;
    r.a = sqrt(r.asqr);
    r.gOverA2 = (gamma - 1) / r.asqr;
    r.inv2a = 0.5 / r.a;
}

// physical flux through n (no grid velocity): Gas.hpp:390-397
// n: real, or dual numbers of the same kind as T for derivatives with respect to the face geometry
template <typename T, typename TN>
DNDSB_HD void phys_flux(const T *U, const TN *n, real gamma, T F[5], T &p, T &asqr)
{
    T ir = 1.0 / U[0];
    T v[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
    p = (gamma - 1) * (U[4] - U[0] * 0.5 * dot3s(v, v));
    asqr = gamma * p * ir;
    T vn = dot3v(v, n);
    F[0] = U[0] * vn;
    F[1] = U[1] * vn + p * n[0];
    F[2] = U[2] * vn + p * n[1];
    F[3] = U[3] * vn + p * n[2];
    F[4] = (U[4] + p) * vn;
}

// Roe wave strengths (Gas.hpp:1098-1109): jump incU projected on the Roe eigenvectors
template <typename T>
struct RoeWavesT
{
    T a0, a1, a4, a23T[3], vRoeN;
};

// nE: normal of the Roe normal velocity (the point normal n, or the face's mean normal for the
// batched mean-value eigenvalues of Gas.hpp:1272-1408)
template <typename T, typename TN>
DNDSB_HD void roe_waves(const T *incU, const TN *n, const RoeAvgT<T> &r, real gamma, RoeWavesT<T> &w, const TN *nE = nullptr)
{
    w.vRoeN = dot3v(r.v, nE ? nE : n);
    T incU123N = incU[1] * n[0] + incU[2] * n[1] + incU[3] * n[2];
    T a23[3] = {incU[1] - incU[0] * r.v[0], incU[2] - incU[0] * r.v[1], incU[3] - incU[0] * r.v[2]};
    T a23n = dot3v(a23, n);
    for (int d = 0; d < 3; d++)
        w.a23T[d] = a23[d] - n[d] * a23n;
    T incU4b = incU[4] - dot3s(w.a23T, r.v);
    w.a1 = r.gOverA2 * (incU[0] * (r.H - w.vRoeN * w.vRoeN) + w.vRoeN * incU123N - incU4b);
    w.a0 = (incU[0] * (w.vRoeN + r.a) - incU123N - r.a * w.a1) * r.inv2a;
    w.a4 = incU[0] - (w.a0 + w.a1);
}

// |A| dU assembled from wave strengths times eigenvalues (Gas.hpp:1110-1124)
template <typename T, typename TN>
DNDSB_HD void roe_dissipation(const RoeWavesT<T> &w, const TN *n, const RoeAvgT<T> &r, const T &l0, const T &l123, const T &l4, T incF[5])
{
    T a0 = w.a0 * l0, a1 = w.a1 * l123, a4 = w.a4 * l4;
    T t[3] = {w.a23T[0] * l123, w.a23T[1] * l123, w.a23T[2] * l123};
    incF[0] = a0 + a1 + a4;
    incF[4] = (r.H - w.vRoeN * r.a) * a0 + 0.5 * r.vsqr * a1 + (r.H + w.vRoeN * r.a) * a4 + dot3s(t, r.v);
    for (int d = 0; d < 3; d++)
        incF[1 + d] = (r.v[d] - r.a * n[d]) * a0 + (r.v[d] + r.a * n[d]) * a4 + r.v[d] * a1 + t[d];
}

// Gas.hpp:878-1007 Roe_EntropyFixer (eigScheme 0,1,3..8)
template <typename T>
DNDSB_HD void roe_entropy_fix(int es, const T &aL, const T &aR, const T &aAve, const T &uL, const T &uR, const T &uAve, const T &VAve,
                              real dLambda, real fixScale, real incFScale, T &lam0, T &lam123, T &lam4)
{
    const real sHY = 0.05 * fixScale, sLD = 0.2 * fixScale, sHF = 0.25 * fixScale;
    if (es == 0)
    {
        auto flim = [&](const T &v, const T &lam, const T &lamL, const T &lamR)
        {
            T th = dmax(dmax(T(0.0), lam - lamL), lamR - lam) * sHY;
            return v < th ? T((v * v / th + th) * 0.5) : v;
        };
        lam0 = flim(lam0, uAve - aAve, uL - aL, uR - aR);
        lam123 = flim(lam123 * incFScale, uAve, uL, uR);
        lam4 = flim(lam4, uAve + aAve, uL + aL, uR + aR);
    }
    else if (es == 1)
    {
        T uLm = sign_tol(uL, T(aL * kSmall)) * dmax(T(fabs(uL) * incFScale), T(aL * sLD));
        T uRm = sign_tol(uR, T(aR * kSmall)) * dmax(T(fabs(uR) * incFScale), T(aR * sLD));
        lam0 = dmax(fabs(uLm - aL), fabs(uRm - aR));
        lam123 = dmax(fabs(uLm), fabs(uRm));
        lam4 = dmax(fabs(uLm + aL), fabs(uRm + aR));
    }
    else if (es == 3)
    {
        T aS = dmin(T(fabs(uAve) / sLD), aAve);
        lam0 = fabs(uAve * incFScale - aS);
        lam4 = fabs(uAve * incFScale + aS);
    }
    else if (es == 4)
    {
        T uS = sign_tol(uAve, T(aAve * kSmall)) * dmax(T(aAve * sLD), T(fabs(uAve) * incFScale));
        lam0 = fabs(uS - aAve), lam123 = fabs(uS), lam4 = fabs(uS + aAve);
    }
    else if (es == 5)
    {
        T vL = uL * incFScale, vR = uR * incFScale;
        T aLm = dmin(aL, T(fabs(vL) / sLD)), aRm = dmin(aR, T(fabs(vR) / sLD));
        lam0 = dmax(fabs(vL - aLm), fabs(vR - aRm));
        lam123 = dmax(fabs(vL), fabs(vR));
        lam4 = dmax(fabs(vL + aLm), fabs(vR + aRm));
    }
    else if (es == 6 || es == 8)
    {
        lam0 = dmax(T(fabs(uAve * incFScale - aAve)), T(dLambda * sHF));
        lam4 = dmax(T(fabs(uAve * incFScale + aAve)), T(dLambda * sHF));
        lam123 = dmax(T(fabs(uAve * incFScale)), T(dLambda * sHF));
    }
    else if (es == 7)
    {
        lam0 = lam0 * fabs(uAve * incFScale - aAve);
        lam4 = lam4 * fabs(uAve * incFScale + aAve);
        lam123 = lam123 * fabs(uAve * incFScale);
    }
    if (es == 7 || es == 8)
    {
        T th = sHY * (VAve + aAve), th2 = th * th;
        if (lam0 < th)
            lam0 = (lam0 * lam0 + th2) / (2 * th);
        if (lam4 < th)
            lam4 = (lam4 * lam4 + th2) / (2 * th);
        if (lam123 < th)
            lam123 = (lam123 * lam123 + th2) / (2 * th);
    }
}

// Approximate Riemann flux F(UL,UR; ULm,URm) . n for the 5 Euler variables.
// Returns false when a state is non-physical (the caller records an error).
// The Roe averages r come from the cell-mean states (Gas.hpp:229-259) and are
// shared by all Gauss points of a face.
// nMean (may be null): the face's mean normal, given when the settings ask for the batched
// mean-value eigenvalues (rsMeanValueEig != 0 with Roe_M1..Roe_M5, EulerEvaluator_EvaluateDt.hxx:1259-1270):
// RoeFlux_IdealGas_HartenYee_Batch (Gas.hpp:1272-1408) then takes the eigenvalues, the entropy fix
// and the Roe normal velocity along it, the physical fluxes and jump projections along n.
template <typename T, typename TN>
DNDSB_HD bool riemann_flux_pre(int rs, const T *UL, const T *UR, const RoeAvgT<T> &r, const TN *n, real gamma, real dLambda, real fixScale,
                               real incFScale, T F[5], T &lam0, T &lam123, T &lam4, const TN *nMean = nullptr)
{
    T FL[5], FR[5], pL, pR, aL2, aR2;
    phys_flux(UL, n, gamma, FL, pL, aL2);
    phys_flux(UR, n, gamma, FR, pR, aR2);
    bool ok = UL[0] > 0 && UR[0] > 0 && r.asqr > 0;
    const TN *nE = (nMean && rs >= RS_Roe_M1 && rs <= RS_Roe_M1 + 4) ? nMean : n;
    T vRoe0 = dot3v(r.v, nE);
    lam0 = fabs(vRoe0 - r.a), lam123 = fabs(vRoe0), lam4 = fabs(vRoe0 + r.a);
    T vLm0 = dot3v(r.vL, nE), vRm0 = dot3v(r.vR, nE);
    T incU[5];
    for (int i = 0; i < 5; i++)
        incU[i] = UR[i] - UL[i];
    if (rs == RS_HLLEP || rs == RS_HLLEP_V1)
    {
        RoeWavesT<T> w;
        roe_waves(incU, n, r, gamma, w);
        T SL = dmin(T(vRoe0 - r.a), T(vLm0 - sqrt(aL2)));
        T SR = dmax(T(vRoe0 + r.a), T(vRm0 + sqrt(aR2)));
        T dfix = r.a / (r.a + dmax(T(fabs(vRoe0)), T(dLambda * fixScale)));
        T SP = dmax(SR, T(0.0)), SM = dmin(SL, T(0.0));
        if (rs == RS_HLLEP)
        {
            T div = SP - SM;
            div = div + (div >= 0 ? 1 : -1) * kVerySmall;
            T id = 1.0 / div;
            T rv1[5] = {T(1), r.v[0], r.v[1], r.v[2], T(0.5 * r.vsqr)};
            for (int i = 0; i < 5; i++)
                F[i] = (SP * FL[i] - SM * FR[i]) * id + (SP * SM * id) * (incU[i] - dfix * rv1[i] * w.a1);
        }
        else
        {
            T dd = 1.0 / (SP - SM);
            lam123 = fabs(((SP + SM) * vRoe0 - 2.0 * (1.0 - dfix) * (SP * SM)) * dd);
            lam4 = fabs(((SP + SM) * (vRoe0 + r.a) - 2.0 * (SP * SM)) * dd);
            lam0 = fabs(((SP + SM) * (vRoe0 - r.a) - 2.0 * (SP * SM)) * dd);
            T incF[5];
            roe_dissipation(w, n, r, lam0, lam123, lam4, incF);
            for (int i = 0; i < 5; i++)
                F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * incF[i];
        }
        return ok;
    }
    if (rs == RS_HLLC)
    {
        auto q = [&](const T &p, const T &pS)
        { return pS <= p ? T(1.0) : T(sqrt(1 + (gamma + 1) / 2 / gamma * (pS / p - 1))); };
        T pS = dmax(T(0.0), T(0.5 * (r.pLm + r.pRm) - 0.5 * (vLm0 - vRm0) * r.rho * r.a));
        T SL = vLm0 - r.aL * q(r.pLm, pS);
        T SR = vRm0 + r.aR * q(r.pRm, pS);
        if (0 <= SL)
        {
            for (int i = 0; i < 5; i++)
                F[i] = FL[i];
            return ok;
        }
        if (SR <= 0)
        {
            for (int i = 0; i < 5; i++)
                F[i] = FR[i];
            return ok;
        }
        T div = UL[0] * (SL - vLm0) - UR[0] * (SR - vRm0);
        T ULn = UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2], URn = UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2];
        T SS = fabs(div) > kVerySmall ? T((pR - pL + ULn * (SL - vLm0) - URn * (SR - vRm0)) / div) : T(0.0);
        T DS[5] = {T(0), T(n[0]), T(n[1]), T(n[2]), SS};
        const T *U = SS >= 0 ? UL : UR;
        const T *FF = SS >= 0 ? FL : FR;
        T S = SS >= 0 ? SL : SR, vm = SS >= 0 ? vLm0 : vRm0, pp = SS >= 0 ? pL : pR;
        T dv = S - SS;
        if (fabs(dv) < kVerySmall)
            for (int i = 0; i < 5; i++)
                F[i] = FF[i];
        else
            for (int i = 0; i < 5; i++)
                F[i] = ((U[i] * S - FF[i]) * SS + DS[i] * ((pp + U[0] * (S - vm) * (SS - vm)) * S)) / dv;
        return ok;
    }
    // Roe family
    int es = rs == RS_Roe ? 0 : rs - 10;
    if (es == 2)
    {
        lam0 = lam123 = lam4 = dmax(T(fabs(vLm0) + r.aL), T(fabs(vRm0) + r.aR));
        for (int i = 0; i < 5; i++)
            F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * lam0 * incU[i];
        return ok;
    }
    T VAve = sqrt(r.vsqr);
    roe_entropy_fix(es, r.aL, r.aR, r.a, vLm0, vRm0, vRoe0, VAve, dLambda, fixScale, incFScale, lam0, lam123, lam4);
    RoeWavesT<T> w;
    roe_waves(incU, n, r, gamma, w, nE);
    T incF[5];
    roe_dissipation(w, n, r, lam0, lam123, lam4, incF);
    for (int i = 0; i < 5; i++)
        F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * incF[i];
    return ok;
}

template <typename T, typename TN>
DNDSB_HD bool riemann_flux(int rs, const T *UL, const T *UR, const T *ULm, const T *URm, const TN *n, real gamma, real dLambda,
                           real fixScale, real incFScale, T F[5], T &lam0, T &lam123, T &lam4, const TN *nMean = nullptr)
{
    RoeAvgT<T> r;
    roe_average(ULm, URm, gamma, r);
    return riemann_flux_pre(rs, UL, UR, r, n, gamma, dLambda, fixScale, incFScale, F, lam0, lam123, lam4, nMean);
}

// Gas.hpp:1677-1698 GradientCons2Prim_IdealGas; G and GP are [3][NV]; ir = 1 / U[0]
template <int NV, typename T>
DNDSB_HD void grad_cons2prim_ir(const T *U, const T &ir, const T *G, T *GP, real gamma)
{
    T v[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
    for (int r = 0; r < 3; r++)
    {
        const T *g = G + r * NV;
        T *gp = GP + r * NV;
        gp[0] = g[0];
        for (int j = 0; j < 3; j++)
            gp[1 + j] = (U[0] * g[1 + j] - g[0] * U[1 + j]) * ir * ir;
        T s = g[1] * v[0] + g[2] * v[1] + g[3] * v[2] + gp[1] * U[1] + gp[2] * U[2] + gp[3] * U[3];
        gp[4] = (gamma - 1) * (g[4] - 0.5 * s);
        for (int j = 5; j < NV; j++)
            gp[j] = (g[j] - g[0] * U[j] * ir) * ir;
    }
}

template <int NV, typename T>
DNDSB_HD void grad_cons2prim(const T *U, const T *G, T *GP, real gamma)
{
    T ir = 1.0 / U[0];
    grad_cons2prim_ir<NV>(U, ir, G, GP, gamma);
}

// Gas.hpp:1594-1655 ViscousFlux_IdealGas without QCR; GP is the primitive gradient [3][NV];
// ir = 1 / U[0], kT = gamma / ((gamma - 1) Cp)
template <int NV, typename T>
DNDSB_HD void viscous_flux_ir(const T *U, const T &ir, const T *GP, const real *n, bool adiabatic, real gamma, T mu, T k, real kT, T *Fv)
{
    T v[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
    T p = (gamma - 1) * (U[4] - U[0] * 0.5 * dot3s(v, v));
    T cT = kT * ir * ir;
    T gT[3];
    for (int i = 0; i < 3; i++)
        gT[i] = cT * (U[0] * GP[i * NV + 4] - p * GP[i * NV + 0]);
    if (adiabatic)
    {
        T gn = dot3v(gT, n);
        for (int i = 0; i < 3; i++)
            gT[i] -= gn * n[i];
    }
    T tr = GP[0 * NV + 1] + GP[1 * NV + 2] + GP[2 * NV + 3];
    T lm = -2.0 / 3.0 * mu * tr;
    T e = 0;
    for (int i = 0; i < 3; i++)
    {
        T fi = 0, si = 0;
        for (int j = 0; j < 3; j++)
        {
            T s = (GP[i * NV + 1 + j] + GP[j * NV + 1 + i]) * mu + (i == j ? lm : T(0.0));
            fi += s * n[j];
            si += s * v[j];
        }
        Fv[1 + i] = fi;
        e += (si + k * gT[i]) * n[i];
    }
    Fv[0] = 0;
    Fv[4] = e;
}

template <int NV, typename T>
DNDSB_HD void viscous_flux(const T *U, const T *GP, const real *n, bool adiabatic, real gamma, T mu, T k, real Cp, T *Fv)
{
    T ir = 1.0 / U[0];
    viscous_flux_ir<NV>(U, ir, GP, n, adiabatic, gamma, mu, k, gamma / ((gamma - 1) * Cp), Fv);
}

// EulerEvaluator.hpp:751-789 muEff: 0 constant, 1 Sutherland, 2 proportional to density
template <typename T>
DNDSB_HD T mu_eff(int model, real muGas, real TRef, real CSuth, T rho, T Temp)
{
    if (model == 0)
        return T(muGas);
    if (model == 1)
    {
        T TRel = Temp / TRef;
        return muGas * TRel * sqrt(TRel) * (TRef + CSuth) / (Temp + CSuth);
    }
    return muGas * rho;
}
} // namespace dndsb
