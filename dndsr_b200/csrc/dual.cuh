// Forward-mode dual numbers: a value and N directional derivatives.  The gas,
// Riemann and boundary routines are templated on their scalar type, so
// instantiating them on Dual<N> yields N columns of their Jacobian in one pass
// (JVP, and the local Jacobian blocks the adjoint kernels transpose).
// Comparisons and min/max act on values, so branches follow the primal path.
#pragma once
#include "platform.cuh"
#include <math.h>

namespace dndsb
{
// keep the plain-real overloads visible next to the Dual ones below
using ::exp;
using ::fabs;
using ::isfinite;
using ::log;
using ::pow;
using ::sqrt;
using ::tanh;

template <int N>
struct Dual
{
    real v;
    real d[N];
    DNDSB_HD Dual() : v(0)
    {
        for (int i = 0; i < N; i++)
            d[i] = 0;
    }
    DNDSB_HD Dual(real x) : v(x)
    {
        for (int i = 0; i < N; i++)
            d[i] = 0;
    }
    // the k-th independent variable with value x
    DNDSB_HD static Dual var(real x, int k)
    {
        Dual r(x);
        if (k >= 0 && k < N)
            r.d[k] = 1;
        return r;
    }
    DNDSB_HD Dual &operator+=(const Dual &b)
    {
        v += b.v;
        for (int i = 0; i < N; i++)
            d[i] += b.d[i];
        return *this;
    }
    DNDSB_HD Dual &operator-=(const Dual &b)
    {
        v -= b.v;
        for (int i = 0; i < N; i++)
            d[i] -= b.d[i];
        return *this;
    }
    DNDSB_HD Dual &operator*=(const Dual &b)
    {
        for (int i = 0; i < N; i++)
            d[i] = d[i] * b.v + v * b.d[i];
        v *= b.v;
        return *this;
    }
};

template <int N>
DNDSB_HD Dual<N> operator+(Dual<N> a, const Dual<N> &b) { return a += b; }
template <int N>
DNDSB_HD Dual<N> operator-(Dual<N> a, const Dual<N> &b) { return a -= b; }
template <int N>
DNDSB_HD Dual<N> operator-(const Dual<N> &a)
{
    Dual<N> r;
    r.v = -a.v;
    for (int i = 0; i < N; i++)
        r.d[i] = -a.d[i];
    return r;
}
template <int N>
DNDSB_HD Dual<N> operator*(const Dual<N> &a, const Dual<N> &b)
{
    Dual<N> r;
    r.v = a.v * b.v;
    for (int i = 0; i < N; i++)
        r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
DNDSB_HD Dual<N> operator/(const Dual<N> &a, const Dual<N> &b)
{
    Dual<N> r;
    real ib = 1.0 / b.v;
    r.v = a.v * ib;
    for (int i = 0; i < N; i++)
        r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
// mixed operations with plain reals
template <int N>
DNDSB_HD Dual<N> operator+(Dual<N> a, real b)
{
    a.v += b;
    return a;
}
template <int N>
DNDSB_HD Dual<N> operator+(real b, Dual<N> a)
{
    a.v += b;
    return a;
}
template <int N>
DNDSB_HD Dual<N> operator-(Dual<N> a, real b)
{
    a.v -= b;
    return a;
}
template <int N>
DNDSB_HD Dual<N> operator-(real b, const Dual<N> &a)
{
    Dual<N> r = -a;
    r.v += b;
    return r;
}
template <int N>
DNDSB_HD Dual<N> operator*(Dual<N> a, real b)
{
    a.v *= b;
    for (int i = 0; i < N; i++)
        a.d[i] *= b;
    return a;
}
template <int N>
DNDSB_HD Dual<N> operator*(real b, Dual<N> a) { return a * b; }
template <int N>
DNDSB_HD Dual<N> operator/(Dual<N> a, real b) { return a * (1.0 / b); }
template <int N>
DNDSB_HD Dual<N> operator/(real a, const Dual<N> &b)
{
    Dual<N> r;
    r.v = a / b.v;
    real s = -r.v / b.v;
    for (int i = 0; i < N; i++)
        r.d[i] = s * b.d[i];
    return r;
}
template <int N>
DNDSB_HD bool operator<(const Dual<N> &a, const Dual<N> &b) { return a.v < b.v; }
template <int N>
DNDSB_HD bool operator>(const Dual<N> &a, const Dual<N> &b) { return a.v > b.v; }
template <int N>
DNDSB_HD bool operator<=(const Dual<N> &a, const Dual<N> &b) { return a.v <= b.v; }
template <int N>
DNDSB_HD bool operator>=(const Dual<N> &a, const Dual<N> &b) { return a.v >= b.v; }
template <int N>
DNDSB_HD bool operator<(const Dual<N> &a, real b) { return a.v < b; }
template <int N>
DNDSB_HD bool operator>(const Dual<N> &a, real b) { return a.v > b; }
template <int N>
DNDSB_HD bool operator<=(const Dual<N> &a, real b) { return a.v <= b; }
template <int N>
DNDSB_HD bool operator>=(const Dual<N> &a, real b) { return a.v >= b; }
template <int N>
DNDSB_HD bool operator<(real a, const Dual<N> &b) { return a < b.v; }
template <int N>
DNDSB_HD bool operator>(real a, const Dual<N> &b) { return a > b.v; }
template <int N>
DNDSB_HD bool operator<=(real a, const Dual<N> &b) { return a <= b.v; }
template <int N>
DNDSB_HD bool operator>=(real a, const Dual<N> &b) { return a >= b.v; }

template <int N>
DNDSB_HD Dual<N> sqrt(const Dual<N> &a)
{
    Dual<N> r;
    r.v = ::sqrt(a.v);
    real s = r.v > 0 ? 0.5 / r.v : 0.0;
    for (int i = 0; i < N; i++)
        r.d[i] = s * a.d[i];
    return r;
}
template <int N>
DNDSB_HD Dual<N> fabs(const Dual<N> &a) { return a.v >= 0 ? a : -a; }
// a^e for a real exponent: d(a^e) = e a^(e-1) da (zero derivative at a = 0)
template <int N>
DNDSB_HD Dual<N> pow(const Dual<N> &a, real e)
{
    Dual<N> r;
    r.v = ::pow(a.v, e);
    real s = a.v != 0 ? e * r.v / a.v : 0.0;
    for (int i = 0; i < N; i++)
        r.d[i] = s * a.d[i];
    return r;
}
template <int N>
DNDSB_HD bool isfinite(const Dual<N> &a) { return ::isfinite(a.v); }
// the elementary functions of the SA model
template <int N>
DNDSB_HD Dual<N> exp(const Dual<N> &a)
{
    Dual<N> r;
    r.v = ::exp(a.v);
    for (int i = 0; i < N; i++)
        r.d[i] = r.v * a.d[i];
    return r;
}
template <int N>
DNDSB_HD Dual<N> log(const Dual<N> &a)
{
    Dual<N> r;
    r.v = ::log(a.v);
    real s = 1.0 / a.v;
    for (int i = 0; i < N; i++)
        r.d[i] = s * a.d[i];
    return r;
}
template <int N>
DNDSB_HD Dual<N> tanh(const Dual<N> &a)
{
    Dual<N> r;
    r.v = ::tanh(a.v);
    real s = 1.0 - r.v * r.v;
    for (int i = 0; i < N; i++)
        r.d[i] = s * a.d[i];
    return r;
}

template <int N>
DNDSB_HD Dual<N> dmax(const Dual<N> &a, const Dual<N> &b) { return a.v > b.v ? a : b; }
template <int N>
DNDSB_HD Dual<N> dmin(const Dual<N> &a, const Dual<N> &b) { return a.v < b.v ? a : b; }
template <int N>
DNDSB_HD Dual<N> dmax(const Dual<N> &a, real b) { return a.v > b ? a : Dual<N>(b); }
template <int N>
DNDSB_HD Dual<N> dmax(real a, const Dual<N> &b) { return a > b.v ? Dual<N>(a) : b; }
template <int N>
DNDSB_HD Dual<N> dmin(const Dual<N> &a, real b) { return a.v < b ? a : Dual<N>(b); }
template <int N>
DNDSB_HD Dual<N> dmin(real a, const Dual<N> &b) { return a < b.v ? Dual<N>(a) : b; }

// value of a real or a dual number
DNDSB_HD real value_of(real x) { return x; }
template <int N>
DNDSB_HD real value_of(const Dual<N> &x) { return x.v; }
} // namespace dndsb
