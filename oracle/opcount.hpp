// Operation-counting scalar for the op-counting build of the oracle (test infrastructure).
//
// Compiled in only with -DORC_OPCOUNT (oracle/Makefile target liboracle_opcount.so): the oracle's
// `real` becomes this wrapper of a double, which counts every floating-point operation the
// restated algorithm performs -- +, -, *, / and sqrt one each, exp / pow / log / trigonometric
// functions one call each -- so that F_alg, the algorithmic flops per cell of an operator, is
// measured on the reference's algorithm rather than on the GPU code.  Comparisons, abs, min and
// max are not counted.  Values are computed in FP64 exactly as in the plain build.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <initializer_list>

namespace orc_cnt
{
struct Counter
{
    uint64_t add = 0, mul = 0, div = 0, sqrt = 0, fn = 0;
};
inline Counter &ctr()
{
    static Counter c; // the counting build runs single-threaded
    return c;
}

struct R
{
    double v;
    R() = default;
    constexpr R(double x) : v(x) {}
    explicit operator double() const { return v; }
    R &operator+=(R o) { ctr().add++, v += o.v; return *this; }
    R &operator-=(R o) { ctr().add++, v -= o.v; return *this; }
    R &operator*=(R o) { ctr().mul++, v *= o.v; return *this; }
    R &operator/=(R o) { ctr().div++, v /= o.v; return *this; }
    R operator-() const { return R(-v); }
    R operator+() const { return *this; }
};
inline R operator+(R a, R b) { ctr().add++; return R(a.v + b.v); }
inline R operator-(R a, R b) { ctr().add++; return R(a.v - b.v); }
inline R operator*(R a, R b) { ctr().mul++; return R(a.v * b.v); }
inline R operator/(R a, R b) { ctr().div++; return R(a.v / b.v); }
inline bool operator<(R a, R b) { return a.v < b.v; }
inline bool operator>(R a, R b) { return a.v > b.v; }
inline bool operator<=(R a, R b) { return a.v <= b.v; }
inline bool operator>=(R a, R b) { return a.v >= b.v; }
inline bool operator==(R a, R b) { return a.v == b.v; }
inline bool operator!=(R a, R b) { return a.v != b.v; }
inline R sqrt(R a) { ctr().sqrt++; return R(std::sqrt(a.v)); }
inline R abs(R a) { return R(std::fabs(a.v)); }
inline R exp(R a) { ctr().fn++; return R(std::exp(a.v)); }
inline R log(R a) { ctr().fn++; return R(std::log(a.v)); }
inline R pow(R a, R b) { ctr().fn++; return R(std::pow(a.v, b.v)); }
inline R cos(R a) { ctr().fn++; return R(std::cos(a.v)); }
inline R sin(R a) { ctr().fn++; return R(std::sin(a.v)); }
inline R tanh(R a) { ctr().fn++; return R(std::tanh(a.v)); }
inline R floor(R a) { return R(std::floor(a.v)); }
inline R round(R a) { return R(std::round(a.v)); }
inline bool isfinite(R a) { return std::isfinite(a.v); }
inline R max(R a, R b) { return a.v < b.v ? b : a; }
inline R min(R a, R b) { return b.v < a.v ? b : a; }
inline R max(std::initializer_list<R> l) { return *std::max_element(l.begin(), l.end(), [](R a, R b) { return a.v < b.v; }); }
inline R min(std::initializer_list<R> l) { return *std::min_element(l.begin(), l.end(), [](R a, R b) { return a.v < b.v; }); }
} // namespace orc_cnt
