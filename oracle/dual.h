// CPU ORACLE — test infrastructure, not product code.
//
// First-order dual number in FP64 (value v, tangent d), the scalar type of the
// oracle's forward-mode derivative (or_dual_steps). Arithmetic is the chain
// rule of each operation; comparisons look at the value only, so every branch
// of the restated kernels takes the side its double instantiation takes.
// Math functions live in namespace sc with a double overload that calls
// <cmath> unchanged, so code templated on the scalar computes, for T = double,
// exactly what it computed before it was templated.
#ifndef ICEMPM_ORACLE_DUAL_H
#define ICEMPM_ORACLE_DUAL_H

#include <cmath>

struct Dual {
    double v, d;
    Dual(double x = 0.0) : v(x), d(0.0) {}
    Dual(double x, double t) : v(x), d(t) {}
    Dual& operator+=(const Dual& b) { d += b.d; v += b.v; return *this; }
    Dual& operator-=(const Dual& b) { d -= b.d; v -= b.v; return *this; }
    Dual& operator*=(const Dual& b) { d = d * b.v + v * b.d; v *= b.v; return *this; }
    Dual& operator/=(const Dual& b) { double q = v / b.v; d = (d - q * b.d) / b.v; v = q; return *this; }
};

inline Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(const Dual& a, const Dual& b) {
    double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
inline Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
inline Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
inline Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
inline Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
inline Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
inline Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
inline Dual operator/(double a, const Dual& b) { double q = a / b.v; return Dual(q, -q * b.d / b.v); }

#define ICEMPM_DUAL_CMP(op)                                                            \
    inline bool operator op(const Dual& a, const Dual& b) { return a.v op b.v; }      \
    inline bool operator op(const Dual& a, double b) { return a.v op b; }             \
    inline bool operator op(double a, const Dual& b) { return a op b.v; }
ICEMPM_DUAL_CMP(<)
ICEMPM_DUAL_CMP(>)
ICEMPM_DUAL_CMP(<=)
ICEMPM_DUAL_CMP(>=)
ICEMPM_DUAL_CMP(==)
ICEMPM_DUAL_CMP(!=)
#undef ICEMPM_DUAL_CMP

namespace sc {

inline double val(double x) { return x; }
inline double val(const Dual& x) { return x.v; }
inline float val(float x) { return x; }

inline double sqrt(double x) { return std::sqrt(x); }
inline float sqrt(float x) { return std::sqrt(x); }
// d sqrt(x) = dx / (2 sqrt x); at x = 0 the tangent is taken as 0 (the
// arguments that reach 0 here are sums of squares whose tangent is 0 there).
inline Dual sqrt(const Dual& x) {
    double r = std::sqrt(x.v);
    return Dual(r, r > 0 ? x.d / (2.0 * r) : 0.0);
}

inline double cbrt(double x) { return std::cbrt(x); }
inline Dual cbrt(const Dual& x) {
    double r = std::cbrt(x.v);
    return Dual(r, r != 0 ? x.d / (3.0 * r * r) : 0.0);
}

inline double pow(double x, double e) { return std::pow(x, e); }
inline Dual pow(const Dual& x, double e) {
    return Dual(std::pow(x.v, e), e * std::pow(x.v, e - 1.0) * x.d);
}

inline double fmin(double a, double b) { return std::fmin(a, b); }
inline Dual fmin(const Dual& a, const Dual& b) { return (b.v < a.v) ? b : a; }
inline double fmax(double a, double b) { return std::fmax(a, b); }
inline float fmax(float a, float b) { return std::fmax(a, b); }
inline Dual fmax(const Dual& a, const Dual& b) { return (b.v > a.v) ? b : a; }

}  // namespace sc

#endif
