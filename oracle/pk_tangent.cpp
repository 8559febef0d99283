/*
 * pk_tangent.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * The tangent-linear (forward-mode) oracle: pk_oracle.c compiled once more
 * with every double replaced by a dual number (value, derivative).  The value
 * part runs exactly the oracle's operations in the oracle's order (same
 * flags: -O2 -ffp-contract=off, no OpenMP), so its branch decisions -- which
 * limiter case, which wave region, which floor -- are those of the oracle and
 * therefore of the CUDA path, which matches the oracle bit for bit.  The
 * derivative part carries J v for a seed direction v through the same
 * branches.  A dot product <w, J v> from here against <J^T w, v> from the
 * CUDA adjoint checks the adjoint to rounding, kinks or not, where central
 * differences cannot.
 *
 * Derivative rules: sum, difference, product and quotient rules; sqrt, exp;
 * fabs and copysign differentiate the side their sign test takes (at an
 * exact zero the positive side); min/max (f_min, f_max in the oracle) pass
 * the derivative of the selected argument; comparisons use values only.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <cstring>
#include <type_traits>

struct pk_dual {
    double v, d;
    pk_dual() : v(0.0), d(0.0) {}
    template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>
    pk_dual(T x) : v((double)x), d(0.0) {}
    pk_dual(double x, double dx) : v(x), d(dx) {}
};

static inline pk_dual operator+(const pk_dual& a, const pk_dual& b) { return pk_dual(a.v + b.v, a.d + b.d); }
static inline pk_dual operator-(const pk_dual& a, const pk_dual& b) { return pk_dual(a.v - b.v, a.d - b.d); }
static inline pk_dual operator*(const pk_dual& a, const pk_dual& b)
{
    return pk_dual(a.v * b.v, a.d * b.v + a.v * b.d);
}
static inline pk_dual operator/(const pk_dual& a, const pk_dual& b)
{
    const double q = a.v / b.v;
    return pk_dual(q, (a.d - q * b.d) / b.v);
}
static inline pk_dual operator-(const pk_dual& a) { return pk_dual(-a.v, -a.d); }
static inline pk_dual& operator+=(pk_dual& a, const pk_dual& b) { return a = a + b; }
static inline pk_dual& operator-=(pk_dual& a, const pk_dual& b) { return a = a - b; }
static inline pk_dual& operator*=(pk_dual& a, const pk_dual& b) { return a = a * b; }
static inline pk_dual& operator/=(pk_dual& a, const pk_dual& b) { return a = a / b; }
static inline bool operator<(const pk_dual& a, const pk_dual& b) { return a.v < b.v; }
static inline bool operator>(const pk_dual& a, const pk_dual& b) { return a.v > b.v; }
static inline bool operator<=(const pk_dual& a, const pk_dual& b) { return a.v <= b.v; }
static inline bool operator>=(const pk_dual& a, const pk_dual& b) { return a.v >= b.v; }
static inline bool operator==(const pk_dual& a, const pk_dual& b) { return a.v == b.v; }
static inline bool operator!=(const pk_dual& a, const pk_dual& b) { return a.v != b.v; }
static inline pk_dual sqrt(const pk_dual& a)
{
    const double r = std::sqrt(a.v);
    return pk_dual(r, r > 0.0 ? a.d / (2.0 * r) : 0.0);
}
static inline pk_dual exp(const pk_dual& a)
{
    const double e = std::exp(a.v);
    return pk_dual(e, e * a.d);
}
static inline pk_dual fabs(const pk_dual& a) { return pk_dual(std::fabs(a.v), std::signbit(a.v) ? -a.d : a.d); }
static inline pk_dual copysign(const pk_dual& a, const pk_dual& b)
{
    const double r = std::copysign(a.v, b.v);
    return pk_dual(r, (std::signbit(a.v) != std::signbit(b.v)) ? -a.d : a.d);
}

#define double pk_dual
#include "pk_oracle.c"
#undef double

/* seeds: every pk_dual argument is laid out as two doubles (value, derivative);
 * the ctypes front end (oracle/tangent.py) builds the structures accordingly */
extern "C" int t_dual_size(void) { return (int)sizeof(pk_dual); }
