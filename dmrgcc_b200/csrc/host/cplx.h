// Complex scalar for the one-time host algebra of complex MPO tensors.  The
// arithmetic follows the reference's Complex (src/tensor/complex.h:112-250)
// formula for formula (a product as ac - bd, ad + bc; a quotient through
// 1 / |z|^2; Norm as sqrt(re^2 + im^2)), so that the MPO it builds rounds as
// the reference's does.  Layout: (re, im) doubles, like the reference's Complex
// and cuDoubleComplex.
#pragma once

#include <cmath>

namespace dmrg {

struct Cplx {
    double re = 0.0, im = 0.0;
    Cplx() = default;
    Cplx(double r) : re(r), im(0.0) {}  // NOLINT: implicit, as the reference's Complex(double)
    Cplx(double r, double i) : re(r), im(i) {}
    Cplx& operator+=(const Cplx& z) {
        re += z.re;
        im += z.im;
        return *this;
    }
};
static_assert(sizeof(Cplx) == 2 * sizeof(double), "Cplx is two doubles");

inline Cplx operator*(const Cplx& a, const Cplx& b) { return Cplx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline Cplx operator*(const Cplx& z, double r) { return Cplx(z.re * r, z.im * r); }
inline Cplx operator*(double r, const Cplx& z) { return Cplx(z.re * r, z.im * r); }
inline Cplx operator/(const Cplx& a, const Cplx& b) {
    const double k = 1.0 / (b.re * b.re + b.im * b.im);
    return Cplx((a.re * b.re + a.im * b.im) * k, (a.im * b.re - a.re * b.im) * k);
}
inline Cplx operator-(const Cplx& a, const Cplx& b) { return Cplx(a.re - b.re, a.im - b.im); }
inline bool operator==(const Cplx& a, const Cplx& b) { return a.re == b.re && a.im == b.im; }
inline bool operator!=(const Cplx& a, const Cplx& b) { return !(a == b); }
inline double norm_of(const Cplx& z) { return std::sqrt(z.re * z.re + z.im * z.im); }
inline double norm_of(double x) { return std::fabs(x); }
inline Cplx conj_of(const Cplx& z) { return Cplx(z.re, -z.im); }
inline Cplx phase_of(double theta) { return Cplx(std::cos(theta), std::sin(theta)); }
inline double real_of(double x) { return x; }
inline double real_of(const Cplx& z) { return z.re; }
inline double imag_of(double) { return 0.0; }
inline double imag_of(const Cplx& z) { return z.im; }

}  // namespace dmrg
