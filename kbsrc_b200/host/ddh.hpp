// Host double-double arithmetic for planning-time work: twiddle tables, kernel taps, Burg LPC.
//
// The results feed byte-identical output, so each operation keeps the reference's IEEE sequence
// (HongYue1/KBSRC src/dsp/double_double.hpp:59-135) and everything that includes this header is compiled
// with -ffp-contract=off. The exact product error uses std::fma (glibc's is correctly rounded), the only
// fused operation the reference performs.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace kbsrc::host {

struct dd {
    double hi = 0, lo = 0;
    constexpr dd() = default;
    constexpr dd(double h) : hi(h), lo(0) {}
    constexpr dd(double h, double l) : hi(h), lo(l) {}
};

inline dd quick_two_sum(double a, double b) {
    double s = a + b;
    return dd(s, b - (s - a));
}
inline dd two_sum(double a, double b) {
    double s = a + b, v = s - a;
    return dd(s, (a - (s - v)) + (b - v));
}
// accurate sum: both halves through two_sum, renormalised twice (double_double.hpp:67-70)
inline dd operator+(const dd& a, const dd& b) {
    dd h = two_sum(a.hi, b.hi), l = two_sum(a.lo, b.lo);
    h.lo = h.lo + l.hi;
    h = quick_two_sum(h.hi, h.lo);
    h.lo = h.lo + l.lo;
    return quick_two_sum(h.hi, h.lo);
}
inline dd operator-(const dd& a) { return dd(-a.hi, -a.lo); }
inline dd operator-(const dd& a, const dd& b) { return a + (-b); }
inline dd operator*(const dd& a, const dd& b) {
    double p = a.hi * b.hi, e = std::fma(a.hi, b.hi, -p);
    e = e + (a.hi * b.lo + a.lo * b.hi);
    return quick_two_sum(p, e);
}
inline dd operator*(const dd& a, double b) {
    double p = a.hi * b, e = std::fma(a.hi, b, -p);
    e = e + a.lo * b;
    return quick_two_sum(p, e);
}
// long division in three quotient digits (double_double.hpp:80-92)
inline dd operator/(const dd& a, double b) {
    double q1 = a.hi / b;
    dd r = a - dd(b) * q1;
    double q2 = r.hi / b;
    r = r - dd(b) * q2;
    double q3 = r.hi / b;
    return quick_two_sum(q1, q2) + dd(q3);
}
inline dd operator/(const dd& a, const dd& b) {
    double q1 = a.hi / b.hi;
    dd r = a - b * q1;
    double q2 = r.hi / b.hi;
    r = r - b * q2;
    double q3 = r.hi / b.hi;
    return quick_two_sum(q1, q2) + dd(q3);
}
inline dd sqrt_dd(const dd& a) {
    if (a.hi <= 0) return dd(0.0);
    double y = std::sqrt(a.hi);
    dd r = a - dd(y) * y;
    return quick_two_sum(y, r.hi / (2 * y));
}
// I0 by its power series, summed until the term drops below 1e-34 of the sum
inline dd bessel_i0(const dd& x) {
    const dd q = x * x / 4.0;
    dd term(1.0), sum(1.0);
    for (int k = 1; k < 2000; k++) {
        term = term * q / (double(k) * double(k));
        sum = sum + term;
        if (term.hi < sum.hi * 1e-34) break;
    }
    return sum;
}
constexpr dd kPi(3.141592653589793116e+00, 1.224646799147353207e-16);

// cos and sin of x in [0, pi/4] by Taylor series in dd
inline void sincos_reduced(const dd& x, dd& c, dd& s) {
    const dd x2 = x * x;
    dd ts = x, ss = x, tc(1.0), cc(1.0);
    for (int k = 1; k < 40; k++) {
        tc = -(tc * x2) / double((2 * k - 1) * (2 * k));
        cc = cc + tc;
        ts = -(ts * x2) / double((2 * k) * (2 * k + 1));
        ss = ss + ts;
        if (std::fabs(ts.hi) < 1e-40 && std::fabs(tc.hi) < 1e-40) break;
    }
    c = cc;
    s = ss;
}

// e^{+2 pi i k / n} = c + i s, with the angle reduced exactly to an octant by integer arithmetic
inline void unit_root(long long k, long long n, dd& c, dd& s) {
    k %= n;
    if (k < 0) k += n;
    const long long eighths = 8 * k, oct = eighths / n, rem = eighths - oct * n;
    const bool mirrored = oct & 1;
    long long quadrant = oct / 2;
    const dd phi = (dd(kPi.hi / 4, kPi.lo / 4) * double(mirrored ? n - rem : rem)) / double(n);
    dd cr, sr;
    sincos_reduced(phi, cr, sr);
    if (mirrored) {
        sr = -sr;
        quadrant += 1;
    }
    switch (quadrant & 3) {
        case 0: c = cr; s = sr; break;
        case 1: c = -sr; s = cr; break;
        case 2: c = -cr; s = -sr; break;
        default: c = sr; s = -cr; break;
    }
}

// Roots of unity e^{2 pi i k/n} for any k, each the dd product of a coarse and a fine table entry
// (the construction of the reference's CisTable, src/dsp/fft.hpp:29-43: the table values are part of the
// output definition).
class RootTable {
public:
    explicit RootTable(long long n) : n_(n) {
        step_ = (long long)std::ceil(std::sqrt((double)n));
        const long long coarse = n / step_ + 1;
        cc_.resize(coarse); cs_.resize(coarse); fc_.resize(step_); fs_.resize(step_);
        for (long long j = 0; j < coarse; j++) unit_root(j * step_, n, cc_[j], cs_[j]);
        for (long long l = 0; l < step_; l++) unit_root(l, n, fc_[l], fs_[l]);
    }
    void get(long long k, dd& c, dd& s) const {
        k %= n_;
        if (k < 0) k += n_;
        const long long j = k / step_, l = k % step_;
        if (l == 0) { c = cc_[j]; s = cs_[j]; return; }
        if (j == 0) { c = fc_[l]; s = fs_[l]; return; }
        c = cc_[j] * fc_[l] - cs_[j] * fs_[l];
        s = cc_[j] * fs_[l] + cs_[j] * fc_[l];
    }

private:
    long long n_, step_;
    std::vector<dd> cc_, cs_, fc_, fs_;
};

inline bool smooth7(long long n) {
    if (n < 1) return false;
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}

}  // namespace kbsrc::host
