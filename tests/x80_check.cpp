// Checks the integer emulation of x87 extended arithmetic (kbsrc_b200/csrc/x80.cuh) against the host's own x87
// long double: sums, differences, products and both float64 conversions, bit for bit, on random operands and on
// the edge cases of the format (ties, cancellation, alignment shifts past the window, denormals, the float64
// subnormal boundary, infinities and NaNs). Prints "cases N mismatches M" and exits non-zero on any mismatch.
// x86-64 only (long double is the x87 80-bit type there).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>

#include "x80.cuh"

using kbsrc::dev::x80;

static x80 to_x80(long double v) {
    unsigned char b[16] = {};
    std::memcpy(b, &v, 10);
    x80 r{};
    std::memcpy(&r.m, b, 8);
    r.se = b[8] | b[9] << 8;
    return r;
}
static long double from_x80(x80 a) {
    unsigned char b[16] = {};
    std::memcpy(b, &a.m, 8);
    b[8] = (unsigned char)(a.se & 255);
    b[9] = (unsigned char)(a.se >> 8 & 255);
    long double v;
    std::memcpy(&v, b, sizeof v);
    return v;
}
static bool same(x80 a, x80 b) { return a.m == b.m && (a.se & 0xffff) == (b.se & 0xffff); }

static long long cases = 0, bad = 0;
static void report(const char* what, x80 a, x80 b, x80 got, x80 want) {
    if (++bad <= 20)
        std::printf("%s: a=%04x:%016llx b=%04x:%016llx got %04x:%016llx want %04x:%016llx\n", what, a.se & 0xffff,
                    a.m, b.se & 0xffff, b.m, got.se & 0xffff, got.m, want.se & 0xffff, want.m);
}

static void check_pair(x80 a, x80 b) {
    const volatile long double la = from_x80(a), lb = from_x80(b);
    const long double s = la + lb, d = la - lb, p = la * lb;
    const x80 gs = kbsrc::dev::x80_add(a, b), gd = kbsrc::dev::x80_sub(a, b), gp = kbsrc::dev::x80_mul(a, b);
    cases += 3;
    if (!same(gs, to_x80(s))) report("add", a, b, gs, to_x80(s));
    if (!same(gd, to_x80(d))) report("sub", a, b, gd, to_x80(d));
    if (!same(gp, to_x80(p))) report("mul", a, b, gp, to_x80(p));
}

static void check_narrow(x80 a) {
    const volatile long double la = from_x80(a);
    const double want = (double)la, got = kbsrc::dev::x80_to_f64(a);
    cases++;
    if (std::memcmp(&want, &got, 8)) {
        if (++bad <= 20)
            std::printf("to_f64: a=%04x:%016llx got %a want %a\n", a.se & 0xffff, a.m, got, want);
    }
}

static void check_widen(double v) {
    const volatile double dv = v;
    const x80 want = to_x80((long double)dv), got = kbsrc::dev::x80_from_f64(v);
    cases++;
    if (!same(got, want)) report("from_f64", got, got, got, want);
}

int main() {
    std::mt19937_64 rng(20240601);
    auto u64 = [&] { return rng(); };
    auto rand_x80 = [&](int emin, int emax) {
        std::uniform_int_distribution<int> E(emin, emax);
        x80 r{};
        r.m = u64() | kbsrc::dev::kX80Top;
        r.se = E(rng) | (int)(u64() & 1) << 15;
        return r;
    };
    // random operands over a wide and a narrow exponent range
    for (int i = 0; i < 300000; i++) check_pair(rand_x80(16383 - 200, 16383 + 200), rand_x80(16383 - 200, 16383 + 200));
    for (int i = 0; i < 300000; i++) check_pair(rand_x80(16383 - 3, 16383 + 3), rand_x80(16383 - 3, 16383 + 3));
    // alignment shifts around the 64- and 128-bit window edges, with few-bit significands (ties) and full ones
    for (int d = 0; d < 140; d++)
        for (int k = 0; k < 400; k++) {
            x80 a = rand_x80(16383, 16383), b = a;
            b.se = (16383 - d) | (int)(u64() & 1) << 15;
            b.m = (k & 1) ? (u64() | kbsrc::dev::kX80Top) : (kbsrc::dev::kX80Top | (u64() & 7ull));
            if (k & 2) a.m = kbsrc::dev::kX80Top | (u64() & 3ull);
            if (k & 4) a.m = ~0ull;
            check_pair(a, b);
            check_pair(b, a);
        }
    // near-cancellation: b = a with a few low bits changed, opposite signs
    for (int k = 0; k < 200000; k++) {
        x80 a = rand_x80(16383 - 50, 16383 + 50), b = a;
        b.m ^= u64() & ((1ull << (k % 64)) - 1);
        b.m |= kbsrc::dev::kX80Top;
        if (k & 1) b.se ^= 1;
        b.se ^= 0x8000;
        check_pair(a, b);
    }
    // values built from float64 as the engine does: (LD)hi + (LD)lo, products of float64
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    for (int k = 0; k < 200000; k++) {
        const double h = U(rng) * std::ldexp(1.0, (int)(u64() % 80) - 40), l = h * 1e-17 * U(rng);
        const long double v = (long double)h + (long double)l;
        const x80 g = kbsrc::dev::x80_add(kbsrc::dev::x80_from_f64(h), kbsrc::dev::x80_from_f64(l));
        cases++;
        if (!same(g, to_x80(v))) report("from_dd", g, g, g, to_x80(v));
    }
    // denormal and near-denormal results of products and sums
    for (int k = 0; k < 200000; k++) check_pair(rand_x80(1, 80), rand_x80(16383 - 80, 16383 + 2));
    for (int k = 0; k < 100000; k++) check_pair(rand_x80(1, 3), rand_x80(1, 3));
    // widening: normal, subnormal, zero, infinity and NaN float64 values
    for (int k = 0; k < 200000; k++) {
        uint64_t b = u64();
        double v;
        std::memcpy(&v, &b, 8);
        if (v != v) continue;  // NaN payload handling of FLD is not compared here
        check_widen(v);
    }
    for (int k = 0; k < 100000; k++) {
        uint64_t b = u64() & ((1ull << 52) - 1) | (u64() & 1) << 63;  // subnormals
        double v;
        std::memcpy(&v, &b, 8);
        check_widen(v);
    }
    // narrowing: the normal range, the subnormal range and its lower edge, overflow, ties
    for (int k = 0; k < 300000; k++) check_narrow(rand_x80(16383 - 1080, 16383 + 1030));
    for (int k = 0; k < 300000; k++) check_narrow(rand_x80(16383 - 1090, 16383 - 1015));
    for (int k = 0; k < 100000; k++) {
        x80 a = rand_x80(16383 - 1080, 16383 + 1023);
        a.m = (a.m & ~0x7ffull) | 0x400ull;  // exactly half an ulp of a normal result
        check_narrow(a);
    }
    // infinities, NaNs and zeros as operands
    const x80 specials[] = {{0, 0, 0}, {0, 0x8000, 0}, {kbsrc::dev::kX80Top, 0x7fff, 0},
                            {kbsrc::dev::kX80Top, 0xffff, 0}, {0xC000000000000000ull, 0x7fff, 0},
                            {0xC000000000001234ull, 0xffff, 0}, {kbsrc::dev::kX80Top, 16383, 0},
                            {0xA000000000000000ull, 16383 | 0x8000, 0}};
    for (const x80& a : specials)
        for (const x80& b : specials) check_pair(a, b);
    for (const x80& a : specials) check_narrow(a);
    std::printf("cases %lld mismatches %lld\n", cases, bad);
    return bad ? 1 : 0;
}
