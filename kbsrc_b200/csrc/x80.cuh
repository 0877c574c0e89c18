// x87 80-bit extended arithmetic in integers, for Precision::LongDouble on the GPU.
//
// The reference's LongDouble engine is run_engine<long double, long double, long double> (HongYue1/KBSRC
// src/resampler.cpp:214-215): every value is an x87 extended real (64-bit significand with an explicit integer
// bit, 15-bit exponent, bias 16383) and every +, -, * rounds once to 64 bits, to nearest-even (the x87 default
// precision and rounding control). The GPU has no such type, so x80 keeps the significand in a 64-bit integer
// and these functions reproduce the x87 result bit for bit: exact alignment into a 128-bit window with a sticky
// bit, normalisation, one round-to-nearest-even, gradual underflow below the normal range, infinities and NaNs
// after the x87 rules (a NaN operand is returned quieted, the larger significand when both are; invalid
// operations give the default NaN, negative with significand 0xC000...). Conversions from and to float64 are
// those of FLD / FST: exact widening, one rounding when narrowing (to the float64 subnormal grid where needed).
//
// The functions are __host__ __device__ so that a CPU test can compare them with the host's own x87 arithmetic.
#pragma once
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define KB_X80_FN __host__ __device__ __forceinline__
#else
#define KB_X80_FN inline
#endif

namespace kbsrc::dev {

struct alignas(16) x80 {
    unsigned long long m;  // significand; bit 63 is the integer bit (set for every normal value)
    int se;                // sign (bit 15) and biased exponent (bits 0-14); 0x7fff: infinity or NaN
    int pad;
};

constexpr unsigned long long kX80Top = 1ull << 63;
constexpr int kX80Bias = 16383;
constexpr int kX80Sign = 0x8000;
constexpr int kX80Inf = 0x7fff;

KB_X80_FN int x80_clz(unsigned long long v) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)v);
#else
    return v ? __builtin_clzll(v) : 64;
#endif
}

// High 64 bits of the 128-bit product
KB_X80_FN unsigned long long x80_mulhi(unsigned long long a, unsigned long long b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (unsigned long long)(((unsigned __int128)a * b) >> 64);
#endif
}

KB_X80_FN x80 x80_make(unsigned long long m, int se) { return x80{m, se, 0}; }
KB_X80_FN x80 x80_neg(x80 a) { return x80{a.m, a.se ^ kX80Sign, 0}; }

// Rounds the 128-bit significand h:l (h normalised, bit 63 set) with unbounded biased exponent e to the format:
// round to nearest-even at 64 bits, infinity on overflow, gradual underflow (denormal or zero) below exponent 1.
KB_X80_FN x80 x80_round(unsigned long long h, unsigned long long l, int e, int sign) {
    if (e <= 0) {  // below the normal range: shift right to exponent field 0 (value m * 2^(1-16383-63)) first
        const int sh = 1 - e;
        if (sh >= 128) {
            l = (h | l) ? 1ull : 0ull;
            h = 0;
        } else if (sh >= 64) {
            const unsigned long long lost = l | (sh > 64 ? h << (128 - sh) : 0ull);
            l = (sh == 64 ? h : h >> (sh - 64)) | (lost ? 1ull : 0ull);
            h = 0;
        } else {
            const unsigned long long lost = l << (64 - sh);
            l = (l >> sh) | (h << (64 - sh)) | (lost ? 1ull : 0ull);
            h >>= sh;
        }
        e = 0;
    }
    const bool rb = (l >> 63) != 0, st = (l << 1) != 0;
    if (rb && (st || (h & 1))) {
        h++;
        if (h == 0) {  // carried out of the significand
            h = kX80Top;
            e++;
        } else if (e == 0 && (h & kX80Top)) {  // a denormal rounded up into the normal range
            e = 1;
        }
    }
    if (e >= kX80Inf) return x80{kX80Top, sign | kX80Inf, 0};
    return x80{h, sign | e, 0};
}

// Operands with exponent 0x7fff (infinity, NaN) of a sum (mul = false) or product.
KB_X80_FN x80 x80_special(x80 a, x80 b, bool mul) {
    const bool an = (a.se & kX80Inf) == kX80Inf && (a.m << 1) != 0;
    const bool bn = (b.se & kX80Inf) == kX80Inf && (b.m << 1) != 0;
    const unsigned long long q = 1ull << 62;
    if (an && bn) {
        const unsigned long long ma = a.m & ~kX80Top, mb = b.m & ~kX80Top;
        const x80 r = ma > mb ? a : ma < mb ? b : (a.se & kX80Sign ? b : a);
        return x80{r.m | q, r.se, 0};
    }
    if (an) return x80{a.m | q, a.se, 0};
    if (bn) return x80{b.m | q, b.se, 0};
    const x80 indefinite{kX80Top | q, kX80Sign | kX80Inf, 0};
    const bool ai = (a.se & kX80Inf) == kX80Inf, bi = (b.se & kX80Inf) == kX80Inf;
    if (mul) {
        if ((ai && b.m == 0) || (bi && a.m == 0)) return indefinite;  // inf * 0
        return x80{kX80Top, ((a.se ^ b.se) & kX80Sign) | kX80Inf, 0};
    }
    if (ai && bi && ((a.se ^ b.se) & kX80Sign)) return indefinite;  // inf - inf
    return ai ? a : b;
}

// Exponent of a finite nonzero operand, normalising a denormal (significand without its integer bit)
KB_X80_FN int x80_unpack(x80& a) {
    const int e = a.se & kX80Inf;
    if (e != 0 || (a.m & kX80Top)) return e ? e : 1;
    const int lz = x80_clz(a.m);
    a.m <<= lz;
    return 1 - lz;
}

KB_X80_FN x80 x80_add(x80 a, x80 b) {
    if ((a.se & kX80Inf) == kX80Inf || (b.se & kX80Inf) == kX80Inf) return x80_special(a, b, false);
    if (b.m == 0) return a.m ? a : x80{0ull, a.se & b.se & kX80Sign, 0};
    if (a.m == 0) return b;
    int ea = x80_unpack(a), eb = x80_unpack(b);
    if (eb > ea || (eb == ea && b.m > a.m)) {  // |a| >= |b|
        const x80 t = a;
        a = b;
        b = t;
        const int te = ea;
        ea = eb;
        eb = te;
    }
    const int d = ea - eb, sign = a.se & kX80Sign;
    unsigned long long bh, bl;  // b aligned to a in a 128-bit window; bits below it folded into a sticky bit
    if (d == 0) {
        bh = b.m;
        bl = 0;
    } else if (d < 64) {
        bh = b.m >> d;
        bl = b.m << (64 - d);
    } else if (d == 64) {
        bh = 0;
        bl = b.m;
    } else if (d < 128) {
        bh = 0;
        bl = (b.m >> (d - 64)) | ((b.m << (128 - d)) ? 1ull : 0ull);
    } else {
        bh = 0;
        bl = 1;
    }
    unsigned long long h, l;
    int e = ea;
    if (((a.se ^ b.se) & kX80Sign) == 0) {
        l = bl;
        h = a.m + bh;
        if (h < a.m) {  // carry: shift the 65-bit sum right by one, keeping the lost bit as sticky
            l = (l >> 1) | (h << 63) | (l & 1);
            h = (h >> 1) | kX80Top;
            e++;
        }
    } else {
        l = 0ull - bl;
        h = a.m - bh - (bl ? 1ull : 0ull);
        if ((h | l) == 0) return x80{0ull, 0, 0};  // exact cancellation is +0 when rounding to nearest
        const int s = h ? x80_clz(h) : 64 + x80_clz(l);
        if (s >= 64) {
            h = l << (s - 64);
            l = 0;
        } else if (s > 0) {
            h = (h << s) | (l >> (64 - s));
            l <<= s;
        }
        e -= s;
    }
    return x80_round(h, l, e, sign);
}

// a - b; a NaN subtrahend keeps its sign (FSUB does not negate it)
KB_X80_FN x80 x80_sub(x80 a, x80 b) {
    if ((b.se & kX80Inf) == kX80Inf && (b.m << 1) != 0) return x80_special(a, b, false);
    return x80_add(a, x80_neg(b));
}

KB_X80_FN x80 x80_mul(x80 a, x80 b) {
    if ((a.se & kX80Inf) == kX80Inf || (b.se & kX80Inf) == kX80Inf) return x80_special(a, b, true);
    const int sign = (a.se ^ b.se) & kX80Sign;
    if (a.m == 0 || b.m == 0) return x80{0ull, sign, 0};
    const int ea = x80_unpack(a), eb = x80_unpack(b);
    unsigned long long h = x80_mulhi(a.m, b.m), l = a.m * b.m;
    int e = ea + eb - kX80Bias;
    if (h & kX80Top) {
        e++;
    } else {
        h = (h << 1) | (l >> 63);
        l <<= 1;
    }
    return x80_round(h, l, e, sign);
}

// float64 -> extended, exact (FLD m64fp; a signalling NaN is quieted)
KB_X80_FN x80 x80_from_f64(double v) {
    unsigned long long u;
    memcpy(&u, &v, 8);
    const int sign = (int)(u >> 48) & kX80Sign;
    const int ex = (int)(u >> 52) & 0x7ff;
    const unsigned long long f = u & ((1ull << 52) - 1);
    if (ex == 0x7ff) return x80{f ? (kX80Top | (1ull << 62) | (f << 11)) : kX80Top, sign | kX80Inf, 0};
    if (ex == 0) {
        if (f == 0) return x80{0ull, sign, 0};
        const int lz = x80_clz(f);
        return x80{f << lz, sign | (kX80Bias - 1011 - lz), 0};
    }
    return x80{(f | (1ull << 52)) << 11, sign | (ex - 1023 + kX80Bias), 0};
}

// extended -> float64, rounded to nearest-even once (FST m64fp)
KB_X80_FN double x80_to_f64(x80 a) {
    unsigned long long sign = (unsigned long long)(a.se & kX80Sign) << 48, u;
    const int e = a.se & kX80Inf;
    double r;
    if (e == kX80Inf) {
        u = sign | (0x7ffull << 52) | ((a.m << 1) ? ((a.m >> 11) & ((1ull << 52) - 1)) : 0ull);
        memcpy(&r, &u, 8);
        return r;
    }
    if (a.m == 0) {
        memcpy(&r, &sign, 8);
        return r;
    }
    int E = x80_unpack(a) - kX80Bias;  // value = (m / 2^63) * 2^E
    if (E > 1023) {
        u = sign | (0x7ffull << 52);
        memcpy(&r, &u, 8);
        return r;
    }
    // keep the bits of the float64 grid at this magnitude: 53 for a normal result, fewer for a subnormal one
    const int shift = E >= -1022 ? 11 : 11 + (-1022 - E);
    unsigned long long mant, rem, half;
    if (shift >= 65) {
        mant = 0;
        rem = 1;  // below half of the smallest subnormal: rounds to zero
        half = 2;
    } else if (shift == 64) {
        mant = 0;
        rem = a.m;
        half = kX80Top;
    } else {
        mant = a.m >> shift;
        rem = a.m & ((1ull << shift) - 1);
        half = 1ull << (shift - 1);
    }
    if (shift >= 65) {
        mant = 0;
    } else if (rem > half || (rem == half && (mant & 1))) {
        mant++;
    }
    if (E >= -1022) {
        if (mant >> 53) {  // rounded up to the next binade
            mant >>= 1;
            E++;
            if (E > 1023) {
                u = sign | (0x7ffull << 52);
                memcpy(&r, &u, 8);
                return r;
            }
        }
        u = sign | ((unsigned long long)(E + 1023) << 52) | (mant & ((1ull << 52) - 1));
    } else {
        u = sign | mant;  // a subnormal; mant == 2^52 is the smallest normal, encoded by the same bits
    }
    memcpy(&r, &u, 8);
    return r;
}

}  // namespace kbsrc::dev
